// Opcode numbers (no dependencies, so that run-time compiled kernels can
// include it too).  The values are part of libfive's on-disk and C API
// contract (libfive/include/libfive/tree/opcode.hpp:23-59, the unpacked
// layout), so they are kept identical.
#pragma once

namespace lfb {
namespace op {

enum Opcode : int {
    INVALID = 0,
    CONSTANT = 1,
    VAR_X = 2,
    VAR_Y = 3,
    VAR_Z = 4,
    VAR_FREE = 5,
    CONST_VAR = 6,
    SQUARE = 7,
    SQRT = 8,
    NEG = 9,
    SIN = 10,
    COS = 11,
    TAN = 12,
    ASIN = 13,
    ACOS = 14,
    ATAN = 15,
    EXP = 16,
    ADD = 17,
    MUL = 18,
    MIN = 19,
    MAX = 20,
    SUB = 21,
    DIV = 22,
    ATAN2 = 23,
    POW = 24,
    NTH_ROOT = 25,
    MOD = 26,
    NANFILL = 27,
    ABS = 28,
    RECIP = 29,
    LOG = 30,
    COMPARE = 31,
    ORACLE = 32,
    LAST_OP = 33,
};

}  // namespace op

/// Extra opcode used only inside pruned device tapes: out = a.
enum : unsigned char { OP_COPY = 40 };

}  // namespace lfb
