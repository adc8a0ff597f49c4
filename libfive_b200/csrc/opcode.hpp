// Opcode numbering and metadata for libfive expression trees.
//
// The numeric values are part of libfive's on-disk and C API contract
// (libfive/include/libfive/tree/opcode.hpp:23-59, the unpacked layout), so
// they are kept identical: a caller that passes `libfive_opcode_enum("min")`
// to `libfive_tree_binary` gets the same node here as in the reference.
#pragma once
#include <cstdint>
#include <string>

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

/// Number of arguments (0, 1, 2) or -1 for INVALID / LAST_OP
/// (reference: libfive/src/tree/opcode.cpp:18-65).
int arity(int op);

/// Upper-case enum name without the OP_ prefix, e.g. "NTH_ROOT".
const char* enum_name(int op);

/// Scheme-style name: lower case, '_' replaced by '-', e.g. "nth-root"
/// (reference: opcode.cpp:91-106).
std::string scm_name(int op);

/// Inverse of scm_name, case-insensitive; INVALID when unknown
/// (reference: opcode.cpp:108-125).
int from_scm_name(const std::string& s);

/// Operator spelling used by the tree printer ("+", "min", "x", ...)
/// (reference: opcode.cpp:127-176).
std::string op_string(int op);

bool is_commutative(int op);   // ADD, MUL, MIN, MAX
bool is_idempotent(int op);    // MIN, MAX

}  // namespace op
}  // namespace lfb
