// Opcode numbering and metadata for libfive expression trees.
//
// The numeric values are part of libfive's on-disk and C API contract
// (libfive/include/libfive/tree/opcode.hpp:23-59, the unpacked layout), so
// they are kept identical: a caller that passes `libfive_opcode_enum("min")`
// to `libfive_tree_binary` gets the same node here as in the reference.
#pragma once
#include <cstdint>
#include <string>

#include "opcode_ids.h"

namespace lfb {
namespace op {

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
