// Flattening of an optimized Tree into evaluation tapes.
//
// Two forms are produced from the same walk:
//
//  * SlotTape: the reference's own layout (libfive/src/eval/deck.cpp:19-94):
//    one slot id per node, clauses stored root-first with the root at slot 1,
//    X/Y/Z/constant/variable slots outside the clause list.  It is exported
//    through the C ABI so that the CPU oracle can evaluate exactly the
//    reference's tape, and so that slot numbering can be checked against the
//    reference's own unit tests.
//
//  * RegTape: the device layout.  Clauses are in evaluation order
//    (leaves first) and their results live in a small register file
//    allocated by liveness (linear scan, lowest free register first), so a
//    GPU thread needs n_regs floats of scratch instead of one per node.
//    Constants and free variables are operands read from a constant pool.
//    X, Y, Z are registers 0, 1, 2.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "tree.hpp"

namespace lfb {

struct SlotClause {
    int32_t op;
    uint32_t id;
    uint32_t a;
    uint32_t b;
};

struct SlotTape {
    std::vector<SlotClause> clauses;                 // root first
    std::vector<std::pair<uint32_t, float>> constants;
    std::vector<std::pair<uint32_t, const Node*>> vars;  // ascending slot id
    uint32_t X = 0, Y = 0, Z = 0;
    uint32_t num_clauses = 0;
    uint32_t root = 1;
};

// Operand kinds packed two bits per operand in RegClause::kinds.
enum : uint8_t {
    OPND_REG = 0,
    OPND_CONST = 1,   // index into the constant pool
    OPND_VAR = 2,     // index into the constant pool (a free variable)
};


struct RegClause {
    uint8_t op;
    uint8_t kinds;   // bits 0-1: kind of a, bits 2-3: kind of b
    uint16_t out;
    uint16_t a;
    uint16_t b;
};
static_assert(sizeof(RegClause) == 8, "RegClause must pack into 8 bytes");

struct RegTape {
    std::vector<RegClause> clauses;   // evaluation order
    std::vector<float> cpool;         // constants, then variables
    uint32_t n_const = 0;
    uint32_t n_vars = 0;
    uint32_t n_regs = 3;              // includes X, Y, Z
    uint8_t root_kind = OPND_REG;
    uint16_t root = 0;
    uint32_t n_choices = 0;           // min / max clauses
    std::vector<const Node*> var_nodes;   // variable i <-> tree node
    std::vector<uint32_t> var_slots;      // variable i <-> SlotTape slot
};

/// Builds the reference-layout tape; returns false (with a message) when the
/// tree holds something the device path cannot evaluate (oracles, invalid
/// nodes, unflattened remaps).
bool build_slot_tape(const Tree& root, SlotTape& out, std::string* err);

/// Derives the register-allocated device tape from a slot tape.
bool build_reg_tape(const SlotTape& st, RegTape& out, std::string* err);

/// One clause of a register tape in dependency-level form, as an entry of a
/// list sorted by level.  Operands name value slots instead of registers:
/// slots 0-2 hold X, Y, Z and slot 3 + k the result of the list's entry k,
/// so the entries of one level are independent.  Constant / variable
/// operands keep their pool index.  `head` packs op (bits 0-7), operand
/// kinds (8-11), pruning state (12-13: WIDE_BOTH, WIDE_A = copy of operand
/// a, WIDE_B = copy of operand b) and the level (14-31, clauses start at
/// level 1); `c` is the clause's index in the register tape.
struct WideEntry {
    uint32_t head;
    uint32_t a;
    uint32_t b;
    uint32_t c;
};
static_assert(sizeof(WideEntry) == 16, "WideEntry must pack into 16 bytes");

enum : uint32_t { WIDE_BOTH = 1, WIDE_A = 2, WIDE_B = 3 };
constexpr uint32_t kWideLevelShift = 14;
constexpr uint32_t kWideMaxLevel = (1u << (32 - kWideLevelShift)) - 1;

/// The register tape's clauses sorted by level (stable within a level), all
/// in state WIDE_BOTH, plus the list slot (or pool index) of the root.  Fails for
/// tapes whose dependency chain is longer than kWideMaxLevel.
bool build_wide_list(const RegTape& t, std::vector<WideEntry>& out,
                     uint32_t& root_slot, std::string* err);

}  // namespace lfb
