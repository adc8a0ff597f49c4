// CPU oracle: TEST INFRASTRUCTURE ONLY.
//
// A plain C++ restatement of libfive's CPU evaluators and dual-contouring
// mesher, used by tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline to check the GPU library.  Nothing in libfive_b200/ links or
// calls this code.
//
// It evaluates the reference-layout slot tape (Deck, libfive/src/eval/
// deck.cpp:19-94) exported by lfb_tree_slot_tape, one slot per node, in
// batches of 256 points exactly like the reference evaluators:
//   values     eval_array.cpp:106-118, 221-369
//   derivs     eval_deriv_array.cpp:101-117, 119-256
//   intervals  eval_interval.cpp:68-93, 189-294 + interval.hpp:31-442, with
//              Boost.Interval's rounded arithmetic restated via fesetround
//              (the reference's rounded_transc_std policy calls the C library
//              under FE_DOWNWARD / FE_UPWARD, as done here)
//   features   eval_feature.cpp:56-372 + feature.cpp:14-284
//   jacobian   eval_jacobian.cpp:49-115
//   mesher     worker_pool.inl, dc_tree.inl, dc_tree3.cpp, dual.hpp,
//              dc_mesher.cpp, marching.cpp (see oracle_dc.cpp)
//
// Parity pins: the known-answer values of libfive/test/eval_array.cpp,
// eval_deriv_array.cpp, eval_interval.cpp, eval_jacobian.cpp, api.cpp,
// xtree.cpp and mesh.cpp are restated in tests/golden/ and checked against
// this oracle in tests/test_oracle_golden.py.
#pragma once
#include <cstdint>
#include <memory>
#include <vector>

namespace ora {

struct Clause {
    int op;
    uint32_t id, a, b;
};

struct Tape {
    std::vector<Clause> t;   // root first; evaluated back to front
    uint32_t root = 1;
    uint32_t X = 0, Y = 0, Z = 0;
    uint32_t num_clauses = 0;
    std::vector<std::pair<uint32_t, float>> constants;
    std::vector<std::pair<uint32_t, float>> vars;   // slot, value
    // Interval-push bookkeeping (Tape::push / getBase, tape.cpp:23-209)
    int type = 0;            // 0 base, 1 interval, 2 specialized
    bool terminal = false;
    float bx[2] = {0, 0}, by[2] = {0, 0}, bz[2] = {0, 0};
    const Tape* parent = nullptr;
    std::shared_ptr<const Tape> parent_keep;
};

enum Keep { KEEP_BOTH, KEEP_A, KEEP_B, KEEP_ALWAYS };

}  // namespace ora
