// Device-side building blocks of the dual-contouring mesher.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "dc_tables.hpp"
#include "dev_ops.cuh"
#include "qef.h"

namespace lfb {

constexpr int kMaxLevels = 24;

enum : uint8_t {
    CELL_EMPTY = 0,
    CELL_FILLED = 1,
    CELL_LEAF = 2,     // ambiguous cell without children (has a record)
    CELL_BRANCH = 3,   // ambiguous cell with eight children
};

// Status bits reported by the kernels.
enum : uint32_t {
    ST_ARENA_OVERFLOW = 1u << 0,
    ST_RECORD_OVERFLOW = 1u << 1,
    ST_QUEUE_OVERFLOW = 1u << 2,
    ST_FEATURE_OVERFLOW = 1u << 3,
    ST_REGS = 1u << 4,
    ST_LIST_OVERFLOW = 1u << 5,
    // which feature-evaluator capacity ST_FEATURE_OVERFLOW ran into
    ST_FEAT_EPS = 1u << 6,    // epsilon directions of one feature
    ST_FEAT_LIST = 1u << 7,   // features of one register
    ST_FEAT_TMP = 1u << 8,    // candidate features of one clause
    ST_EDGE_OVERFLOW = 1u << 9,   // leaf edge records
};

/// A level-ordered clause list (WideEntry) in a list arena, with the list
/// slot of the tape's root (or its pool index when the root is a constant).
struct ListRef {
    uint32_t off;
    uint32_t len;
    uint32_t root;
    uint32_t pad;
};

struct TapeRef {
    uint32_t off;     // first clause in the arena
    uint32_t len;     // clauses
    uint32_t nregs;   // registers the tape uses (X, Y, Z included)
    uint32_t root;    // root operand: index | kind << 16
};

__host__ __device__ inline TapeRef root_tape_ref(const DevTape& bt)
{
    return {0u, bt.n, bt.n_regs, static_cast<uint32_t>(bt.root) |
                                     (static_cast<uint32_t>(bt.root_kind) << 16)};
}

/// The device tape with the register count and root of a pruned tape.
__host__ __device__ inline DevTape with_tape(const DevTape& bt, const TapeRef& tr)
{
    DevTape t = bt;
    t.n_regs = tr.nregs;
    t.root = static_cast<uint16_t>(tr.root & 0xffff);
    t.root_kind = static_cast<uint8_t>(tr.root >> 16);
    return t;
}

/// Per-leaf data: DCLeaf (libfive/include/libfive/render/brep/dc/dc_tree.hpp:34-89).
struct LeafRec {
    double vert[4][3];
    double mass[4];
    double ata[6];
    double atb[3];
    double btb;
    int32_t level;
    uint8_t corner_mask;
    uint8_t vertex_count;
    uint8_t rank;
    uint8_t manifold;
};

/// Views of one octree depth.
struct LevelView {
    uint32_t n_cells;
    uint64_t* coords;        // x | y << 21 | z << 42 at this depth
    uint8_t* type;
    int32_t* rec;
    int32_t* child_group;    // group index at depth + 1 (branch cells)
    TapeRef* cell_tape;      // tape valid in this cell (given to children)
    uint32_t n_groups;       // groups of 8 cells at this depth (depth > 0)
    uint32_t* group_parent;  // cell index at depth - 1
    TapeRef* group_tape;
    ListRef* cell_list;      // level-ordered form of cell_tape
    ListRef* group_list;
};

struct Octree {
    double lo[3], hi[3];     // root region
    int levels;              // L: leaves at depth L
    LevelView lv[kMaxLevels + 1];
};

__device__ __forceinline__ uint64_t pack_coords(uint32_t x, uint32_t y, uint32_t z)
{
    return static_cast<uint64_t>(x) | (static_cast<uint64_t>(y) << 21) |
           (static_cast<uint64_t>(z) << 42);
}

__device__ __forceinline__ void unpack_coords(uint64_t c, uint32_t& x,
                                              uint32_t& y, uint32_t& z)
{
    x = static_cast<uint32_t>(c & 0x1fffff);
    y = static_cast<uint32_t>((c >> 21) & 0x1fffff);
    z = static_cast<uint32_t>((c >> 42) & 0x1fffff);
}

/// Region bounds of a cell, computed by the same chain of midpoint splits as
/// Region::subdivide (region.hpp:89-114) so that shared faces of neighbouring
/// cells have bit-identical coordinates.
__device__ __forceinline__ void cell_bounds(const Octree& o, int depth,
                                            uint64_t c, double lo[3],
                                            double hi[3])
{
    uint32_t idx[3];
    unpack_coords(c, idx[0], idx[1], idx[2]);
    for (int a = 0; a < 3; ++a) {
        double l = o.lo[a], h = o.hi[a];
        for (int b = depth - 1; b >= 0; --b) {
            const double m = (l + h) / 2;
            if ((idx[a] >> b) & 1) l = m; else h = m;
        }
        lo[a] = l;
        hi[a] = h;
    }
}

}  // namespace lfb
