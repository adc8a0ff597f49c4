// Breadth-first dual contouring on the GPU.
//
// The reference builds its octree depth-first with a CPU thread pool
// (WorkerPool::run, libfive/src/render/brep/worker_pool.inl:93-255) and walks
// the dual grid with another pool (Dual<3>::walk, dual.hpp:126-385).  Here
// every stage is a level-synchronous pass over compacted arrays:
//
//   1. k_interval_level   (once per depth d < L)
//        DCTree::evalInterval (dc_tree.inl:94-128): interval-evaluate every
//        cell of depth d with the tape of its parent, classify it
//        EMPTY / FILLED / AMBIGUOUS, and prune the tape for its children
//        (Tape::push, tape.cpp:23-160) as a backward liveness pass over the
//        register tape; decided min/max clauses become register copies.
//   2. k_leaf_groups      (depth L)
//        DCTree::evalLeaf (dc_tree.inl:131-552) for the eight children of
//        each ambiguous depth L-1 cell, one warp per sibling group: the 27
//        shared corners, the crossing edges of the 3x3x3 lattice (each
//        searched once), the QEFs and the per-patch vertices.
//   3. k_collapse_level   (depths L-1 .. 0)
//        DCTree::collectChildren (dc_tree.inl:581-735).
//   4. k_dual_round       (until no task is left)
//        Dual<3>::work / face3 / edge3 as a breadth-first task expansion and
//        DCMesher::load (dc_mesher.cpp:18-169) at minimal edges.
//
// Every numeric decision uses the same float32 / float64 operations as the
// reference's scalar code, so the octree and the mesh are reproducible.
#include <cub/cub.cuh>

#include "dc_device.cuh"
#include "dc_features.cuh"

namespace lfb {

__constant__ DcTables c_tab;

////////////////////////////////////////////////////////////////////////////////
// 1. Interval classification and tape pruning

__device__ __forceinline__ Iv iv_fetch(uint8_t kind, uint16_t idx,
                                       const float* L, const float* H,
                                       const uint8_t* N, int tid, int B,
                                       const float* __restrict__ cp)
{
    if (kind == OPND_REG) {
        return {L[idx * B + tid], H[idx * B + tid], N[idx * B + tid] != 0};
    }
    const float v = __ldg(cp + idx);
    return iv_make(v, v);
}

__global__ void __launch_bounds__(128)
k_interval_level(Octree o, int d, DevTape bt, RegClause* arena,
                 uint32_t* arena_top, uint32_t arena_cap, uint8_t* dec,
                 uint32_t* status)
{
    extern __shared__ float smem[];
    const int B = blockDim.x;
    const int tid = threadIdx.x;
    float* L = smem;
    float* H = smem + bt.n_regs * B;
    uint8_t* N = reinterpret_cast<uint8_t*>(smem + 2 * bt.n_regs * B);

    const LevelView& lv = o.lv[d];
    const uint32_t i = blockIdx.x * B + tid;
    if (i >= lv.n_cells) return;

    TapeRef tr;
    uint64_t dec_base;
    if (d == 0) {
        tr = {0u, bt.n, bt.n_choices, 0u};
        dec_base = 0;
    } else {
        tr = lv.group_tape[i >> 3];
        dec_base = lv.group_dec[i >> 3] + static_cast<uint64_t>(i & 7) * tr.nch;
    }

    double blo[3], bhi[3];
    cell_bounds(o, d, lv.coords[i], blo, bhi);
    for (int a = 0; a < 3; ++a) {
        const Iv v = iv_make(static_cast<float>(blo[a]), static_cast<float>(bhi[a]));
        L[a * B + tid] = v.lo;
        H[a * B + tid] = v.hi;
        N[a * B + tid] = v.nan;
    }

    // Forward interval pass, recording the push decision of every min/max
    // (IntervalEvaluator::push, eval_interval.cpp:116-167).
    const RegClause* cl = arena + tr.off;
    bool changed = false;
    uint32_t ch = 0;
    for (uint32_t c = 0; c < tr.len; ++c) {
        const uint2 raw = *reinterpret_cast<const uint2*>(cl + c);
        const uint8_t op_ = raw.x & 0xff;
        const uint8_t kinds = (raw.x >> 8) & 0xff;
        const uint16_t ro = raw.x >> 16;
        const Iv a = iv_fetch(kinds & 3, raw.y & 0xffff, L, H, N, tid, B, bt.cpool);
        const Iv b = iv_fetch((kinds >> 2) & 3, raw.y >> 16, L, H, N, tid, B, bt.cpool);
        const Iv r = iv_apply(op_, a, b);
        if (op_ == op::MIN || op_ == op::MAX) {
            uint8_t keep = 0;   // 0 both, 1 a, 2 b
            if (a.lo > b.hi) keep = (op_ == op::MAX) ? 1 : 2;
            else if (b.lo > a.hi) keep = (op_ == op::MAX) ? 2 : 1;
            changed |= keep != 0;
            dec[dec_base + ch++] = keep;
        }
        L[ro * B + tid] = r.lo;
        H[ro * B + tid] = r.hi;
        N[ro * B + tid] = r.nan;
    }
    const Iv root = iv_fetch(bt.root_kind, bt.root, L, H, N, tid, B, bt.cpool);
    const uint8_t state = iv_state(root);
    lv.type[i] = state == ST_EMPTY ? CELL_EMPTY
               : state == ST_FILLED ? CELL_FILLED : CELL_BRANCH;
    if (state != ST_AMBIGUOUS) {
        return;
    }
    // NaN-unsafe results keep the unpruned tape (dc_tree.inl:107-111).
    if (root.nan || !changed) {
        lv.cell_tape[i] = tr;
        return;
    }

    // Backward liveness pass over the register tape: N now marks registers
    // whose value is still needed.  Count first, then allocate and write.
    uint32_t kept = 0, kept_ch = 0;
    for (int pass = 0; pass < 2; ++pass) {
        for (uint32_t r = 0; r < bt.n_regs; ++r) N[r * B + tid] = 0;
        if (bt.root_kind == OPND_REG) N[bt.root * B + tid] = 1;
        uint32_t out_pos = kept;
        uint32_t chi = ch;
        uint32_t off = 0;
        if (pass == 1) {
            off = atomicAdd(arena_top, kept);
            if (off + kept > arena_cap || off + kept < off) {
                atomicOr(status, ST_ARENA_OVERFLOW);
                lv.cell_tape[i] = tr;
                return;
            }
        }
        for (int64_t c = static_cast<int64_t>(tr.len) - 1; c >= 0; --c) {
            const uint2 raw = *reinterpret_cast<const uint2*>(cl + c);
            const uint8_t op_ = raw.x & 0xff;
            const uint8_t kinds = (raw.x >> 8) & 0xff;
            const uint16_t ro = raw.x >> 16;
            const bool is_choice = (op_ == op::MIN || op_ == op::MAX);
            uint8_t keep = 0;
            if (is_choice) keep = dec[dec_base + (--chi)];
            if (!N[ro * B + tid]) continue;
            N[ro * B + tid] = 0;
            RegClause outc;
            bool emit = true;
            if (keep) {
                const uint8_t k = keep == 1 ? (kinds & 3) : ((kinds >> 2) & 3);
                const uint16_t src = keep == 1 ? (raw.y & 0xffff) : (raw.y >> 16);
                if (k == OPND_REG) {
                    N[src * B + tid] = 1;
                    emit = (src != ro);
                }
                outc.op = OP_COPY;
                outc.kinds = k;
                outc.out = ro;
                outc.a = src;
                outc.b = 0;
            } else {
                if ((kinds & 3) == OPND_REG) N[(raw.y & 0xffff) * B + tid] = 1;
                if (dev_is_binary(op_) && ((kinds >> 2) & 3) == OPND_REG) {
                    N[(raw.y >> 16) * B + tid] = 1;
                }
                *reinterpret_cast<uint2*>(&outc) = raw;
            }
            if (!emit) continue;
            if (pass == 0) {
                ++kept;
                if (is_choice && !keep) ++kept_ch;
            } else {
                arena[off + (--out_pos)] = outc;
            }
        }
        if (pass == 1) {
            lv.cell_tape[i] = {off, kept, kept_ch, 0u};
        }
    }
}

////////////////////////////////////////////////////////////////////////////////
// 2. Leaves: one warp per group of eight sibling cells

struct EdgeSlot {
    double t0[3], t1[3];   // current search bracket: inside, outside
    Qef q;
    float g0[4], g1[4];    // gradient + value at t0 / t1
    int32_t rank;
    uint8_t lat;           // lattice edge id
    uint8_t exists;        // received at least one sample
    uint8_t amb[2];        // tied min/max at t0 / t1
};

struct LeafWarpShared {
    FeatureScratch fs;
    EdgeSlot e[54];
    int8_t slot_of[54];    // lattice edge -> slot, -1 if not crossing
    uint8_t st[27];        // corner states (CELL_EMPTY / CELL_FILLED)
    int32_t rec[8];
    uint8_t nslots;
};

__device__ __forceinline__ float warp_fetch_v(uint8_t kind, uint16_t idx,
                                              const float* R, int lane,
                                              const float* __restrict__ cp)
{
    return kind == OPND_REG ? R[idx * 32 + lane] : __ldg(cp + idx);
}

/// Value of the tape at (x, y, z) for this lane, plus whether any min/max
/// saw equal arguments (ArrayEvaluator::getAmbiguous, eval_array.cpp:197-217).
__device__ float warp_value(const DevTape& bt, const RegClause* cl,
                            uint32_t len, float* R, int lane, float x,
                            float y, float z, bool* ambig, uint64_t* evals,
                            bool active = true)
{
    R[0 * 32 + lane] = x;
    R[1 * 32 + lane] = y;
    R[2 * 32 + lane] = z;
    bool amb = false;
    for (uint32_t c = 0; c < len; ++c) {
        const uint2 raw = __ldg(reinterpret_cast<const uint2*>(cl + c));
        const uint8_t o = raw.x & 0xff;
        const uint8_t kinds = (raw.x >> 8) & 0xff;
        const float a = warp_fetch_v(kinds & 3, raw.y & 0xffff, R, lane, bt.cpool);
        const float b = warp_fetch_v((kinds >> 2) & 3, raw.y >> 16, R, lane, bt.cpool);
        if (o == op::MIN || o == op::MAX) amb |= (a == b);
        R[(raw.x >> 16) * 32 + lane] = dv_value(o, a, b);
    }
    if (ambig) *ambig = amb;
    const uint32_t act = __ballot_sync(0xffffffffu, active);
    if (evals && lane == 0) *evals += static_cast<uint64_t>(__popc(act)) * len;
    return warp_fetch_v(bt.root_kind, bt.root, R, lane, bt.cpool);
}

__device__ __forceinline__ D4 warp_fetch_d(uint8_t kind, uint16_t idx,
                                           const float* R, int lane,
                                           const float* __restrict__ cp)
{
    if (kind == OPND_REG) {
        const float* r = R + idx * 128 + lane;
        return {r[0], r[32], r[64], r[96]};
    }
    return {__ldg(cp + idx), 0.0f, 0.0f, 0.0f};
}

__device__ D4 warp_deriv(const DevTape& bt, const RegClause* cl, uint32_t len,
                         float* R, int lane, float x, float y, float z,
                         bool* ambig, uint64_t* evals, bool active = true)
{
    const float in[3] = {x, y, z};
    for (int a = 0; a < 3; ++a) {
        float* r = R + a * 128 + lane;
        r[0] = in[a];
        r[32] = a == 0 ? 1.0f : 0.0f;
        r[64] = a == 1 ? 1.0f : 0.0f;
        r[96] = a == 2 ? 1.0f : 0.0f;
    }
    bool amb = false;
    for (uint32_t c = 0; c < len; ++c) {
        const uint2 raw = __ldg(reinterpret_cast<const uint2*>(cl + c));
        const uint8_t o = raw.x & 0xff;
        const uint8_t kinds = (raw.x >> 8) & 0xff;
        const D4 a = warp_fetch_d(kinds & 3, raw.y & 0xffff, R, lane, bt.cpool);
        const D4 b = warp_fetch_d((kinds >> 2) & 3, raw.y >> 16, R, lane, bt.cpool);
        if (o == op::MIN || o == op::MAX) amb |= (a.v == b.v);
        const D4 r = dv_deriv(o, a, b, false);
        float* out = R + (raw.x >> 16) * 128 + lane;
        out[0] = r.v; out[32] = r.dx; out[64] = r.dy; out[96] = r.dz;
    }
    if (ambig) *ambig = amb;
    const uint32_t act = __ballot_sync(0xffffffffu, active);
    if (evals && lane == 0) *evals += static_cast<uint64_t>(__popc(act)) * len;
    return warp_fetch_d(bt.root_kind, bt.root, R, lane, bt.cpool);
}

struct LeafArgs {
    Octree o;
    DevTape bt;
    const RegClause* arena;
    LeafRec* recs;
    uint32_t* rec_top;
    uint32_t rec_cap;
    uint32_t* status;
    unsigned long long* evals;
};

__global__ void __launch_bounds__(128)
k_leaf_groups(LeafArgs A, uint32_t n_groups)
{
    extern __shared__ __align__(16) unsigned char lsmem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    LeafWarpShared* S = reinterpret_cast<LeafWarpShared*>(lsmem) + warp;
    float* R = reinterpret_cast<float*>(reinterpret_cast<LeafWarpShared*>(lsmem) + wpb) +
               static_cast<size_t>(warp) * A.bt.n_regs * 128;
    const uint32_t g = blockIdx.x * wpb + warp;
    if (g >= n_groups) return;

    const Octree& o = A.o;
    const int Ld = o.levels;
    const bool single = (Ld == 0);       // the root itself is the only leaf
    const int n = single ? 2 : 3;        // lattice points per axis
    const int ncell = single ? 1 : 8;

    // Lattice coordinates along each axis (double), from the parent region
    // split at its centre exactly like Region::subdivide.
    double lat[3][3];
    TapeRef tr;
    uint64_t base_coords;
    if (single) {
        for (int a = 0; a < 3; ++a) {
            lat[a][0] = o.lo[a];
            lat[a][1] = o.hi[a];
        }
        tr = {0u, A.bt.n, A.bt.n_choices, 0u};
        base_coords = 0;
    } else {
        const LevelView& lv = o.lv[Ld];
        const uint32_t parent = lv.group_parent[g];
        const uint64_t pc = o.lv[Ld - 1].coords[parent];
        double plo[3], phi[3];
        cell_bounds(o, Ld - 1, pc, plo, phi);
        for (int a = 0; a < 3; ++a) {
            lat[a][0] = plo[a];
            lat[a][1] = (plo[a] + phi[a]) / 2;
            lat[a][2] = phi[a];
        }
        tr = lv.group_tape[g];
        base_coords = pc;
    }
    const RegClause* cl = A.arena + tr.off;
    uint64_t my_evals = 0, my_devals = 0;
    const FeatCtx fc{R, &S->fs, A.status};

    // --- corners (dc_tree.inl:156-239) ---------------------------------
    const int npts = n * n * n;
    float cv = 0.0f;
    bool camb = false;
    float px = 0, py = 0, pz = 0;
    if (lane < npts) {
        const int ia = lane % n, ib = (lane / n) % n, ic = lane / (n * n);
        px = static_cast<float>(lat[0][ia]);
        py = static_cast<float>(lat[1][ib]);
        pz = static_cast<float>(lat[2][ic]);
    }
    cv = warp_value(A.bt, cl, tr.len, R, lane, px, py, pz, &camb, &my_evals,
                    lane < npts);
    uint8_t cst = CELL_EMPTY;
    bool need_d = false, need_f = false;
    if (lane < npts) {
        if (cv > 0 || cv != cv) cst = CELL_EMPTY;
        else if (cv < 0) cst = CELL_FILLED;
        else if (!camb) need_d = true;
        else need_f = true;
    }
    if (__any_sync(0xffffffffu, need_d)) {
        const D4 d = warp_deriv(A.bt, cl, tr.len, R, lane, px, py, pz, nullptr,
                                &my_devals, need_d);
        if (need_d) {
            cst = (d.dx != 0 || d.dy != 0 || d.dz != 0) ? CELL_FILLED : CELL_EMPTY;
        }
    }
    {
        uint32_t pending = __ballot_sync(0xffffffffu, need_f);
        while (pending) {
            const int src = __ffs(pending) - 1;
            pending &= pending - 1;
            const float qx = __shfl_sync(0xffffffffu, px, src);
            const float qy = __shfl_sync(0xffffffffu, py, src);
            const float qz = __shfl_sync(0xffffffffu, pz, src);
            const bool inside = dev_is_inside(fc, A.bt, cl, tr.len, qx, qy, qz, lane);
            if (lane == src) cst = inside ? CELL_FILLED : CELL_EMPTY;
        }
    }
    if (lane < npts) S->st[lane] = cst;
    __syncwarp();

    // --- cell classification --------------------------------------------
    auto lat_pt = [&](int cell, int corner) {
        const int cx = cell & 1, cy = (cell >> 1) & 1, cz = (cell >> 2) & 1;
        return (cx + (corner & 1)) + n * ((cy + ((corner >> 1) & 1)) +
                                          n * (cz + ((corner >> 2) & 1)));
    };
    const LevelView& lvL = o.lv[Ld];
    if (lane < ncell) {
        uint8_t mask = 0;
        for (int k = 0; k < 8; ++k) {
            mask |= (S->st[lat_pt(lane, k)] == CELL_FILLED ? 1 : 0) << k;
        }
        const uint32_t ci = single ? 0 : (g * 8 + lane);
        int32_t rec = -1;
        uint8_t type = mask == 0 ? CELL_EMPTY : mask == 0xff ? CELL_FILLED : CELL_LEAF;
        if (type == CELL_LEAF) {
            const uint32_t r = atomicAdd(A.rec_top, 1u);
            if (r >= A.rec_cap) {
                atomicOr(A.status, ST_RECORD_OVERFLOW);
            } else {
                rec = static_cast<int32_t>(r);
                LeafRec& L = A.recs[r];
                L.corner_mask = mask;
                L.manifold = c_tab.manifold[mask];
                L.vertex_count = c_tab.npatch[mask];
                L.level = 0;
                L.rank = 0;
            }
        }
        lvL.type[ci] = type;
        lvL.rec[ci] = rec;
        S->rec[lane] = rec;
    }

    // --- crossing lattice edges -----------------------------------------
    const int seg = n - 1;
    const int n_lat_edges = 3 * seg * n * n;
    auto lat_edge_ends = [&](int e, int& p0, int& p1) {
        const int ax = e / (seg * n * n);
        const int r = e % (seg * n * n);
        const int s = r % seg;
        const int u = (r / seg) % n;
        const int w = r / (seg * n);
        int c0[3], c1[3];
        if (ax == 0) { c0[0] = s; c0[1] = u; c0[2] = w; }
        else if (ax == 1) { c0[1] = s; c0[0] = u; c0[2] = w; }
        else { c0[2] = s; c0[0] = u; c0[1] = w; }
        c1[0] = c0[0]; c1[1] = c0[1]; c1[2] = c0[2];
        c1[ax] += 1;
        p0 = c0[0] + n * (c0[1] + n * c0[2]);
        p1 = c1[0] + n * (c1[1] + n * c1[2]);
    };
    auto pt_pos = [&](int p, double out[3]) {
        out[0] = lat[0][p % n];
        out[1] = lat[1][(p / n) % n];
        out[2] = lat[2][p / (n * n)];
    };
    if (lane == 0) S->nslots = 0;
    __syncwarp();
    for (int base = 0; base < n_lat_edges; base += 32) {
        const int e = base + lane;
        bool crossing = false;
        int p0 = 0, p1 = 0;
        if (e < n_lat_edges) {
            lat_edge_ends(e, p0, p1);
            crossing = S->st[p0] != S->st[p1];
        }
        const uint32_t m = __ballot_sync(0xffffffffu, crossing);
        const int before = __popc(m & ((1u << lane) - 1));
        const int first_slot = S->nslots;
        if (e < n_lat_edges) {
            S->slot_of[e] = crossing ? static_cast<int8_t>(first_slot + before) : -1;
        }
        if (crossing) {
            EdgeSlot& es = S->e[first_slot + before];
            const bool f0 = S->st[p0] == CELL_FILLED;
            double a[3], b[3];
            pt_pos(f0 ? p0 : p1, a);
            pt_pos(f0 ? p1 : p0, b);
            for (int k = 0; k < 3; ++k) { es.t0[k] = a[k]; es.t1[k] = b[k]; }
            es.lat = static_cast<uint8_t>(e);
            es.exists = 0;
            qef_zero(es.q);
        }
        __syncwarp();
        if (lane == 0) S->nslots = static_cast<uint8_t>(first_slot + __popc(m));
        __syncwarp();
    }
    const int E = S->nslots;

    // --- edge search: 4 rounds of 16 points (dc_tree.inl:326-410) -------
    for (int round = 0; round < 4; ++round) {
        for (int base = 0; base < E; base += 2) {
            const int slot = base + (lane >> 4);
            const int j = lane & 15;
            const bool active = slot < E;
            double q[3] = {0, 0, 0};
            if (active) {
                const double frac = j / (16 - 1.0);
                const EdgeSlot& es = S->e[slot];
                for (int k = 0; k < 3; ++k) {
                    q[k] = es.t0[k] * (1 - frac) + es.t1[k] * frac;
                }
            }
            const float v = warp_value(A.bt, cl, tr.len, R, lane,
                                       static_cast<float>(q[0]),
                                       static_cast<float>(q[1]),
                                       static_cast<float>(q[2]), nullptr,
                                       &my_evals, active);
            // A sample exactly on the surface is resolved with
            // FeatureEvaluator::isInside: for a point without tied min/max
            // that is "gradient is non-zero" (one feature), otherwise the
            // full feature search.
            const bool zero = active && j >= 1 && v == 0;
            bool inside = true;
            if (__any_sync(0xffffffffu, zero)) {
                bool amb = false;
                const D4 dg = warp_deriv(A.bt, cl, tr.len, R, lane, static_cast<float>(q[0]),
                                         static_cast<float>(q[1]), static_cast<float>(q[2]),
                                         &amb, &my_devals, zero);
                if (zero && !amb) {
                    const float g[3] = {dg.dx, dg.dy, dg.dz};
                    inside = sqrtf(fdot(g, g)) > 0;
                }
                uint32_t full = __ballot_sync(0xffffffffu, zero && amb);
                while (full) {
                    const int src = __ffs(full) - 1;
                    full &= full - 1;
                    const float zx = __shfl_sync(0xffffffffu, static_cast<float>(q[0]), src);
                    const float zy = __shfl_sync(0xffffffffu, static_cast<float>(q[1]), src);
                    const float zz = __shfl_sync(0xffffffffu, static_cast<float>(q[2]), src);
                    const bool in = dev_is_inside(fc, A.bt, cl, tr.len, zx, zy, zz, lane);
                    if (lane == src) inside = in;
                }
            }
            // dc_tree.inl:372-407: the bracket ends at the first sample that
            // is outside (value > 0, or an exact zero that is not inside);
            // failing that, at the last sample unless it is an inside zero.
            const uint32_t term = __ballot_sync(0xffffffffu,
                active && j >= 1 && (v > 0 || (v == 0 && !inside)));
            const uint32_t last_ok = __ballot_sync(0xffffffffu,
                active && j == 15 && !(v > 0) && !(v == 0));
            for (int h = 0; h < 2; ++h) {
                const int s = base + h;
                if (s >= E) break;
                const uint32_t ht = (term >> (16 * h)) & 0xffff;
                int pick = -1;
                if (ht) pick = __ffs(ht) - 1;
                else if ((last_ok >> (16 * h + 15)) & 1) pick = 15;
                if (pick > 0) {
                    const int lo_lane = 16 * h + pick - 1, hi_lane = 16 * h + pick;
                    double nt0[3], nt1[3];
                    for (int k = 0; k < 3; ++k) {
                        nt0[k] = __shfl_sync(0xffffffffu, q[k], lo_lane);
                        nt1[k] = __shfl_sync(0xffffffffu, q[k], hi_lane);
                    }
                    if (lane == 0) {
                        EdgeSlot& es = S->e[s];
                        for (int k = 0; k < 3; ++k) { es.t0[k] = nt0[k]; es.t1[k] = nt1[k]; }
                    }
                }
                __syncwarp();
            }
        }
    }

    // --- gradients at the bracket ends and QEFs (dc_tree.inl:412-471) ---
    for (int base = 0; base < 2 * E; base += 32) {
        const int p = base + lane;
        const bool active = p < 2 * E;
        double q[3] = {0, 0, 0};
        if (active) {
            const EdgeSlot& es = S->e[p >> 1];
            for (int k = 0; k < 3; ++k) q[k] = (p & 1) ? es.t1[k] : es.t0[k];
        }
        bool amb = false;
        const D4 d = warp_deriv(A.bt, cl, tr.len, R, lane, static_cast<float>(q[0]),
                                static_cast<float>(q[1]), static_cast<float>(q[2]),
                                &amb, &my_devals, active);
        if (active) {
            EdgeSlot& es = S->e[p >> 1];
            float* g = (p & 1) ? es.g1 : es.g0;
            g[0] = d.dx; g[1] = d.dy; g[2] = d.dz; g[3] = d.v;
            es.amb[p & 1] = amb;
        }
    }
    __syncwarp();
    // Samples are pushed inside end first, then outside end; edges are
    // independent, so each lane owns whole edges.  Points where a min/max
    // is tied use every feature gradient instead (eval_feature.cpp:125-169).
    const uint32_t any_amb = __ballot_sync(0xffffffffu, [&] {
        bool a = false;
        for (int s = lane; s < E; s += 32) a |= S->e[s].amb[0] || S->e[s].amb[1];
        return a;
    }());
    if (!any_amb) {
        for (int s = lane; s < E; s += 32) {
            EdgeSlot& es = S->e[s];
            for (int side = 0; side < 2; ++side) {
                const float* g = side ? es.g1 : es.g0;
                const double* pos = side ? es.t1 : es.t0;
                const double gd[3] = {g[0], g[1], g[2]};
                qef_push(es.q, pos, gd, static_cast<double>(g[3]));
            }
            es.exists = 1;
        }
    } else {
        for (int s = 0; s < E; ++s) {
            EdgeSlot& es = S->e[s];
            for (int side = 0; side < 2; ++side) {
                const float* g = side ? es.g1 : es.g0;
                const double* pos = side ? es.t1 : es.t0;
                if (es.amb[side]) {
                    dev_push_features(fc, A.bt, cl, tr.len, pos,
                                      static_cast<double>(g[3]), &es.q,
                                      &es.exists, lane);
                } else if (lane == 0) {
                    const double gd[3] = {g[0], g[1], g[2]};
                    qef_push(es.q, pos, gd, static_cast<double>(g[3]));
                    es.exists = 1;
                }
                __syncwarp();
            }
        }
    }
    __syncwarp();
    for (int s = lane; s < E; s += 32) {
        S->e[s].rank = qef_rank(S->e[s].q);
    }
    __syncwarp();

    // --- vertices: one lane per (cell, patch) (dc_tree.inl:474-549) -----
    {
        const int cell = lane >> 2, patch = lane & 3;
        if (cell < ncell && S->rec[cell] >= 0) {
            LeafRec& L = A.recs[S->rec[cell]];
            const uint8_t mask = L.corner_mask;
            if (patch < c_tab.npatch[mask]) {
                const int ne = c_tab.nedge[mask][patch];
                int slots[12];
                for (int k = 0; k < ne; ++k) {
                    const int ca = c_tab.v[mask][patch][k][0];
                    const int cb = c_tab.v[mask][patch][k][1];
                    // lattice edge between the two corners of this cell
                    const int pa = lat_pt(cell, ca), pb = lat_pt(cell, cb);
                    const int lo_p = pa < pb ? pa : pb;
                    const int diff = (pa < pb ? pb - pa : pa - pb);
                    const int ax = diff == 1 ? 0 : diff == n ? 1 : 2;
                    const int c0 = lo_p % n, c1 = (lo_p / n) % n, c2 = lo_p / (n * n);
                    int le;
                    if (ax == 0) le = c0 + seg * (c1 + n * c2);
                    else if (ax == 1) le = c1 + seg * (c0 + n * c2);
                    else le = c2 + seg * (c0 + n * c1);
                    le += ax * seg * n * n;
                    slots[k] = S->slot_of[le];
                }
                int max_rank = 0;
                for (int k = 0; k < ne; ++k) {
                    if (slots[k] >= 0 && S->e[slots[k]].exists &&
                        S->e[slots[k]].rank > max_rank) {
                        max_rank = S->e[slots[k]].rank;
                    }
                }
                Qef q;
                qef_zero(q);
                for (int k = 0; k < ne; ++k) {
                    if (slots[k] < 0 || !S->e[slots[k]].exists) continue;
                    const EdgeSlot& es = S->e[slots[k]];
                    if (es.rank == max_rank) {
                        q.mass[0] += es.q.mass[0] / es.q.mass[3];
                        q.mass[1] += es.q.mass[1] / es.q.mass[3];
                        q.mass[2] += es.q.mass[2] / es.q.mass[3];
                        q.mass[3] += 1.0;
                    }
                }
                for (int k = 0; k < ne; ++k) {
                    if (slots[k] < 0 || !S->e[slots[k]].exists) continue;
                    qef_add(q, S->e[slots[k]].q);
                }
                double v[3];
                int rank = 0;
                qef_vertex(q, v, &rank);
                for (int k = 0; k < 3; ++k) L.vert[patch][k] = v[k];
                if (patch == c_tab.npatch[mask] - 1) {
                    for (int k = 0; k < 4; ++k) L.mass[k] = q.mass[k];
                    for (int k = 0; k < 6; ++k) L.ata[k] = q.ata[k];
                    for (int k = 0; k < 3; ++k) L.atb[k] = q.atb[k];
                    L.btb = q.btb;
                    L.rank = static_cast<uint8_t>(rank);
                }
            }
        }
    }
    if (lane == 0) {
        atomicAdd(A.evals, static_cast<unsigned long long>(my_evals));
        atomicAdd(A.evals + 1, static_cast<unsigned long long>(my_devals));
    }
    (void)base_coords;
}

}  // namespace lfb

namespace lfb {

////////////////////////////////////////////////////////////////////////////////
// 3. Bottom-up collapse (DCTree::collectChildren, dc_tree.inl:581-735)

struct CollapseArgs {
    Octree o;
    DevTape bt;
    const RegClause* arena;
    LeafRec* recs;
    uint32_t* rec_top;
    uint32_t rec_cap;
    uint32_t* status;
    double max_err;
};

__device__ __forceinline__ uint8_t corner_state(uint8_t type, const LeafRec* r,
                                                int corner)
{
    if (type == CELL_LEAF) {
        return ((r->corner_mask >> corner) & 1) ? CELL_FILLED : CELL_EMPTY;
    }
    return type;
}

/// Serial value evaluation of one point by one thread (registers in R with
/// stride B), used for the collapse test at a candidate vertex.
__device__ float thread_value(const DevTape& bt, const RegClause* cl,
                              uint32_t len, float* R, int tid, int B, float x,
                              float y, float z)
{
    R[0 * B + tid] = x;
    R[1 * B + tid] = y;
    R[2 * B + tid] = z;
    for (uint32_t c = 0; c < len; ++c) {
        const uint2 raw = __ldg(reinterpret_cast<const uint2*>(cl + c));
        const uint8_t o = raw.x & 0xff;
        const uint8_t kinds = (raw.x >> 8) & 0xff;
        const uint16_t ra = raw.y & 0xffff, rb = raw.y >> 16;
        const float a = (kinds & 3) == OPND_REG ? R[ra * B + tid] : __ldg(bt.cpool + ra);
        const float b = ((kinds >> 2) & 3) == OPND_REG ? R[rb * B + tid] : __ldg(bt.cpool + rb);
        R[(raw.x >> 16) * B + tid] = dv_value(o, a, b);
    }
    return bt.root_kind == OPND_REG ? R[bt.root * B + tid] : __ldg(bt.cpool + bt.root);
}

__global__ void __launch_bounds__(128)
k_collapse_level(CollapseArgs A, int d)
{
    extern __shared__ float csmem[];
    const int B = blockDim.x, tid = threadIdx.x;
    const Octree& o = A.o;
    const LevelView& lv = o.lv[d];
    const uint32_t i = blockIdx.x * B + tid;
    if (i >= lv.n_cells || lv.type[i] != CELL_BRANCH) return;

    const LevelView& cv = o.lv[d + 1];
    const uint32_t k = static_cast<uint32_t>(lv.child_group[i]);
    uint8_t ct[8];
    const LeafRec* cr[8];
    bool any_branch = false, all_empty = true, all_filled = true;
    for (int j = 0; j < 8; ++j) {
        ct[j] = cv.type[8 * k + j];
        const int32_t r = cv.rec[8 * k + j];
        cr[j] = (ct[j] == CELL_LEAF && r >= 0) ? &A.recs[r] : nullptr;
        any_branch |= ct[j] == CELL_BRANCH;
        all_empty &= ct[j] == CELL_EMPTY;
        all_filled &= ct[j] == CELL_FILLED;
    }
    if (any_branch) return;
    if (all_empty || all_filled) {
        lv.type[i] = all_empty ? CELL_EMPTY : CELL_FILLED;
        return;
    }
    auto cs = [&](int child, int corner) { return corner_state(ct[child], cr[child], corner); };
    uint8_t corners[8];
    uint8_t mask = 0;
    for (int j = 0; j < 8; ++j) {
        corners[j] = cs(j, j);
        mask |= (corners[j] == CELL_FILLED ? 1 : 0) << j;
    }
    bool manifold = c_tab.manifold[mask];
    for (int j = 0; j < 8 && manifold; ++j) {
        if (ct[j] == CELL_LEAF) manifold = cr[j]->manifold;
    }
    if (manifold) {
        // Ju et al. 2002 sign checks at coarse edge, face and cube centres
        // (dc_tree3.cpp:16-109): the child at corner a holds the midpoint of
        // the coarse edge a -> a|bit as its corner a|bit.
        for (int a = 0; a < 8 && manifold; ++a) {
            for (int bit = 1; bit < 8 && manifold; bit <<= 1) {
                if (a & bit) continue;
                const uint8_t m = cs(a, a | bit);
                manifold = (m == corners[a] || m == corners[a | bit]);
            }
        }
        const int faces[6][5] = {
            {0, 5, 0, 1, 4}, {0, 6, 0, 2, 4}, {0, 3, 0, 2, 1},
            {7, 1, 1, 5, 3}, {7, 2, 2, 6, 3}, {7, 4, 4, 6, 5}};
        for (int f = 0; f < 6 && manifold; ++f) {
            const uint8_t m = cs(faces[f][0], faces[f][1]);
            const int c3 = faces[f][0] == 0 ? faces[f][1] : 7;
            manifold = m == corners[faces[f][2]] || m == corners[faces[f][3]] ||
                       m == corners[faces[f][4]] || m == corners[c3];
        }
        if (manifold) {
            const uint8_t m = cs(0, 7);
            bool ok = false;
            for (int j = 0; j < 8; ++j) ok |= m == corners[j];
            manifold = ok;
        }
    }
    if (!manifold) return;

    unsigned rank = 0;
    for (int j = 0; j < 8; ++j) {
        if (cr[j] && cr[j]->rank > rank) rank = cr[j]->rank;
    }
    Qef q;
    qef_zero(q);
    for (int j = 0; j < 8; ++j) {
        if (!cr[j]) continue;
        if (cr[j]->rank == rank) {
            for (int t = 0; t < 4; ++t) q.mass[t] += cr[j]->mass[t];
        }
        for (int t = 0; t < 6; ++t) q.ata[t] += cr[j]->ata[t];
        for (int t = 0; t < 3; ++t) q.atb[t] += cr[j]->atb[t];
        q.btb += cr[j]->btb;
    }
    double v[3];
    const double err = qef_vertex(q, v, nullptr);
    double lo[3], hi[3];
    cell_bounds(o, d, lv.coords[i], lo, hi);
    bool inside = true;
    for (int a = 0; a < 3; ++a) {
        inside &= (v[a] >= lo[a] - 1e-6) && (v[a] <= hi[a] + 1e-6);
    }
    if (!(err < A.max_err) || !inside) return;

    // Value at the vertex with a tape that is valid there: walk up from this
    // cell to the first ancestor whose (float) box contains the point
    // (Tape::getBase, tape.cpp:188-209); the unpruned tape otherwise.
    const float vf[3] = {static_cast<float>(v[0]), static_cast<float>(v[1]),
                         static_cast<float>(v[2])};
    TapeRef tr = {0u, A.bt.n, A.bt.n_choices, 0u};
    {
        int dd = d;
        uint32_t ii = i;
        while (dd >= 0) {
            double blo[3], bhi[3];
            cell_bounds(o, dd, o.lv[dd].coords[ii], blo, bhi);
            bool in = true;
            for (int a = 0; a < 3; ++a) {
                in &= vf[a] >= static_cast<float>(blo[a]) &&
                      vf[a] <= static_cast<float>(bhi[a]);
            }
            if (in) {
                tr = o.lv[dd].cell_tape[ii];
                break;
            }
            if (dd == 0) break;
            ii = o.lv[dd].group_parent[ii >> 3];
            --dd;
        }
    }
    const float value = thread_value(A.bt, A.arena + tr.off, tr.len, csmem, tid, B,
                                     vf[0], vf[1], vf[2]);
    if (!(fabsf(value) < A.max_err)) return;

    const uint32_t r = atomicAdd(A.rec_top, 1u);
    if (r >= A.rec_cap) {
        atomicOr(A.status, ST_RECORD_OVERFLOW);
        return;
    }
    LeafRec& L = A.recs[r];
    for (int t = 0; t < 3; ++t) L.vert[0][t] = v[t];
    for (int t = 0; t < 4; ++t) L.mass[t] = q.mass[t];
    for (int t = 0; t < 6; ++t) L.ata[t] = q.ata[t];
    for (int t = 0; t < 3; ++t) L.atb[t] = q.atb[t];
    L.btb = q.btb;
    L.level = o.levels - d;
    L.corner_mask = mask;
    L.vertex_count = 1;
    L.rank = static_cast<uint8_t>(rank);
    L.manifold = 1;
    lv.rec[i] = static_cast<int32_t>(r);
    lv.type[i] = CELL_LEAF;
}

////////////////////////////////////////////////////////////////////////////////
// 4. Dual walk (Dual<3>::work / face3 / edge3, dual.hpp:126-203) and
//    DCMesher::load (dc_mesher.cpp:18-169)

enum : uint8_t { TASK_CELL = 0, TASK_FACE = 1, TASK_EDGE = 2 };

struct DualTask {
    uint8_t kind;
    uint8_t axis;   // 1, 2, 4
    uint8_t pad[2];
    uint32_t ref[4];
};

__device__ __forceinline__ uint32_t make_ref(int depth, uint32_t idx)
{
    return (static_cast<uint32_t>(depth) << 27) | idx;
}
__device__ __forceinline__ int ref_depth(uint32_t r) { return r >> 27; }
__device__ __forceinline__ uint32_t ref_idx(uint32_t r) { return r & 0x7ffffff; }

__device__ __forceinline__ int axis_q(int a) { return a == 1 ? 2 : a == 2 ? 4 : 1; }
__device__ __forceinline__ int axis_r(int a) { return a == 1 ? 4 : a == 2 ? 1 : 2; }

struct DualArgs {
    Octree o;
    const LeafRec* recs;
    uint32_t* status;
    DualTask* out;
    uint32_t* n_out;
    uint32_t out_cap;
    uint32_t* tris;      // 3 vertex keys per triangle (record * 4 + vertex)
    uint32_t* n_tris;
    uint32_t tri_cap;
    uint8_t* used;       // per vertex key
};

__device__ __forceinline__ uint8_t ref_type(const Octree& o, uint32_t r)
{
    return o.lv[ref_depth(r)].type[ref_idx(r)];
}

__device__ __forceinline__ uint32_t ref_child(const Octree& o, uint32_t r, int k)
{
    const int d = ref_depth(r);
    const uint32_t i = ref_idx(r);
    if (o.lv[d].type[i] != CELL_BRANCH) return r;
    return make_ref(d + 1, 8u * static_cast<uint32_t>(o.lv[d].child_group[i]) + k);
}

__device__ __forceinline__ void push_task(const DualArgs& A, uint8_t kind,
                                          uint8_t axis, const uint32_t* refs,
                                          int nref)
{
    // A task holding an EMPTY / FILLED leaf can never produce a face: that
    // leaf stays in every task derived from it and DCMesher::load exits on
    // it (dc_mesher.cpp:23-28).
    bool branch = false;
    for (int k = 0; k < nref; ++k) {
        const uint8_t t = ref_type(A.o, refs[k]);
        if (t == CELL_EMPTY || t == CELL_FILLED) return;
        branch |= t == CELL_BRANCH;
    }
    if (kind == TASK_FACE && !branch) return;
    const uint32_t slot = atomicAdd(A.n_out, 1u);
    if (slot >= A.out_cap) {
        atomicOr(A.status, ST_QUEUE_OVERFLOW);
        return;
    }
    DualTask t;
    t.kind = kind;
    t.axis = axis;
    t.pad[0] = t.pad[1] = 0;
    for (int k = 0; k < 4; ++k) t.ref[k] = k < nref ? refs[k] : 0;
    A.out[slot] = t;
}

__device__ void emit_edge(const DualArgs& A, int ax, const uint32_t ts[4])
{
    const Octree& o = A.o;
    const LeafRec* R[4];
    int32_t ri[4];
    for (int k = 0; k < 4; ++k) {
        ri[k] = o.lv[ref_depth(ts[k])].rec[ref_idx(ts[k])];
        if (ri[k] < 0) return;
        R[k] = &A.recs[ri[k]];
    }
    int index = 0;
    for (int k = 1; k < 4; ++k) {
        if (R[k]->level < R[index]->level) index = k;
    }
    const int Q = axis_q(ax), Rr = axis_r(ax);
    const int corners[4] = {Q | Rr, Rr, Q, 0};
    const int ca = (R[index]->corner_mask >> corners[index]) & 1;
    const int cb = (R[index]->corner_mask >> (corners[index] | ax)) & 1;
    if (ca == cb) return;
    const bool D = ca != 0;   // a is FILLED
    const int ev[4][2] = {{Q | Rr, Q | Rr | ax}, {Rr, Rr | ax}, {Q, Q | ax}, {0, ax}};
    uint32_t vs[4];
    float P[4][3];
    for (int k = 0; k < 4; ++k) {
        const int e = D ? c_tab.e[ev[k][0]][ev[k][1]] : c_tab.e[ev[k][1]][ev[k][0]];
        const int vi = R[k]->level > 0 ? 0 : c_tab.p[R[k]->corner_mask][e];
        vs[k] = static_cast<uint32_t>(ri[k]) * 4u + static_cast<uint32_t>(vi < 0 ? 0 : vi);
        for (int t = 0; t < 3; ++t) P[k][t] = static_cast<float>(R[k]->vert[vi < 0 ? 0 : vi][t]);
    }
    if (!D) {
        const uint32_t tv = vs[1]; vs[1] = vs[2]; vs[2] = tv;
        for (int t = 0; t < 3; ++t) {
            const float tp = P[1][t]; P[1][t] = P[2][t]; P[2][t] = tp;
        }
    }
    float N[4][3];
    auto save_norm = [&](int a, int b, int c) {
        const float u[3] = {__fsub_rn(P[b][0], P[a][0]), __fsub_rn(P[b][1], P[a][1]),
                            __fsub_rn(P[b][2], P[a][2])};
        const float w[3] = {__fsub_rn(P[c][0], P[a][0]), __fsub_rn(P[c][1], P[a][1]),
                            __fsub_rn(P[c][2], P[a][2])};
        float n[3] = {__fsub_rn(__fmul_rn(u[1], w[2]), __fmul_rn(u[2], w[1])),
                      __fsub_rn(__fmul_rn(u[2], w[0]), __fmul_rn(u[0], w[2])),
                      __fsub_rn(__fmul_rn(u[0], w[1]), __fmul_rn(u[1], w[0]))};
        const float z = __fadd_rn(__fadd_rn(__fmul_rn(n[0], n[0]), __fmul_rn(n[1], n[1])),
                                  __fmul_rn(n[2], n[2]));
        if (z > 0) {
            const float s = __fsqrt_rn(z);
            n[0] = __fdiv_rn(n[0], s);
            n[1] = __fdiv_rn(n[1], s);
            n[2] = __fdiv_rn(n[2], s);
        }
        N[a][0] = n[0]; N[a][1] = n[1]; N[a][2] = n[2];
    };
    save_norm(0, 1, 2);
    save_norm(1, 3, 0);
    save_norm(2, 0, 3);
    save_norm(3, 2, 1);
    auto dot = [](const float* a, const float* b) {
        return __fadd_rn(__fadd_rn(__fmul_rn(a[0], b[0]), __fmul_rn(a[1], b[1])),
                         __fmul_rn(a[2], b[2]));
    };
    uint32_t tri[2][3];
    if (dot(N[0], N[3]) > dot(N[1], N[2])) {
        tri[0][0] = vs[0]; tri[0][1] = vs[1]; tri[0][2] = vs[2];
        tri[1][0] = vs[2]; tri[1][1] = vs[1]; tri[1][2] = vs[3];
    } else {
        tri[0][0] = vs[0]; tri[0][1] = vs[1]; tri[0][2] = vs[3];
        tri[1][0] = vs[0]; tri[1][1] = vs[3]; tri[1][2] = vs[2];
    }
    for (int t = 0; t < 2; ++t) {
        const uint32_t a = tri[t][0], b = tri[t][1], c = tri[t][2];
        if (a == b || b == c || a == c) continue;
        const uint32_t slot = atomicAdd(A.n_tris, 1u);
        if (slot >= A.tri_cap) {
            atomicOr(A.status, ST_QUEUE_OVERFLOW);
            return;
        }
        A.tris[3 * slot + 0] = a;
        A.tris[3 * slot + 1] = b;
        A.tris[3 * slot + 2] = c;
        A.used[a] = 1;
        A.used[b] = 1;
        A.used[c] = 1;
    }
}

__global__ void __launch_bounds__(128)
k_dual_round(DualArgs A, const DualTask* in, uint32_t n_in)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_in) return;
    const DualTask task = in[t];
    const Octree& o = A.o;
    const int ax = task.axis;
    if (task.kind == TASK_CELL) {
        const uint32_t c = task.ref[0];
        uint32_t ch[8];
        for (int k = 0; k < 8; ++k) ch[k] = ref_child(o, c, k);
        for (int k = 0; k < 8; ++k) {
            if (ref_type(o, ch[k]) == CELL_BRANCH) {
                push_task(A, TASK_CELL, 0, &ch[k], 1);
            }
        }
        for (int a = 1; a <= 4; a <<= 1) {
            const int q = axis_q(a), r = axis_r(a);
            const int pairs[4][2] = {{0, a}, {q, q | a}, {r, r | a}, {q | r, q | r | a}};
            for (int p = 0; p < 4; ++p) {
                const uint32_t f[2] = {ch[pairs[p][0]], ch[pairs[p][1]]};
                push_task(A, TASK_FACE, static_cast<uint8_t>(a), f, 2);
            }
        }
        for (int a = 1; a <= 4; a <<= 1) {
            const int q = axis_q(a), r = axis_r(a);
            for (int s = 0; s < 2; ++s) {
                const int b = s ? a : 0;
                const uint32_t e[4] = {ch[b], ch[q | b], ch[r | b], ch[q | r | b]};
                push_task(A, TASK_EDGE, static_cast<uint8_t>(a), e, 4);
            }
        }
    } else if (task.kind == TASK_FACE) {
        const uint32_t t0 = task.ref[0], t1 = task.ref[1];
        const int Q = axis_q(ax), R = axis_r(ax);
        const int ks[4] = {0, Q, R, Q | R};
        for (int k = 0; k < 4; ++k) {
            const uint32_t f[2] = {ref_child(o, t0, ks[k] | ax), ref_child(o, t1, ks[k])};
            push_task(A, TASK_FACE, static_cast<uint8_t>(ax), f, 2);
        }
        const uint32_t e0[4] = {ref_child(o, t0, ax), ref_child(o, t0, R | ax),
                                ref_child(o, t1, 0), ref_child(o, t1, R)};
        push_task(A, TASK_EDGE, static_cast<uint8_t>(Q), e0, 4);
        const uint32_t e1[4] = {ref_child(o, t0, Q | ax), ref_child(o, t0, Q | R | ax),
                                ref_child(o, t1, Q), ref_child(o, t1, Q | R)};
        push_task(A, TASK_EDGE, static_cast<uint8_t>(Q), e1, 4);
        const uint32_t e2[4] = {ref_child(o, t0, ax), ref_child(o, t1, 0),
                                ref_child(o, t0, ax | Q), ref_child(o, t1, Q)};
        push_task(A, TASK_EDGE, static_cast<uint8_t>(R), e2, 4);
        const uint32_t e3[4] = {ref_child(o, t0, R | ax), ref_child(o, t1, R),
                                ref_child(o, t0, R | ax | Q), ref_child(o, t1, R | Q)};
        push_task(A, TASK_EDGE, static_cast<uint8_t>(R), e3, 4);
    } else {
        bool branch = false;
        for (int k = 0; k < 4; ++k) branch |= ref_type(o, task.ref[k]) == CELL_BRANCH;
        if (!branch) {
            emit_edge(A, ax, task.ref);
            return;
        }
        const int Q = axis_q(ax), R = axis_r(ax);
        const uint32_t a[4] = {ref_child(o, task.ref[0], Q | R), ref_child(o, task.ref[1], R),
                               ref_child(o, task.ref[2], Q), ref_child(o, task.ref[3], 0)};
        push_task(A, TASK_EDGE, static_cast<uint8_t>(ax), a, 4);
        const uint32_t b[4] = {ref_child(o, task.ref[0], Q | R | ax),
                               ref_child(o, task.ref[1], R | ax),
                               ref_child(o, task.ref[2], Q | ax),
                               ref_child(o, task.ref[3], ax)};
        push_task(A, TASK_EDGE, static_cast<uint8_t>(ax), b, 4);
    }
}

////////////////////////////////////////////////////////////////////////////////
// Small helpers for the host driver

__global__ void k_init_root(Octree o)
{
    o.lv[0].coords[0] = 0;
}

__global__ void k_branch_flags(const uint8_t* type, uint32_t n, uint32_t* flags)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[i] = type[i] == CELL_BRANCH ? 1u : 0u;
}

/// For each branch cell at depth d: its group index at d + 1, and the
/// group's parent, tape, decision scratch size and child coordinates.
__global__ void k_build_groups(Octree o, int d, const uint32_t* scan,
                               uint64_t* dec_sizes)
{
    const LevelView& lv = o.lv[d];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= lv.n_cells) return;
    if (lv.type[i] != CELL_BRANCH) {
        lv.child_group[i] = -1;
        return;
    }
    const uint32_t g = scan[i];
    lv.child_group[i] = static_cast<int32_t>(g);
    LevelView& nv = o.lv[d + 1];
    nv.group_parent[g] = i;
    const TapeRef tr = lv.cell_tape[i];
    nv.group_tape[g] = tr;
    dec_sizes[g] = 8ull * tr.nch;
    uint32_t x, y, z;
    unpack_coords(lv.coords[i], x, y, z);
    for (int k = 0; k < 8; ++k) {
        nv.coords[8 * g + k] = pack_coords(2 * x + (k & 1), 2 * y + ((k >> 1) & 1),
                                           2 * z + ((k >> 2) & 1));
    }
}

__global__ void k_vertex_ids(const uint8_t* used, const uint32_t* scan,
                             uint32_t n_keys, const LeafRec* recs,
                             float* verts)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_keys || !used[k]) return;
    const LeafRec& r = recs[k >> 2];
    const uint32_t id = scan[k] + 1;   // index 0 is the placeholder vertex
    for (int t = 0; t < 3; ++t) verts[3 * id + t] = static_cast<float>(r.vert[k & 3][t]);
}

__global__ void k_u8_to_u32(const uint8_t* in, uint32_t* out, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i];
}

__global__ void k_remap_tris(uint32_t* tris, uint32_t n, const uint32_t* scan)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 3 * n) tris[i] = scan[tris[i]] + 1;
}

}  // namespace lfb

////////////////////////////////////////////////////////////////////////////////
// Host driver

#include <chrono>
#include <map>
#include <vector>

#include "mesher.hpp"

namespace lfb {

namespace {

/// Grow-only device buffers keyed by purpose, reused across calls.
struct Workspace {
    std::map<int, DevBuf> bufs;
    template <class T>
    T* get(int key, size_t count)
    {
        DevBuf& b = bufs[key];
        if (!b.reserve(std::max<size_t>(count, 1) * sizeof(T))) return nullptr;
        return b.as<T>();
    }
};

Workspace& workspace()
{
    static Workspace w;
    return w;
}

enum BufKey {
    K_ARENA = 1, K_DEC, K_STATUS, K_COUNTERS, K_RECS, K_FLAGS, K_SCAN,
    K_CUBTMP, K_DECSZ, K_DECOFF, K_TASK_A, K_TASK_B, K_TRIS, K_USED,
    K_VSCAN, K_VERTS, K_FEAT, K_LEVEL = 100,
};

bool tables_ready = false;

bool upload_tables()
{
    if (tables_ready) return true;
    static DcTables t;
    build_dc_tables(t);
    if (!cuda_ok(cudaMemcpyToSymbol(c_tab, &t, sizeof(t)), "dc tables")) return false;
    tables_ready = true;
    return true;
}

int level_from_resolution(const double lo[3], const double hi[3], double min_feature)
{
    // Region::withResolution (region.hpp:226-231), including its float logf.
    double md = hi[0] - lo[0];
    for (int a = 1; a < 3; ++a) md = std::min(md, hi[a] - lo[a]);
    const float l = std::ceil(std::fmax(0.0f, logf(static_cast<float>(md / min_feature))) /
                              logf(2.0f));
    return static_cast<int>(l);
}

template <class T>
bool exclusive_scan(const T* in, T* out, uint32_t n, cudaStream_t s)
{
    auto& ws = workspace();
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, n, s);
    void* t = ws.get<unsigned char>(K_CUBTMP, tmp);
    if (!t) return false;
    return cuda_ok(cub::DeviceScan::ExclusiveSum(t, tmp, in, out, n, s), "scan");
}

}  // namespace

int render_dc_mesh(GpuTape& g, const libfive_region3& R, double min_feature,
                   double max_err, MeshOut& out, lfb_mesh_stats* stats)
{
    if (!require_device()) return LFB_E_CUDA;
    std::lock_guard<std::mutex> lock(global_mutex());
    if (!upload_tables()) return LFB_E_CUDA;
    auto& ws = workspace();
    cudaStream_t s = 0;
    const auto t_start = std::chrono::steady_clock::now();

    Octree o{};
    o.lo[0] = R.X.lower; o.hi[0] = R.X.upper;
    o.lo[1] = R.Y.lower; o.hi[1] = R.Y.upper;
    o.lo[2] = R.Z.lower; o.hi[2] = R.Z.upper;
    const int L = level_from_resolution(o.lo, o.hi, min_feature);
    if (L > kMaxLevels) {
        return set_error(LFB_E_UNSUPPORTED, "octree deeper than 24 levels");
    }
    o.levels = L;
    const DevTape bt = g.dev();
    if (bt.n_regs > 400) {
        return set_error(LFB_E_UNSUPPORTED, "tape needs more than 400 registers");
    }

    uint32_t* status = ws.get<uint32_t>(K_STATUS, 1);
    unsigned long long* counters = ws.get<unsigned long long>(K_COUNTERS, 8);
    if (!status || !counters) return LFB_E_CUDA;
    cudaMemsetAsync(status, 0, sizeof(uint32_t), s);
    cudaMemsetAsync(counters, 0, 8 * sizeof(unsigned long long), s);
    uint32_t* arena_top = reinterpret_cast<uint32_t*>(counters + 1);
    uint32_t* rec_top = reinterpret_cast<uint32_t*>(counters + 2);
    unsigned long long* evals = counters + 3;

    // Tape arena: the unpruned tape first, pruned tapes appended.
    size_t arena_cap = std::max<size_t>(bt.n * 64 + (1u << 20), 1u << 22);
    RegClause* arena = ws.get<RegClause>(K_ARENA, arena_cap);
    if (!arena) return LFB_E_CUDA;
    if (bt.n && !cuda_ok(cudaMemcpyAsync(arena, bt.clauses, bt.n * sizeof(RegClause),
                                         cudaMemcpyDeviceToDevice, s), "arena")) {
        return LFB_E_CUDA;
    }
    uint32_t top_host = bt.n;
    cudaMemcpyAsync(arena_top, &top_host, sizeof(uint32_t), cudaMemcpyHostToDevice, s);

    // Level 0: the root cell.
    auto alloc_level = [&](int d, uint32_t n_cells, uint32_t n_groups) -> bool {
        LevelView& lv = o.lv[d];
        lv.n_cells = n_cells;
        lv.n_groups = n_groups;
        const int k = K_LEVEL + 16 * d;
        lv.coords = ws.get<uint64_t>(k + 0, n_cells);
        lv.type = ws.get<uint8_t>(k + 1, n_cells);
        lv.rec = ws.get<int32_t>(k + 2, n_cells);
        lv.child_group = ws.get<int32_t>(k + 3, n_cells);
        lv.cell_tape = ws.get<TapeRef>(k + 4, n_cells);
        lv.group_parent = ws.get<uint32_t>(k + 5, n_groups);
        lv.group_tape = ws.get<TapeRef>(k + 6, n_groups);
        lv.group_dec = ws.get<uint64_t>(k + 7, n_groups);
        if (!lv.coords || !lv.type || !lv.rec || !lv.child_group || !lv.cell_tape ||
            !lv.group_parent || !lv.group_tape || !lv.group_dec) {
            return false;
        }
        cudaMemsetAsync(lv.rec, 0xff, n_cells * sizeof(int32_t), s);
        return true;
    };
    if (!alloc_level(0, 1, 0)) return LFB_E_CUDA;
    k_init_root<<<1, 1, 0, s>>>(o);
    if (L == 0) {
        // No interval pass: the root is evaluated as a leaf right away.
        cudaMemsetAsync(o.lv[0].type, CELL_BRANCH, 1, s);
    }

    // Stage timing with CUDA events on the pipeline's stream (only when the
    // caller asks for statistics).
    cudaEvent_t ev[5] = {};
    if (stats) {
        for (auto& e : ev) cudaEventCreate(&e);
        cudaEventRecord(ev[0], s);
    }
    uint64_t n_launch = 1;   // k_init_root
    uint64_t cells_evaluated = 0;
    uint64_t dec_total = bt.n_choices;   // decision bytes needed by level 0
    for (int d = 0; d < L; ++d) {
        LevelView& lv = o.lv[d];
        cells_evaluated += lv.n_cells;
        uint8_t* dec = ws.get<uint8_t>(K_DEC, std::max<uint64_t>(dec_total, 1));
        if (!dec) return LFB_E_CUDA;
        // Arena: worst case every cell writes a tape as long as its input.
        uint64_t need = 0;
        {
            // Upper bound: n_cells * (longest group tape) is cheap to get as
            // dec_total/choices is not a length; use the running input size.
            need = static_cast<uint64_t>(lv.n_cells) * std::max<uint32_t>(bt.n, 1);
        }
        (void)need;
        int block = 128;
        while (block > 32 && static_cast<size_t>(bt.n_regs) * block * 9 > 96 * 1024) block /= 2;
        const size_t smem = static_cast<size_t>(bt.n_regs) * block * 9 + 16;
        if (smem > 48 * 1024) {
            cudaFuncSetAttribute(k_interval_level, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem));
        }
        for (int attempt = 0; attempt < 6; ++attempt) {
            const uint32_t saved_top_dummy = 0;
            (void)saved_top_dummy;
            uint32_t top_before = 0;
            cudaMemcpyAsync(&top_before, arena_top, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
            cudaStreamSynchronize(s);
            k_interval_level<<<(lv.n_cells + block - 1) / block, block, smem, s>>>(
                o, d, bt, arena, arena_top, static_cast<uint32_t>(arena_cap), dec, status);
            ++n_launch;
            if (!cuda_ok(cudaGetLastError(), "interval kernel")) return LFB_E_CUDA;
            uint32_t st = 0;
            cudaMemcpyAsync(&st, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
            if (!cuda_ok(cudaStreamSynchronize(s), "interval kernel")) return LFB_E_CUDA;
            if (!(st & ST_ARENA_OVERFLOW)) break;
            // Grow the arena (keeping its contents) and redo this level.
            const size_t new_cap = arena_cap * 4;
            RegClause* bigger = nullptr;
            if (!cuda_ok(cudaMalloc(&bigger, new_cap * sizeof(RegClause)), "arena grow")) {
                return LFB_E_CUDA;
            }
            cudaMemcpyAsync(bigger, arena, static_cast<size_t>(top_before) * sizeof(RegClause),
                            cudaMemcpyDeviceToDevice, s);
            DevBuf& b = ws.bufs[K_ARENA];
            cudaStreamSynchronize(s);
            cudaFree(b.ptr);
            b.ptr = bigger;
            b.bytes = new_cap * sizeof(RegClause);
            arena = bigger;
            arena_cap = new_cap;
            cudaMemcpyAsync(arena_top, &top_before, sizeof(uint32_t), cudaMemcpyHostToDevice, s);
            const uint32_t zero = 0;
            cudaMemcpyAsync(status, &zero, sizeof(uint32_t), cudaMemcpyHostToDevice, s);
            if (attempt == 5) return set_error(LFB_E_CAPACITY, "tape arena overflow");
        }

        // Compact the branch cells into the groups of depth d + 1.
        uint32_t* flags = ws.get<uint32_t>(K_FLAGS, lv.n_cells + 1);
        uint32_t* scan = ws.get<uint32_t>(K_SCAN, lv.n_cells + 1);
        if (!flags || !scan) return LFB_E_CUDA;
        k_branch_flags<<<(lv.n_cells + 255) / 256, 256, 0, s>>>(lv.type, lv.n_cells, flags);
        cudaMemsetAsync(flags + lv.n_cells, 0, sizeof(uint32_t), s);
        if (!exclusive_scan(flags, scan, lv.n_cells + 1, s)) return LFB_E_CUDA;
        uint32_t n_groups = 0;
        cudaMemcpyAsync(&n_groups, scan + lv.n_cells, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if (!cuda_ok(cudaStreamSynchronize(s), "scan")) return LFB_E_CUDA;
        if (static_cast<uint64_t>(n_groups) * 8 >= (1u << 27)) {
            return set_error(LFB_E_CAPACITY, "more than 2^27 cells on one octree level");
        }
        if (!alloc_level(d + 1, n_groups * 8, n_groups)) return LFB_E_CUDA;
        uint64_t* dec_sizes = ws.get<uint64_t>(K_DECSZ, n_groups + 1);
        if (!dec_sizes) return LFB_E_CUDA;
        k_build_groups<<<(lv.n_cells + 255) / 256, 256, 0, s>>>(o, d, scan, dec_sizes);
        n_launch += 2;   // k_branch_flags + k_build_groups
        cudaMemsetAsync(dec_sizes + n_groups, 0, sizeof(uint64_t), s);
        if (!exclusive_scan(dec_sizes, o.lv[d + 1].group_dec, n_groups, s)) return LFB_E_CUDA;
        // total decision bytes of the next level
        uint64_t last_off = 0, last_sz = 0;
        if (n_groups) {
            cudaMemcpyAsync(&last_off, o.lv[d + 1].group_dec + n_groups - 1, 8, cudaMemcpyDeviceToHost, s);
            cudaMemcpyAsync(&last_sz, dec_sizes + n_groups - 1, 8, cudaMemcpyDeviceToHost, s);
        }
        if (!cuda_ok(cudaStreamSynchronize(s), "groups")) return LFB_E_CUDA;
        dec_total = last_off + last_sz;
        if (n_groups == 0) {
            // Nothing ambiguous below this depth: no leaves, no faces.
            o.levels = L;
            for (int dd = d + 1; dd <= L; ++dd) {
                if (!alloc_level(dd, 0, 0)) return LFB_E_CUDA;
            }
            break;
        }
    }

    if (stats) cudaEventRecord(ev[1], s);
    // Leaves.
    const uint32_t n_leaf_groups = (L == 0) ? 1 : o.lv[L].n_groups;
    const size_t rec_cap = static_cast<size_t>(n_leaf_groups) * 8 + cells_evaluated + 16;
    LeafRec* recs = ws.get<LeafRec>(K_RECS, rec_cap);
    if (!recs) return LFB_E_CUDA;
    if (n_leaf_groups) {
        LeafArgs A{o, bt, arena, recs, rec_top, static_cast<uint32_t>(rec_cap), status,
                   evals};
        int wpb = 4;
        const size_t per_warp = sizeof(LeafWarpShared) + static_cast<size_t>(bt.n_regs) * 128 * 4;
        while (wpb > 1 && per_warp * wpb > 200 * 1024) --wpb;
        const size_t smem = per_warp * wpb;
        if (smem > 220 * 1024) {
            return set_error(LFB_E_UNSUPPORTED, "tape register file too large for the leaf kernel");
        }
        cudaFuncSetAttribute(k_leaf_groups, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
        k_leaf_groups<<<(n_leaf_groups + wpb - 1) / wpb, 32 * wpb, smem, s>>>(A, n_leaf_groups);
        if (!cuda_ok(cudaGetLastError(), "leaf kernel")) return LFB_E_CUDA;
        ++n_launch;
    }
    if (stats) cudaEventRecord(ev[2], s);

    // Bottom-up collapse.
    {
        CollapseArgs C{o, bt, arena, recs, rec_top, static_cast<uint32_t>(rec_cap), status,
                       max_err};
        int block = 128;
        while (block > 32 && static_cast<size_t>(bt.n_regs) * block * 4 > 96 * 1024) block /= 2;
        const size_t smem = static_cast<size_t>(bt.n_regs) * block * 4;
        if (smem > 48 * 1024) {
            cudaFuncSetAttribute(k_collapse_level, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem));
        }
        for (int d = L - 1; d >= 0; --d) {
            const uint32_t n = o.lv[d].n_cells;
            if (!n) continue;
            k_collapse_level<<<(n + block - 1) / block, block, smem, s>>>(C, d);
            ++n_launch;
        }
        if (!cuda_ok(cudaGetLastError(), "collapse kernel")) return LFB_E_CUDA;
    }

    if (stats) cudaEventRecord(ev[3], s);
    uint32_t st = 0, n_recs = 0;
    cudaMemcpyAsync(&st, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&n_recs, rec_top, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (!cuda_ok(cudaStreamSynchronize(s), "leaf/collapse")) return LFB_E_CUDA;
    if (st & ST_RECORD_OVERFLOW) return set_error(LFB_E_CAPACITY, "leaf record overflow");
    if (st & ST_FEATURE_OVERFLOW) {
        return set_error(LFB_E_CAPACITY,
                         "feature list overflow at a non-smooth sample point");
    }

    // Dual walk.
    out.verts.assign(3, 0.0f);
    out.tris.clear();
    uint8_t root_type = 0;
    cudaMemcpyAsync(&root_type, o.lv[0].type, 1, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    const uint32_t n_keys = n_recs * 4;
    if (root_type == CELL_BRANCH && n_recs) {
        size_t task_cap = std::max<size_t>(1u << 16, static_cast<size_t>(n_recs) * 24);
        size_t tri_cap = std::max<size_t>(1u << 16, static_cast<size_t>(n_recs) * 16);
        for (int attempt = 0; attempt < 5; ++attempt) {
            DualTask* qa = ws.get<DualTask>(K_TASK_A, task_cap);
            DualTask* qb = ws.get<DualTask>(K_TASK_B, task_cap);
            uint32_t* tris = ws.get<uint32_t>(K_TRIS, 3 * tri_cap);
            uint8_t* used = ws.get<uint8_t>(K_USED, n_keys + 1);
            if (!qa || !qb || !tris || !used) return LFB_E_CUDA;
            cudaMemsetAsync(used, 0, n_keys + 1, s);
            uint32_t* n_out = reinterpret_cast<uint32_t*>(counters + 5);
            uint32_t* n_tris = reinterpret_cast<uint32_t*>(counters + 6);
            cudaMemsetAsync(n_tris, 0, sizeof(uint32_t), s);
            cudaMemsetAsync(status, 0, sizeof(uint32_t), s);
            DualTask root{};
            root.kind = TASK_CELL;
            cudaMemcpyAsync(qa, &root, sizeof(root), cudaMemcpyHostToDevice, s);
            uint32_t n_in = 1;
            DualArgs D{o, recs, status, qb, n_out, static_cast<uint32_t>(task_cap),
                       tris, n_tris, static_cast<uint32_t>(tri_cap), used};
            bool overflow = false;
            while (n_in) {
                cudaMemsetAsync(n_out, 0, sizeof(uint32_t), s);
                D.out = qb;
                k_dual_round<<<(n_in + 127) / 128, 128, 0, s>>>(D, qa, n_in);
                ++n_launch;
                uint32_t st2 = 0;
                cudaMemcpyAsync(&n_in, n_out, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
                cudaMemcpyAsync(&st2, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
                if (!cuda_ok(cudaStreamSynchronize(s), "dual walk")) return LFB_E_CUDA;
                if (st2 & ST_QUEUE_OVERFLOW) {
                    overflow = true;
                    break;
                }
                std::swap(qa, qb);
            }
            if (overflow) {
                task_cap *= 4;
                tri_cap *= 4;
                continue;
            }
            uint32_t n_tri = 0;
            cudaMemcpyAsync(&n_tri, n_tris, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
            // Vertex numbering: ids in record order, 0 is the placeholder.
            uint32_t* flags = ws.get<uint32_t>(K_FLAGS, n_keys + 1);
            uint32_t* vscan = ws.get<uint32_t>(K_VSCAN, n_keys + 1);
            if (!flags || !vscan) return LFB_E_CUDA;
            k_u8_to_u32<<<(n_keys + 1 + 255) / 256, 256, 0, s>>>(used, flags, n_keys + 1);
            if (!exclusive_scan(flags, vscan, n_keys + 1, s)) return LFB_E_CUDA;
            uint32_t n_verts = 0;
            cudaMemcpyAsync(&n_verts, vscan + n_keys, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
            if (!cuda_ok(cudaStreamSynchronize(s), "vertex scan")) return LFB_E_CUDA;
            float* verts = ws.get<float>(K_VERTS, 3 * (static_cast<size_t>(n_verts) + 1));
            if (!verts) return LFB_E_CUDA;
            cudaMemsetAsync(verts, 0, 3 * sizeof(float), s);
            k_vertex_ids<<<(n_keys + 255) / 256, 256, 0, s>>>(used, vscan, n_keys, recs, verts);
            n_launch += 2;   // k_u8_to_u32 + k_vertex_ids
            if (n_tri) {
                k_remap_tris<<<(3 * n_tri + 255) / 256, 256, 0, s>>>(tris, n_tri, vscan);
                ++n_launch;
            }
            out.verts.resize(3 * (static_cast<size_t>(n_verts) + 1));
            out.tris.resize(3 * static_cast<size_t>(n_tri));
            cudaMemcpyAsync(out.verts.data(), verts, out.verts.size() * sizeof(float),
                            cudaMemcpyDeviceToHost, s);
            if (n_tri) {
                cudaMemcpyAsync(out.tris.data(), tris, out.tris.size() * sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, s);
            }
            if (!cuda_ok(cudaStreamSynchronize(s), "mesh download")) return LFB_E_CUDA;
            break;
        }
    }

    note_launches(n_launch);
    if (stats) {
        cudaEventRecord(ev[4], s);
        cudaEventSynchronize(ev[4]);
        unsigned long long ce[2] = {0, 0};
        cudaMemcpy(ce, evals, sizeof(ce), cudaMemcpyDeviceToHost);
        stats->levels = static_cast<uint32_t>(L);
        stats->cells_evaluated = cells_evaluated;
        stats->leaf_groups = n_leaf_groups;
        stats->leaves_ambiguous = n_recs;
        stats->clause_evals = ce[0];
        stats->clause_evals_grad = ce[1];
        stats->triangles = out.tris.size() / 3;
        stats->vertices = out.verts.size() / 3 - 1;
        stats->kernel_launches = n_launch;
        float ms[4];
        for (int k = 0; k < 4; ++k) cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]);
        stats->ms_interval = ms[0];
        stats->ms_leaf = ms[1];
        stats->ms_collapse = ms[2];
        stats->ms_dual = ms[3];
        for (auto& e : ev) cudaEventDestroy(e);
        stats->ms_total = std::chrono::duration<double, std::milli>(
                              std::chrono::steady_clock::now() - t_start).count();
    }
    return 0;
}

}  // namespace lfb
