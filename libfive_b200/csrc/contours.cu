// 2D contours of a slice z = perp (Contours::render, libfive/src/render/brep/
// contours.cpp:25-49) on the GPU: the quadtree form of the dual-contouring
// mesher.
//
//  * Quadtree build (DCWorkerPool<2>::build, DCTree<2>::evalInterval,
//    dc_tree.inl:94-128): level by level, one thread per cell evaluates the
//    cell's interval over its parent's pruned register tape and prunes it
//    for its children (Tape::push as liveness, like the mesher's group
//    kernel), with the interval register file in global scratch.
//  * Leaves (DCTree<2>::evalLeaf, dc_tree.inl:131-552 with N = 2): one warp
//    per cell; corners, edge search (four rounds of 16 samples per edge,
//    lanes over samples), gradients and features at the brackets, the
//    FP64 QEF solve (qef.h, qef2_*) on one lane.
//  * Collapse (DCTree<2>::collectChildren, dc_tree.inl:581-735 and
//    dc_tree2.cpp:14-46): one thread per branch cell, bottom-up.
//  * Dual walk (Dual<2>::work / edge2, dual.hpp:82-110) as breadth-first
//    rounds of edge tasks; DCContourer::load (dc_contourer.cpp:16-104)
//    writes one segment per sign-changing minimal edge.
//  * Contours::collect (contours.cpp:118-184): the segments are welded into
//    polylines on the host, in the reference's order of operations.
#include <algorithm>
#include <cmath>
#include <list>
#include <map>
#include <mutex>
#include <vector>

#include "contours.hpp"
#include "dc_device.cuh"
#include "dc_features.cuh"
#include "eval_kernels.cuh"
#include "libfive_b200.h"

namespace lfb {

namespace {

__constant__ DcTables2 c_tab2;

constexpr uint32_t kNone = 0xffffffffu;
constexpr int QX = 1, QY = 2;   // Axis::X, Axis::Y bits

/// One quadtree leaf (DCLeaf<2>): vertices, QEF, corner mask, rank, level.
struct QLeaf {
    double vert[2][2];
    Qef2 q;
    int32_t level;     // region level of a collapsed cell, 0 at the finest
    uint8_t mask;
    uint8_t nvert;
    uint8_t manifold;
    uint8_t rank;
};

/// Per depth: cells as (x, y) indices at that depth, the tape each is
/// evaluated with, its type (CELL_*), first child (branches) and leaf
/// record (ambiguous leaves).
struct QLevel {
    uint2* xy;
    TapeRef* tape;
    uint8_t* type;
    uint32_t* child;
    uint32_t* leaf;
    uint32_t n;
};

struct QTree {
    QLevel lv[kMaxLevels + 1];
    double lo[2], hi[2];
    float perp;
    int L;
};

__device__ __forceinline__ void qcell_bounds(const QTree& t, int d, uint2 xy, double lo[2],
                                             double hi[2])
{
    const uint32_t idx[2] = {xy.x, xy.y};
    for (int a = 0; a < 2; ++a) {
        double l = t.lo[a], h = t.hi[a];
        for (int b = d - 1; b >= 0; --b) {
            const double m = (l + h) / 2;
            if ((idx[a] >> b) & 1) l = m; else h = m;
        }
        lo[a] = l;
        hi[a] = h;
    }
}

////////////////////////////////////////////////////////////////////////////////
// Interval stage: one thread per cell

struct QIntervalArgs {
    QTree t;
    int d;
    DevTape bt;
    RegClause* arena;
    unsigned long long* arena_top;
    uint64_t arena_cap;
    TapeRef* out_tape;         // the pruned tape for the cell's children
    float* rlo;                // [nregs][T] interval registers
    float* rhi;
    uint8_t* rnan;
    uint8_t* live;             // [nregs][T] liveness flags
    uint8_t* dec;              // [dec_cap][T] min/max decisions
    uint32_t dec_cap;
    uint32_t T;
    uint32_t* status;
};

__global__ void __launch_bounds__(256)
k_q_interval(QIntervalArgs A)
{
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t T = A.T;
    const QLevel& lv = A.t.lv[A.d];
    const float* cp = A.bt.cpool;
    auto fetch = [&](uint32_t kind, uint32_t idx) -> Iv {
        if (kind == OPND_REG) {
            return {A.rlo[idx * T + tid], A.rhi[idx * T + tid], A.rnan[idx * T + tid] != 0};
        }
        const float v = __ldg(cp + idx);
        return iv_make(v, v);
    };
    for (uint32_t i = tid; i < lv.n; i += T) {
        const TapeRef tr = lv.tape[i];
        const RegClause* cl = A.arena + tr.off;
        const uint32_t rk = tr.root >> 16, rr = tr.root & 0xffff;
        double lo[2], hi[2];
        qcell_bounds(A.t, A.d, lv.xy[i], lo, hi);
        const Iv in[3] = {iv_make(static_cast<float>(lo[0]), static_cast<float>(hi[0])),
                          iv_make(static_cast<float>(lo[1]), static_cast<float>(hi[1])),
                          iv_make(A.t.perp, A.t.perp)};
        for (int a = 0; a < 3; ++a) {
            A.rlo[a * T + tid] = in[a].lo;
            A.rhi[a * T + tid] = in[a].hi;
            A.rnan[a * T + tid] = in[a].nan;
        }
        // Forward pass, recording the push decision of every min/max
        // (IntervalEvaluator::push, eval_interval.cpp:116-167).
        bool changed = false;
        uint32_t ch = 0;
        for (uint32_t c = 0; c < tr.len; ++c) {
            const uint2 raw = __ldg(reinterpret_cast<const uint2*>(cl + c));
            const uint8_t o = raw.x & 0xff;
            const uint32_t kinds = (raw.x >> 8) & 0xff;
            const uint32_t ro = raw.x >> 16;
            const Iv a = fetch(kinds & 3, raw.y & 0xffff);
            const Iv b = fetch((kinds >> 2) & 3, raw.y >> 16);
            const Iv r = iv_apply(o, a, b);
            if (o == op::MIN || o == op::MAX) {
                uint8_t keep = 0;   // 0 both, 1 a, 2 b
                if (a.lo > b.hi) keep = (o == op::MAX) ? 1 : 2;
                else if (b.lo > a.hi) keep = (o == op::MAX) ? 2 : 1;
                changed |= keep != 0;
                if (ch < A.dec_cap) A.dec[static_cast<size_t>(ch) * T + tid] = keep;
                ++ch;
            }
            A.rlo[ro * T + tid] = r.lo;
            A.rhi[ro * T + tid] = r.hi;
            A.rnan[ro * T + tid] = r.nan;
        }
        const Iv root = fetch(rk, rr);
        const uint8_t state = iv_state(root);
        lv.type[i] = state == ST_EMPTY ? CELL_EMPTY : state == ST_FILLED ? CELL_FILLED
                                                                          : CELL_BRANCH;
        A.out_tape[i] = tr;
        if (state != ST_AMBIGUOUS || root.nan || !changed) continue;
        if (ch > A.dec_cap) {
            atomicOr(A.status, ST_REGS);
            continue;
        }
        // Backward liveness pass: count, then allocate and write the kept
        // clauses from the back (they stay in evaluation order).
        uint32_t kept = 0;
        for (int pass = 0; pass < 2; ++pass) {
            for (uint32_t r = 0; r < tr.nregs; ++r) A.live[r * T + tid] = 0;
            if (rk == OPND_REG) A.live[rr * T + tid] = 1;
            uint32_t pos = kept;
            uint32_t chi = ch;
            unsigned long long off = 0;
            if (pass == 1) {
                off = atomicAdd(A.arena_top, static_cast<unsigned long long>(kept));
                if (off + kept > A.arena_cap) {
                    atomicOr(A.status, ST_ARENA_OVERFLOW);
                    break;
                }
            }
            for (int64_t c = static_cast<int64_t>(tr.len) - 1; c >= 0; --c) {
                const uint2 raw = __ldg(reinterpret_cast<const uint2*>(cl + c));
                const uint8_t o = raw.x & 0xff;
                const uint32_t kinds = (raw.x >> 8) & 0xff;
                const uint32_t ro = raw.x >> 16;
                uint8_t keep = 0;
                if (o == op::MIN || o == op::MAX) keep = A.dec[static_cast<size_t>(--chi) * T + tid];
                if (!A.live[ro * T + tid]) continue;
                A.live[ro * T + tid] = 0;
                uint2 outc = raw;
                bool emit = true;
                if (keep) {
                    const uint32_t k = keep == 1 ? (kinds & 3) : ((kinds >> 2) & 3);
                    const uint32_t src = keep == 1 ? (raw.y & 0xffff) : (raw.y >> 16);
                    if (k == OPND_REG) {
                        A.live[src * T + tid] = 1;
                        emit = src != ro;
                    }
                    outc.x = OP_COPY | (k << 8) | (ro << 16);
                    outc.y = src;
                } else {
                    if ((kinds & 3) == OPND_REG) A.live[(raw.y & 0xffff) * T + tid] = 1;
                    if (dev_is_binary(o) && ((kinds >> 2) & 3) == OPND_REG) {
                        A.live[(raw.y >> 16) * T + tid] = 1;
                    }
                }
                if (!emit) continue;
                if (pass == 0) {
                    ++kept;
                } else {
                    *reinterpret_cast<uint2*>(A.arena + off + (--pos)) = outc;
                }
            }
            if (pass == 1) A.out_tape[i] = {static_cast<uint32_t>(off), kept, tr.nregs, tr.root};
        }
    }
}

/// Children of the branch cells of depth d: four each, in the order of
/// Region::subdivide (bit 0 = x upper half, bit 1 = y upper half), with
/// their parent's pruned tape.
__global__ void k_q_children(QTree t, int d, const uint32_t* scan, const TapeRef* out_tape)
{
    const QLevel& lv = t.lv[d];
    const QLevel& nx = t.lv[d + 1];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= lv.n) return;
    lv.leaf[i] = kNone;
    if (lv.type[i] != CELL_BRANCH) {
        lv.child[i] = kNone;
        return;
    }
    const uint32_t c0 = 4 * scan[i];
    lv.child[i] = c0;
    const uint2 p = lv.xy[i];
    for (uint32_t k = 0; k < 4; ++k) {
        nx.xy[c0 + k] = make_uint2(2 * p.x + (k & 1), 2 * p.y + ((k >> 1) & 1));
        nx.tape[c0 + k] = out_tape[i];
    }
}

__global__ void k_q_branch_flags(const uint8_t* type, uint32_t n, uint32_t* flags)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[i] = type[i] == CELL_BRANCH ? 1u : 0u;
}

////////////////////////////////////////////////////////////////////////////////
// Leaves: one warp per cell

/// Values at one point per lane (register file R: [nregs][32] floats), and
/// whether some min/max of the tape has equal arguments there
/// (ArrayEvaluator::getAmbiguous, eval_array.cpp:198-217).
__device__ float q_value(const DevTape& tb, const RegClause* cl, uint32_t len, float* R,
                         int lane, float x, float y, float z, bool* amb)
{
    R[0 * 32 + lane] = x;
    R[1 * 32 + lane] = y;
    R[2 * 32 + lane] = z;
    bool tie = false;
    for (uint32_t c = 0; c < len; ++c) {
        const uint2 raw = __ldg(reinterpret_cast<const uint2*>(cl + c));
        const uint8_t o = raw.x & 0xff;
        const uint32_t kinds = (raw.x >> 8) & 0xff;
        const uint32_t ro = raw.x >> 16;
        const uint32_t ia = raw.y & 0xffff, ib = raw.y >> 16;
        const float a = (kinds & 3) == OPND_REG ? R[ia * 32 + lane] : __ldg(tb.cpool + ia);
        const float b = ((kinds >> 2) & 3) == OPND_REG ? R[ib * 32 + lane] : __ldg(tb.cpool + ib);
        if (o == op::MIN || o == op::MAX) tie |= a == b;
        R[ro * 32 + lane] = dv_value(o, a, b);
    }
    *amb = tie;
    return tb.root_kind == OPND_REG ? R[tb.root * 32 + lane] : __ldg(tb.cpool + tb.root);
}

/// Value and d/dx, d/dy, d/dz at one point per lane (R: [nregs][4][32]),
/// with the ambiguity of the values.
__device__ D4 q_deriv(const DevTape& tb, const RegClause* cl, uint32_t len, float* R, int lane,
                      float x, float y, float z, bool* amb)
{
    auto put = [&](uint32_t r, const D4& d) {
        R[(r * 4 + 0) * 32 + lane] = d.v;
        R[(r * 4 + 1) * 32 + lane] = d.dx;
        R[(r * 4 + 2) * 32 + lane] = d.dy;
        R[(r * 4 + 3) * 32 + lane] = d.dz;
    };
    auto get = [&](uint32_t kind, uint32_t idx) -> D4 {
        if (kind == OPND_REG) {
            return {R[(idx * 4 + 0) * 32 + lane], R[(idx * 4 + 1) * 32 + lane],
                    R[(idx * 4 + 2) * 32 + lane], R[(idx * 4 + 3) * 32 + lane]};
        }
        return {__ldg(tb.cpool + idx), 0.0f, 0.0f, 0.0f};
    };
    put(0, {x, 1.0f, 0.0f, 0.0f});
    put(1, {y, 0.0f, 1.0f, 0.0f});
    put(2, {z, 0.0f, 0.0f, 1.0f});
    bool tie = false;
    for (uint32_t c = 0; c < len; ++c) {
        const uint2 raw = __ldg(reinterpret_cast<const uint2*>(cl + c));
        const uint8_t o = raw.x & 0xff;
        const uint32_t kinds = (raw.x >> 8) & 0xff;
        const D4 a = get(kinds & 3, raw.y & 0xffff);
        const D4 b = get((kinds >> 2) & 3, raw.y >> 16);
        if (o == op::MIN || o == op::MAX) tie |= a.v == b.v;
        put(raw.x >> 16, dv_deriv(o, a, b, false));
    }
    *amb = tie;
    return get(tb.root_kind, tb.root);
}

/// FeatureEvaluator::features (eval_feature.cpp:125-169), warp-collective:
/// pushes every distinct feature gradient at p into q (Intersection::push
/// with the sample's value).
__device__ void q_push_features(const FeatCtx& fc, const DevTape& tb, const RegClause* cl,
                                uint32_t len, const double p[2], float z, double value,
                                Qef2* q, int lane)
{
    __syncwarp();
    if (lane == 0) {
        float v;
        const float* fs;
        int n;
        feat_eval(fc, tb, cl, len, static_cast<float>(p[0]), static_cast<float>(p[1]), z, &v, &fs,
                  &n);
        for (int i = 0; i < n; ++i) {
            const float* f = fs + i * kFeatFloats;
            bool seen = false;
            for (int j = 0; j < i && !seen; ++j) seen = vcmp3(f, fs + j * kFeatFloats) == 0;
            if (seen) continue;
            const double g[2] = {f[0], f[1]};
            qef2_push(*q, p, g, value);
        }
        feat_done(fc);
    } else {
        feat_serve(fc, lane);
    }
    __syncwarp();
}

constexpr int kLeafWarps = 4;

struct QLeafShared {
    double ps[64][2];
    double tg[4][2][2];
    float out[64];
    Qef2 inter[8];
    uint8_t used[8];
};

struct QLeafArgs {
    QTree t;
    DevTape bt;
    const RegClause* arena;
    float* regs;               // [warps][nregs][4][32]
    uint32_t nregs;
    float* featws;             // [warps][nregs * kRegBlock]
    FeatureScratch* fscratch;  // [warps]
    QLeaf* recs;
    uint32_t* rec_top;
    uint32_t rec_cap;
    uint32_t* status;
};

__global__ void __launch_bounds__(32 * kLeafWarps)
k_q_leaf(QLeafArgs A)
{
    __shared__ QLeafShared S_all[kLeafWarps];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const uint32_t warp = blockIdx.x * kLeafWarps + wib;
    const uint32_t n_warps = gridDim.x * kLeafWarps;
    QLeafShared& S = S_all[wib];
    float* R = A.regs + static_cast<size_t>(warp) * A.nregs * 4 * 32;
    const FeatCtx fc{A.featws + static_cast<size_t>(warp) * A.bt.n_regs * kRegBlock,
                     A.fscratch + warp, A.status};
    const int d = A.t.L;
    const QLevel& lv = A.t.lv[d];
    const float z = A.t.perp;

    for (uint32_t i = warp; i < lv.n; i += n_warps) {
        const TapeRef tr = lv.tape[i];
        const DevTape tb = with_tape(A.bt, tr);
        const RegClause* cl = A.arena + tr.off;
        double lo[2], hi[2];
        qcell_bounds(A.t, d, lv.xy[i], lo, hi);

        // corners (dc_tree.inl:156-239)
        const int ci = lane & 3;
        const float cx = static_cast<float>((ci & 1) ? hi[0] : lo[0]);
        const float cy = static_cast<float>((ci & 2) ? hi[1] : lo[1]);
        bool amb = false;
        const float v = q_value(tb, cl, tr.len, R, lane, cx, cy, z, &amb);
        uint8_t cst = CELL_EMPTY;
        bool need_d = false, need_f = false;
        if (lane < 4) {
            if (v > 0 || v != v) cst = CELL_EMPTY;
            else if (v < 0) cst = CELL_FILLED;
            else if (!amb) need_d = true;
            else need_f = true;
        }
        if (__any_sync(0xffffffffu, need_d)) {
            bool a2 = false;
            const D4 g = q_deriv(tb, cl, tr.len, R, lane, cx, cy, z, &a2);
            if (need_d) cst = (g.dx != 0 || g.dy != 0 || g.dz != 0) ? CELL_FILLED : CELL_EMPTY;
        }
        uint32_t pending = __ballot_sync(0xffffffffu, need_f);
        while (pending) {
            const int src = __ffs(pending) - 1;
            pending &= pending - 1;
            const float qx = __shfl_sync(0xffffffffu, cx, src);
            const float qy = __shfl_sync(0xffffffffu, cy, src);
            const bool in = dev_is_inside(fc, tb, cl, tr.len, qx, qy, z, lane);
            if (lane == src) cst = in ? CELL_FILLED : CELL_EMPTY;
        }
        const uint32_t filled = __ballot_sync(0xffffffffu, lane < 4 && cst == CELL_FILLED) & 0xf;
        if (filled == 0 || filled == 0xf) {
            if (lane == 0) {
                lv.type[i] = filled ? CELL_FILLED : CELL_EMPTY;
                lv.leaf[i] = kNone;
            }
            continue;
        }
        const uint32_t mask = filled;
        uint32_t rec = 0;
        if (lane == 0) rec = atomicAdd(A.rec_top, 1u);
        rec = __shfl_sync(0xffffffffu, rec, 0);
        if (rec >= A.rec_cap) {
            if (lane == 0) {
                atomicOr(A.status, ST_RECORD_OVERFLOW);
                lv.type[i] = CELL_LEAF;
                lv.leaf[i] = kNone;
            }
            continue;
        }
        if (lane < 8) {
            qef2_zero(S.inter[lane]);
            S.used[lane] = 0;
        }
        __syncwarp();
        QLeaf L{};
        L.mask = static_cast<uint8_t>(mask);
        L.manifold = c_tab2.manifold[mask];
        L.level = 0;
        const int npatch = c_tab2.npatch[mask];
        for (int patch = 0; patch < npatch; ++patch) {
            const int ne = c_tab2.nedge[mask][patch];
            int edges[4];
            for (int k = 0; k < ne; ++k) {
                const int a = c_tab2.v[mask][patch][k][0];
                const int b = c_tab2.v[mask][patch][k][1];
                edges[k] = c_tab2.e[a][b];
                if (lane == 0) {
                    S.tg[k][0][0] = (a & 1) ? hi[0] : lo[0];
                    S.tg[k][0][1] = (a & 2) ? hi[1] : lo[1];
                    S.tg[k][1][0] = (b & 1) ? hi[0] : lo[0];
                    S.tg[k][1][1] = (b & 2) ? hi[1] : lo[1];
                }
            }
            __syncwarp();
            // edge search (dc_tree.inl:339-410)
            for (int s = 0; s < 4; ++s) {
                for (int h = 0; h < 2; ++h) {
                    const int idx = lane + 32 * h;
                    const int k = idx / 16, j = idx % 16;
                    if (k < ne) {
                        const double frac = j / (16 - 1.0);
                        for (int a = 0; a < 2; ++a) {
                            S.ps[idx][a] = S.tg[k][0][a] * (1 - frac) + S.tg[k][1][a] * frac;
                        }
                    }
                }
                __syncwarp();
                for (int h = 0; h < 2 && 32 * h < 16 * ne; ++h) {
                    const int idx = lane + 32 * h;
                    const bool on = idx < 16 * ne;
                    const float px = static_cast<float>(on ? S.ps[idx][0] : S.ps[0][0]);
                    const float py = static_cast<float>(on ? S.ps[idx][1] : S.ps[0][1]);
                    bool a2 = false;
                    const float o = q_value(tb, cl, tr.len, R, lane, px, py, z, &a2);
                    if (on) S.out[idx] = o;
                }
                __syncwarp();
                for (int k = 0; k < ne; ++k) {
                    for (int j = 1; j < 16; ++j) {
                        const int idx = j + 16 * k;
                        const float o = S.out[idx];
                        bool hit = false;
                        if (o > 0) {
                            hit = true;
                        } else if (o == 0) {
                            hit = !dev_is_inside(fc, tb, cl, tr.len, static_cast<float>(S.ps[idx][0]),
                                                 static_cast<float>(S.ps[idx][1]), z, lane);
                        } else if (j == 15) {
                            hit = true;
                        }
                        if (hit) {
                            if (lane == 0) {
                                for (int a = 0; a < 2; ++a) {
                                    S.tg[k][0][a] = S.ps[idx - 1][a];
                                    S.tg[k][1][a] = S.ps[idx][a];
                                }
                            }
                            break;
                        }
                    }
                }
                __syncwarp();
            }
            // value and derivatives at both ends of each bracket
            const bool on = lane < 2 * ne;
            const int kk = on ? lane / 2 : 0, side = on ? (lane & 1) : 0;
            const double pxd = S.tg[kk][side][0], pyd = S.tg[kk][side][1];
            bool a2 = false;
            const D4 g = q_deriv(tb, cl, tr.len, R, lane, static_cast<float>(pxd),
                                 static_cast<float>(pyd), z, &a2);
            for (int q = 0; q < 2 * ne; ++q) {
                const int k = q / 2;
                const bool qa = __shfl_sync(0xffffffffu, a2, q);
                const float gv = __shfl_sync(0xffffffffu, g.v, q);
                const float gx = __shfl_sync(0xffffffffu, g.dx, q);
                const float gy = __shfl_sync(0xffffffffu, g.dy, q);
                const double p[2] = {S.tg[k][q & 1][0], S.tg[k][q & 1][1]};
                Qef2* it = &S.inter[edges[k]];
                if (!qa) {
                    if (lane == 0) {
                        const double gd[2] = {gx, gy};
                        qef2_push(*it, p, gd, static_cast<double>(gv));
                        S.used[edges[k]] = 1;
                    }
                } else {
                    q_push_features(fc, tb, cl, tr.len, p, z, static_cast<double>(gv), it, lane);
                    if (lane == 0) S.used[edges[k]] = 1;
                }
                __syncwarp();
            }
            // mass point from the max-rank intersections, the QEF sums and
            // the vertex (one lane, FP64)
            if (lane == 0) {
                Qef2 q;
                qef2_zero(q);
                int max_rank = 0;
                for (int k = 0; k < ne; ++k) {
                    if (S.used[edges[k]]) max_rank = max(max_rank, qef2_rank(S.inter[edges[k]]));
                }
                for (int k = 0; k < ne; ++k) {
                    const Qef2& it = S.inter[edges[k]];
                    if (S.used[edges[k]] && qef2_rank(it) == max_rank) {
                        for (int a = 0; a < 2; ++a) q.mass[a] += it.mass[a] / it.mass[2];
                        q.mass[2] += 1.0;
                    }
                }
                for (int k = 0; k < ne; ++k) {
                    if (S.used[edges[k]]) qef2_add(q, S.inter[edges[k]]);
                }
                int rank = 0;
                qef2_vertex(q, L.vert[patch], &rank);
                L.rank = static_cast<uint8_t>(rank);
                L.q = q;
                L.nvert = static_cast<uint8_t>(patch + 1);
            }
            __syncwarp();
        }
        if (lane == 0) {
            A.recs[rec] = L;
            lv.type[i] = CELL_LEAF;
            lv.leaf[i] = rec;
        }
    }
}

////////////////////////////////////////////////////////////////////////////////
// Collapse: one thread per branch cell of one depth

__device__ __forceinline__ int q_corner_state(const QTree& t, const QLeaf* recs, int d, uint32_t i,
                                              int corner)
{
    const QLevel& lv = t.lv[d];
    const uint8_t ty = lv.type[i];
    if (ty == CELL_LEAF) {
        const uint32_t r = lv.leaf[i];
        return r == kNone ? CELL_EMPTY : (((recs[r].mask >> corner) & 1) ? CELL_FILLED : CELL_EMPTY);
    }
    return ty;
}

struct QCollapseArgs {
    QTree t;
    int d;
    DevTape bt;                // the unpruned tape
    const RegClause* arena;    // the unpruned and pruned tapes
    QLeaf* recs;
    uint32_t* rec_top;
    uint32_t rec_cap;
    double max_err;
    float* regs;               // [nregs][T]
    uint32_t T;
    uint32_t* status;
};

__global__ void k_q_collapse(QCollapseArgs A)
{
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const QLevel& lv = A.t.lv[A.d];
    const QLevel& nx = A.t.lv[A.d + 1];
    for (uint32_t i = tid; i < lv.n; i += A.T) {
        if (lv.type[i] != CELL_BRANCH) continue;
        const uint32_t c0 = lv.child[i];
        bool any_branch = false, all_empty = true, all_full = true;
        int corners[4];
        for (int k = 0; k < 4; ++k) {
            const uint8_t ty = nx.type[c0 + k];
            any_branch |= ty == CELL_BRANCH;
            all_empty &= ty == CELL_EMPTY;
            all_full &= ty == CELL_FILLED;
        }
        if (any_branch) continue;
        for (int k = 0; k < 4; ++k) corners[k] = q_corner_state(A.t, A.recs, A.d + 1, c0 + k, k);
        if (all_empty || all_full) {
            lv.type[i] = all_empty ? CELL_EMPTY : CELL_FILLED;
            lv.child[i] = kNone;
            continue;
        }
        uint32_t mask = 0;
        for (int k = 0; k < 4; ++k) mask |= (corners[k] == CELL_FILLED ? 1u : 0u) << k;
        bool manifold = c_tab2.manifold[mask] != 0;
        int rank = 0;
        for (int k = 0; k < 4; ++k) {
            if (nx.type[c0 + k] == CELL_LEAF) {
                const uint32_t r = nx.leaf[c0 + k];
                if (r == kNone) {
                    manifold = false;
                    continue;
                }
                manifold = manifold && A.recs[r].manifold;
                rank = max(rank, static_cast<int>(A.recs[r].rank));
            }
        }
        // leafsAreManifold<2> (dc_tree2.cpp:22-46)
        auto cs = [&](int child, int corner) {
            return q_corner_state(A.t, A.recs, A.d + 1, c0 + child, corner);
        };
        const bool edges_safe =
            (cs(0, QX) == corners[0] || cs(0, QX) == corners[QX]) &&
            (cs(0, QY) == corners[0] || cs(0, QY) == corners[QY]) &&
            (cs(QX, QX | QY) == corners[QX] || cs(QX, QX | QY) == corners[QX | QY]) &&
            (cs(QY, QY | QX) == corners[QY] || cs(QY, QY | QX) == corners[QY | QX]);
        const int m = cs(0, QX | QY);
        const bool faces_safe = m == corners[0] || m == corners[QY] || m == corners[QX] ||
                                m == corners[QX | QY];
        if (!manifold || !edges_safe || !faces_safe) continue;

        Qef2 q;
        qef2_zero(q);
        for (int k = 0; k < 4; ++k) {
            if (nx.type[c0 + k] != CELL_LEAF) continue;
            const QLeaf& c = A.recs[nx.leaf[c0 + k]];
            if (c.rank == rank) {
                for (int a = 0; a < 3; ++a) q.mass[a] += c.q.mass[a];
            }
            qef2_add(q, c.q);
        }
        double v[2];
        const double err = qef2_vertex(q, v, nullptr);
        double lo[2], hi[2];
        qcell_bounds(A.t, A.d, lv.xy[i], lo, hi);
        bool inside = true;
        for (int a = 0; a < 2; ++a) inside = inside && v[a] >= lo[a] - 1e-6 && v[a] <= hi[a] + 1e-6;
        if (!(err < A.max_err && inside)) continue;
        // Value at the vertex with a tape valid there (Tape::getBase,
        // tape.cpp:188-209): every valid tape gives the same value, so the
        // shortest is taken: the one pruned over this cell's box (its
        // children's) when the vertex lies in that box, else the unpruned.
        const float vx = static_cast<float>(v[0]), vy = static_cast<float>(v[1]);
        const bool in_cell = vx >= static_cast<float>(lo[0]) && vx <= static_cast<float>(hi[0]) &&
                             vy >= static_cast<float>(lo[1]) && vy <= static_cast<float>(hi[1]);
        const TapeRef tr = in_cell ? nx.tape[c0] : root_tape_ref(A.bt);
        const RegClause* cl = A.arena + tr.off;
        const uint32_t rk = tr.root >> 16, rr = tr.root & 0xffff;
        float* R = A.regs;
        const uint32_t T = A.T;
        R[0 * T + tid] = vx;
        R[1 * T + tid] = vy;
        R[2 * T + tid] = A.t.perp;
        const float* cp = A.bt.cpool;
        for (uint32_t c = 0; c < tr.len; ++c) {
            const RegClause k = cl[c];
            const uint8_t ka = k.kinds & 3, kb = (k.kinds >> 2) & 3;
            const float a = ka == OPND_REG ? R[k.a * T + tid] : __ldg(cp + k.a);
            const float b = kb == OPND_REG ? R[k.b * T + tid] : __ldg(cp + k.b);
            R[k.out * T + tid] = dv_value(k.op, a, b);
        }
        const float value = rk == OPND_REG ? R[rr * T + tid] : __ldg(cp + rr);
        if (!(fabsf(value) < A.max_err)) continue;
        const uint32_t rec = atomicAdd(A.rec_top, 1u);
        if (rec >= A.rec_cap) {
            atomicOr(A.status, ST_RECORD_OVERFLOW);
            continue;
        }
        QLeaf L{};
        L.vert[0][0] = v[0];
        L.vert[0][1] = v[1];
        L.q = q;
        L.level = A.t.L - A.d;
        L.mask = static_cast<uint8_t>(mask);
        L.nvert = 1;
        L.manifold = 1;
        L.rank = static_cast<uint8_t>(rank);
        A.recs[rec] = L;
        lv.type[i] = CELL_LEAF;
        lv.leaf[i] = rec;
        lv.child[i] = kNone;
    }
}

////////////////////////////////////////////////////////////////////////////////
// Dual walk: breadth-first rounds of edge tasks

/// An edge task: axis A, two cells (depth, index).
struct QTask {
    uint32_t a;        // A | d0 << 8 | d1 << 16
    uint32_t i0, i1;
};

__device__ __forceinline__ void q_kid(const QTree& t, int d, uint32_t i, int k, int* od,
                                      uint32_t* oi)
{
    if (t.lv[d].type[i] == CELL_BRANCH) {
        *od = d + 1;
        *oi = t.lv[d].child[i] + k;
    } else {
        *od = d;
        *oi = i;
    }
}

__device__ __forceinline__ void q_push_task(QTask* q, uint32_t* n, uint32_t cap, uint32_t* status,
                                            int A, int d0, uint32_t i0, int d1, uint32_t i1)
{
    const uint32_t k = atomicAdd(n, 1u);
    if (k >= cap) {
        atomicOr(status, ST_QUEUE_OVERFLOW);
        return;
    }
    q[k] = {static_cast<uint32_t>(A) | (static_cast<uint32_t>(d0) << 8) |
                (static_cast<uint32_t>(d1) << 16),
            i0, i1};
}

struct QDualArgs {
    QTree t;
    const QLeaf* recs;
    QTask* out;
    uint32_t* n_out;
    uint32_t cap;
    uint2* segs;
    uint32_t* n_segs;
    uint32_t seg_cap;
    uint32_t* status;
};

/// Dual<2>::work of every branch cell of depth d: its four inner edges.
__global__ void k_q_dual_init(QDualArgs D, int d)
{
    const QLevel& lv = D.t.lv[d];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= lv.n || lv.type[i] != CELL_BRANCH) return;
    const uint32_t c0 = lv.child[i];
    const int e = d + 1;
    q_push_task(D.out, D.n_out, D.cap, D.status, QY, e, c0 + 0, e, c0 + QX);
    q_push_task(D.out, D.n_out, D.cap, D.status, QY, e, c0 + QY, e, c0 + (QY | QX));
    q_push_task(D.out, D.n_out, D.cap, D.status, QX, e, c0 + 0, e, c0 + QY);
    q_push_task(D.out, D.n_out, D.cap, D.status, QX, e, c0 + QX, e, c0 + (QX | QY));
}

__global__ void k_q_dual_round(QDualArgs D, const QTask* in, uint32_t n_in)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_in) return;
    const QTask task = in[k];
    const int A = task.a & 0xff;
    const int d0 = (task.a >> 8) & 0xff, d1 = (task.a >> 16) & 0xff;
    const uint32_t i0 = task.i0, i1 = task.i1;
    const int perp = (QX | QY) ^ A;
    const uint8_t t0 = D.t.lv[d0].type[i0], t1 = D.t.lv[d1].type[i1];
    if (t0 == CELL_BRANCH || t1 == CELL_BRANCH) {
        // edge2 (dual.hpp:82-97)
        int a0, a1, b0, b1;
        uint32_t j0, j1, m0, m1;
        q_kid(D.t, d0, i0, perp, &a0, &j0);
        q_kid(D.t, d1, i1, 0, &a1, &j1);
        q_kid(D.t, d0, i0, A | perp, &b0, &m0);
        q_kid(D.t, d1, i1, A, &b1, &m1);
        q_push_task(D.out, D.n_out, D.cap, D.status, A, a0, j0, a1, j1);
        q_push_task(D.out, D.n_out, D.cap, D.status, A, b0, m0, b1, m1);
        return;
    }
    if (t0 != CELL_LEAF || t1 != CELL_LEAF) return;
    const uint32_t r[2] = {D.t.lv[d0].leaf[i0], D.t.lv[d1].leaf[i1]};
    if (r[0] == kNone || r[1] == kNone) return;
    // DCContourer::load<A> (dc_contourer.cpp:16-60)
    const QLeaf* L[2] = {D.recs + r[0], D.recs + r[1]};
    const int index = L[1]->level < L[0]->level ? 1 : 0;
    const int corners[2] = {perp, 0};
    const int ca = (L[index]->mask >> corners[index]) & 1;
    const int cb = (L[index]->mask >> (corners[index] | A)) & 1;
    if (ca == cb) return;
    const bool fwd = (ca && A == QY) || (cb && A == QX);
    const bool Dd = !fwd;
    // DCContourer::load<A, D> (dc_contourer.cpp:63-104)
    int es[2];
    if (Dd ^ (A == QX)) {
        es[0] = c_tab2.e[3][3 ^ A];
        es[1] = c_tab2.e[A][0];
    } else {
        es[0] = c_tab2.e[3 ^ A][3];
        es[1] = c_tab2.e[0][A];
    }
    uint32_t vs[2];
    for (int j = 0; j < 2; ++j) {
        const int vi = L[j]->level > 0 ? 0 : c_tab2.p[L[j]->mask][es[j]];
        vs[j] = r[j] * 2 + static_cast<uint32_t>(vi < 0 ? 0 : vi);
    }
    const uint32_t s = atomicAdd(D.n_segs, 1u);
    if (s >= D.seg_cap) {
        atomicOr(D.status, ST_QUEUE_OVERFLOW);
        return;
    }
    // {vs[!D], vs[D]}: the winding of dc_contourer.cpp:102
    D.segs[s] = make_uint2(vs[Dd ? 0 : 1], vs[Dd ? 1 : 0]);
}

bool upload_tables2()
{
    static std::mutex mu;
    static uint64_t ready = 0;   // one bit per device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 64 && ((ready >> dev) & 1)) return true;
    DcTables2 t;
    build_dc_tables2(t);
    if (!cuda_ok(cudaMemcpyToSymbol(c_tab2, &t, sizeof(t)), "contour tables")) return false;
    if (dev < 64) ready |= 1ull << dev;
    return true;
}

}  // namespace

/// Contours::collect (contours.cpp:118-184): directed segments welded into
/// polylines, first by extending a polyline whose tail is the segment's
/// start, else one whose head is its end, else starting a new one; then
/// polylines are joined forward through their heads.
void weld_segments(const std::vector<std::pair<uint32_t, uint32_t>>& segs,
                   std::vector<std::vector<uint32_t>>& out)
{
    std::map<uint32_t, uint32_t> heads, tails;
    std::vector<std::list<uint32_t>> cs;
    for (const auto& s : segs) {
        auto t = tails.find(s.first);
        if (t != tails.end()) {
            const uint32_t k = t->second;
            cs[k].push_back(s.second);
            tails.insert({s.second, k});
            tails.erase(t);
            continue;
        }
        auto h = heads.find(s.second);
        if (h != heads.end()) {
            const uint32_t k = h->second;
            cs[k].push_front(s.first);
            heads.insert({s.first, k});
            heads.erase(h);
            continue;
        }
        heads[s.first] = static_cast<uint32_t>(cs.size());
        tails[s.second] = static_cast<uint32_t>(cs.size());
        cs.push_back({s.first, s.second});
    }
    std::vector<bool> done(cs.size(), false);
    for (size_t i = 0; i < cs.size(); ++i) {
        if (done[i]) continue;
        out.emplace_back();
        size_t target = i;
        for (;;) {
            for (uint32_t p : cs[target]) out.back().push_back(p);
            done[target] = true;
            auto h = heads.find(cs[target].back());
            if (h != heads.end() && !done[h->second]) {
                out.back().pop_back();
                target = h->second;
            } else {
                break;
            }
        }
    }
}

int render_contours(GpuTape& g, const double lo[2], const double hi[2], double z,
                    double min_feature, double max_err, ContoursOut& out)
{
    if (!require_device()) return LFB_E_CUDA;
    if (!g.on_current_device()) {
        return set_error(LFB_E_INVALID, "tape was created on another device");
    }
    if (!upload_tables2()) return LFB_E_CUDA;
    out.pts.clear();
    out.counts.clear();
    // Region<2>::withResolution (region.hpp:226-231)
    const double md = std::min(hi[0] - lo[0], hi[1] - lo[1]);
    const int L = static_cast<int>(
        std::ceil(std::fmax(0.0f, std::log(static_cast<float>(md / min_feature))) /
                  std::log(2.0f)));
    if (L > kMaxLevels) return set_error(LFB_E_INVALID, "slice resolution too fine");

    const DevTape bt = g.dev();
    const uint32_t nregs = std::max<uint32_t>(bt.n_regs, 3);
    const uint32_t dec_cap = std::max<uint32_t>(bt.n_choices, 1);
    const int sms = device_sm_count();
    const uint32_t T = static_cast<uint32_t>(sms) * 256;
    const uint32_t leaf_warps = static_cast<uint32_t>(sms) * 8;
    cudaStream_t s = 0;

    uint64_t arena_cap = std::max<uint64_t>(static_cast<uint64_t>(bt.n) * 64, 1u << 20);
    uint32_t rec_cap = 1u << 16, task_cap = 1u << 18, seg_cap = 1u << 16;
    for (int attempt = 0; attempt < 4; ++attempt) {
        DevBuf b_arena, b_ctr, b_rlo, b_rhi, b_rnan, b_live, b_dec, b_out_tape, b_scan, b_flags;
        DevBuf b_regs, b_featws, b_fs, b_recs, b_tasks_a, b_tasks_b, b_segs, b_cregs;
        std::vector<DevBuf> lv_bufs(static_cast<size_t>(L) + 1);
        const size_t tr_bytes = static_cast<size_t>(nregs) * T;
        if (!b_arena.reserve(arena_cap * sizeof(RegClause)) || !b_ctr.reserve(64) ||
            !b_rlo.reserve(tr_bytes * 4) || !b_rhi.reserve(tr_bytes * 4) ||
            !b_rnan.reserve(tr_bytes) || !b_live.reserve(tr_bytes) ||
            !b_dec.reserve(static_cast<size_t>(dec_cap) * T) ||
            !b_regs.reserve(static_cast<size_t>(leaf_warps) * nregs * 4 * 32 * sizeof(float)) ||
            !b_featws.reserve(static_cast<size_t>(leaf_warps) * bt.n_regs * kRegBlock * sizeof(float) + 16) ||
            !b_fs.reserve(static_cast<size_t>(leaf_warps) * sizeof(FeatureScratch)) ||
            !b_recs.reserve(static_cast<size_t>(rec_cap) * sizeof(QLeaf)) ||
            !b_tasks_a.reserve(static_cast<size_t>(task_cap) * sizeof(QTask)) ||
            !b_tasks_b.reserve(static_cast<size_t>(task_cap) * sizeof(QTask)) ||
            !b_segs.reserve(static_cast<size_t>(seg_cap) * sizeof(uint2)) ||
            !b_cregs.reserve(tr_bytes * 4)) {
            return LFB_E_CUDA;
        }
        RegClause* arena = b_arena.as<RegClause>();
        unsigned long long* ctr = b_ctr.as<unsigned long long>();
        // ctr[0] arena top, [1] record top (u32), [2] status (u32), [3] task
        // count, [4] segment count
        unsigned long long* arena_top = ctr;
        uint32_t* rec_top = reinterpret_cast<uint32_t*>(ctr + 1);
        uint32_t* status = reinterpret_cast<uint32_t*>(ctr + 2);
        uint32_t* n_tasks = reinterpret_cast<uint32_t*>(ctr + 3);
        uint32_t* n_segs = reinterpret_cast<uint32_t*>(ctr + 4);
        cudaMemsetAsync(ctr, 0, 64, s);
        if (bt.n) {
            cudaMemcpyAsync(arena, bt.clauses, bt.n * sizeof(RegClause), cudaMemcpyDeviceToDevice, s);
        }
        const unsigned long long top0 = bt.n;
        cudaMemcpyAsync(arena_top, &top0, sizeof(top0), cudaMemcpyHostToDevice, s);

        QTree t{};
        t.lo[0] = lo[0]; t.lo[1] = lo[1];
        t.hi[0] = hi[0]; t.hi[1] = hi[1];
        t.perp = static_cast<float>(z);
        t.L = L;
        auto alloc_level = [&](int d, uint32_t n) {
            const size_t m = std::max<uint32_t>(n, 1);
            const size_t bytes = m * (sizeof(uint2) + sizeof(TapeRef) + 1 + 4 + 4) + 64;
            if (!lv_bufs[d].reserve(bytes)) return false;
            unsigned char* p = lv_bufs[d].as<unsigned char>();
            QLevel& q = t.lv[d];
            q.n = n;
            q.xy = reinterpret_cast<uint2*>(p);
            q.tape = reinterpret_cast<TapeRef*>(q.xy + m);
            q.child = reinterpret_cast<uint32_t*>(q.tape + m);
            q.leaf = q.child + m;
            q.type = reinterpret_cast<uint8_t*>(q.leaf + m);
            return true;
        };
        if (!alloc_level(0, 1)) return LFB_E_CUDA;
        const uint2 root_xy = make_uint2(0, 0);
        const TapeRef root_ref = root_tape_ref(bt);
        cudaMemcpyAsync(t.lv[0].xy, &root_xy, sizeof(root_xy), cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(t.lv[0].tape, &root_ref, sizeof(root_ref), cudaMemcpyHostToDevice, s);

        // quadtree build, level by level
        for (int d = 0; d < L; ++d) {
            const uint32_t n = t.lv[d].n;
            if (n == 0) {
                // every cell was decided above: the deeper levels are empty
                if (!alloc_level(d + 1, 0)) return LFB_E_CUDA;
                continue;
            }
            if (!b_out_tape.reserve(static_cast<size_t>(n) * sizeof(TapeRef)) ||
                !b_flags.reserve(static_cast<size_t>(n + 1) * 4) ||
                !b_scan.reserve(static_cast<size_t>(n + 1) * 4)) {
                return LFB_E_CUDA;
            }
            QIntervalArgs A{t, d, bt, arena, arena_top, arena_cap, b_out_tape.as<TapeRef>(),
                            b_rlo.as<float>(), b_rhi.as<float>(), b_rnan.as<uint8_t>(),
                            b_live.as<uint8_t>(), b_dec.as<uint8_t>(), dec_cap, T, status};
            k_q_interval<<<T / 256, 256, 0, s>>>(A);
            k_q_branch_flags<<<(n + 255) / 256, 256, 0, s>>>(t.lv[d].type, n, b_flags.as<uint32_t>());
            note_launches(2);
            // exclusive scan of the branch flags on the host (quadtree
            // levels are small; the counts decide the next level's size)
            std::vector<uint32_t> flags(n);
            if (!cuda_ok(cudaMemcpyAsync(flags.data(), b_flags.as<uint32_t>(), n * 4,
                                         cudaMemcpyDeviceToHost, s), "download") ||
                !cuda_ok(cudaStreamSynchronize(s), "contour intervals")) {
                return LFB_E_CUDA;
            }
            std::vector<uint32_t> scan(n + 1, 0);
            for (uint32_t k = 0; k < n; ++k) scan[k + 1] = scan[k] + flags[k];
            const uint32_t n_next = 4 * scan[n];
            cudaMemcpyAsync(b_scan.as<uint32_t>(), scan.data(), (n + 1) * 4, cudaMemcpyHostToDevice, s);
            if (!alloc_level(d + 1, n_next)) return LFB_E_CUDA;
            k_q_children<<<(n + 255) / 256, 256, 0, s>>>(t, d, b_scan.as<uint32_t>(),
                                                         b_out_tape.as<TapeRef>());
            note_launches(1);
            if (!cuda_ok(cudaGetLastError(), "contour intervals")) return LFB_E_CUDA;
        }

        // leaves at the finest depth
        if (t.lv[L].n) {
            QLeafArgs A{t, bt, arena, b_regs.as<float>(), nregs, b_featws.as<float>(),
                        b_fs.as<FeatureScratch>(), b_recs.as<QLeaf>(), rec_top, rec_cap, status};
            const uint32_t blocks = std::min<uint32_t>(leaf_warps / kLeafWarps,
                                                       (t.lv[L].n + kLeafWarps - 1) / kLeafWarps);
            k_q_leaf<<<std::max<uint32_t>(blocks, 1), 32 * kLeafWarps, 0, s>>>(A);
            note_launches(1);
        }
        // collapse, bottom-up
        for (int d = L - 1; d >= 0; --d) {
            QCollapseArgs C{t, d, bt, arena, b_recs.as<QLeaf>(), rec_top, rec_cap, max_err,
                            b_cregs.as<float>(), T, status};
            k_q_collapse<<<T / 256, 256, 0, s>>>(C);
            note_launches(1);
        }
        uint32_t st = 0;
        cudaMemcpyAsync(&st, status, 4, cudaMemcpyDeviceToHost, s);
        if (!cuda_ok(cudaStreamSynchronize(s), "contour leaves")) return LFB_E_CUDA;
        if (st & ST_ARENA_OVERFLOW) { arena_cap *= 4; continue; }
        if (st & ST_RECORD_OVERFLOW) { rec_cap *= 4; continue; }
        if (st & (ST_FEATURE_OVERFLOW | ST_REGS)) {
            return set_error(LFB_E_CAPACITY, "contours: feature list or decision capacity exceeded");
        }

        // dual walk
        QDualArgs D{t, b_recs.as<QLeaf>(), b_tasks_a.as<QTask>(), n_tasks, task_cap,
                    b_segs.as<uint2>(), n_segs, seg_cap, status};
        for (int d = 0; d < L; ++d) {
            if (t.lv[d].n) k_q_dual_init<<<(t.lv[d].n + 255) / 256, 256, 0, s>>>(D, d);
            note_launches(1);
        }
        QTask* qa = b_tasks_a.as<QTask>();
        QTask* qb = b_tasks_b.as<QTask>();
        uint32_t n_in = 0;
        cudaMemcpyAsync(&n_in, n_tasks, 4, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&st, status, 4, cudaMemcpyDeviceToHost, s);
        if (!cuda_ok(cudaStreamSynchronize(s), "contour walk")) return LFB_E_CUDA;
        bool overflow = (st & ST_QUEUE_OVERFLOW) != 0;
        while (n_in && !overflow) {
            cudaMemsetAsync(n_tasks, 0, 4, s);
            D.out = qb;
            k_q_dual_round<<<(n_in + 127) / 128, 128, 0, s>>>(D, qa, n_in);
            note_launches(1);
            cudaMemcpyAsync(&n_in, n_tasks, 4, cudaMemcpyDeviceToHost, s);
            cudaMemcpyAsync(&st, status, 4, cudaMemcpyDeviceToHost, s);
            if (!cuda_ok(cudaStreamSynchronize(s), "contour walk")) return LFB_E_CUDA;
            overflow = (st & ST_QUEUE_OVERFLOW) != 0;
            std::swap(qa, qb);
        }
        if (overflow) {
            task_cap *= 4;
            seg_cap *= 4;
            continue;
        }
        uint32_t ns = 0, nr = 0;
        cudaMemcpyAsync(&ns, n_segs, 4, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&nr, rec_top, 4, cudaMemcpyDeviceToHost, s);
        if (!cuda_ok(cudaStreamSynchronize(s), "contour walk")) return LFB_E_CUDA;
        std::vector<uint2> segs(ns);
        std::vector<QLeaf> recs(nr);
        if ((ns && !cuda_ok(cudaMemcpy(segs.data(), b_segs.as<uint2>(), ns * sizeof(uint2),
                                       cudaMemcpyDeviceToHost), "download")) ||
            (nr && !cuda_ok(cudaMemcpy(recs.data(), b_recs.as<QLeaf>(), nr * sizeof(QLeaf),
                                       cudaMemcpyDeviceToHost), "download"))) {
            return LFB_E_CUDA;
        }
        std::vector<std::pair<uint32_t, uint32_t>> sp(ns);
        for (uint32_t k = 0; k < ns; ++k) sp[k] = {segs[k].x, segs[k].y};
        std::vector<std::vector<uint32_t>> welded;
        weld_segments(sp, welded);
        for (const auto& c : welded) {
            out.counts.push_back(static_cast<uint32_t>(c.size()));
            for (uint32_t key : c) {
                const QLeaf& r = recs[key >> 1];
                out.pts.push_back(static_cast<float>(r.vert[key & 1][0]));
                out.pts.push_back(static_cast<float>(r.vert[key & 1][1]));
            }
        }
        return 0;
    }
    return set_error(LFB_E_CAPACITY, "contours: capacity retries exhausted");
}

}  // namespace lfb
