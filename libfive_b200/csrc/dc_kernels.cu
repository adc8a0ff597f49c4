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
#include <sys/mman.h>
#include <thread>
#include <cstdlib>
#include <cstring>

#include "dc_device.cuh"
#include "dc_features.cuh"
#include "eval_kernels.cuh"
#include "leaf_interp.cuh"

namespace lfb {

__constant__ DcTables c_tab;

////////////////////////////////////////////////////////////////////////////////
// 1. Interval classification and tape pruning

// One warp per cell.  The tape a cell inherits is held twice: as a register
// tape (for point evaluation) and as a list of its clauses sorted by
// dependency level whose operands name list slots (WideEntry), so the lanes
// of a warp evaluate the independent clauses of one level at once.  The
// per-slot state of a list of up to kWideSmemSlots entries lives in shared
// memory, that of longer lists in a per-warp global scratch slice.

constexpr uint32_t kWideSmemSlots = 512;
constexpr uint32_t kMaxTapeRegs = 400;
constexpr uint32_t kRenumberMax = kWideSmemSlots;   // tapes up to this length get compact registers
constexpr uint32_t kGroupModeCells = 8192;          // cells per level from which k_interval_group runs
constexpr uint32_t kBlockModeCells = 2048;          // cells per level up to which k_interval_block runs

struct WideSmem {
    float2 S[kWideSmemSlots + 3];      // slot intervals
    uint32_t newpos[kWideSmemSlots];   // entry -> position in the child list
    uint32_t mask[(kMaxTapeRegs + 31) / 32];   // register bitmask (renumbering)
    uint16_t regmap[kMaxTapeRegs];     // old -> new register (renumbering)
    uint8_t SN[kWideSmemSlots + 3];    // slot maybe-NaN flags
    uint8_t pst[kWideSmemSlots];       // entry state for the children
    uint8_t live[kWideSmemSlots];      // entry still needed by the children
};

struct WideArgs {
    Octree o;
    DevTape bt;
    uint32_t n;                    // clauses of the unpruned tape
    const WideEntry* in_lists;     // lists of this depth's groups
    ListRef root_list;             // the unpruned list (depth 0)
    WideEntry* out_lists;          // lists handed to the next depth
    unsigned long long* out_top;
    uint64_t out_cap;
    int write_lists;
    RegClause* arena;              // register tapes
    unsigned long long* arena_top;
    uint64_t arena_cap;
    // Per-warp global scratch: slot state of long lists, and the two-level
    // bitmap of clause states that orders the register tape (zero between
    // cells).
    float2* S;                     // [warps][n + 3]
    uint8_t* SN;                   // [warps][n + 3]
    uint8_t* pst;                  // [warps][n]
    uint8_t* live;                 // [warps][n]
    uint32_t* newpos;              // [warps][n]
    uint32_t* st2;                 // [warps][nw]   2-bit state per clause
    uint32_t* l1;                  // [warps][nw1]  non-zero words of st2
    uint32_t* wl;                  // [warps][nw]   word list
    uint32_t* status;
    uint32_t* next_cell;           // work counter (zero at launch)
};

__device__ __forceinline__ Iv wide_fetch(uint32_t kind, uint32_t idx,
                                         const float2* S, const uint8_t* SN,
                                         const float* __restrict__ cp)
{
    if (kind == OPND_REG) {
        const float2 v = S[idx];
        return {v.x, v.y, SN[idx] != 0};
    }
    const float v = __ldg(cp + idx);
    return iv_make(v, v);
}

/// Interval of list entry k, stored in slot 3 + k, and the entry's state for
/// the cell's children; returns whether a min/max got decided
/// (IntervalEvaluator::eval + push, eval_interval.cpp:116-167).
__device__ __forceinline__ bool wide_forward(const uint4& e, uint32_t k, const float* cp,
                                             float2* S, uint8_t* SN, uint8_t* pst)
{
    const uint8_t o = e.x & 0xff;
    const uint32_t kinds = (e.x >> 8) & 0xf;
    const uint32_t st = (e.x >> 12) & 3;
    Iv r;
    uint8_t ps = static_cast<uint8_t>(st);
    bool decided = false;
    if (st == WIDE_A) {
        r = wide_fetch(kinds & 3, e.y, S, SN, cp);
    } else if (st == WIDE_B) {
        r = wide_fetch((kinds >> 2) & 3, e.z, S, SN, cp);
    } else {
        const Iv a = wide_fetch(kinds & 3, e.y, S, SN, cp);
        const Iv b = dev_is_binary(o) ? wide_fetch((kinds >> 2) & 3, e.z, S, SN, cp) : a;
        r = iv_apply(o, a, b);
        if (o == op::MIN || o == op::MAX) {
            uint8_t keep = 0;   // 0 both, 1 a, 2 b
            if (a.lo > b.hi) keep = (o == op::MAX) ? 1 : 2;
            else if (b.lo > a.hi) keep = (o == op::MAX) ? 2 : 1;
            if (keep) {
                ps = keep == 1 ? WIDE_A : WIDE_B;
                decided = true;
            }
        }
    }
    S[3 + k] = make_float2(r.lo, r.hi);
    SN[3 + k] = r.nan;
    pst[k] = ps;
    return decided;
}

/// Marks the operands a live entry still needs (Tape::push's remapping,
/// tape.cpp:23-160, as liveness).
__device__ __forceinline__ void wide_mark(const uint4& e, uint8_t ps, uint8_t* live)
{
    const uint8_t o = e.x & 0xff;
    const uint32_t kinds = (e.x >> 8) & 0xf;
    if (ps != WIDE_B && (kinds & 3) == OPND_REG && e.y >= 3) live[e.y - 3] = 1;
    if (ps != WIDE_A && dev_is_binary(o) && ((kinds >> 2) & 3) == OPND_REG && e.z >= 3) {
        live[e.z - 3] = 1;
    }
}

/// Register clauses emitted for one 16-clause word of 2-bit states.
__device__ __forceinline__ uint32_t wide_word_emits(uint32_t word, uint32_t w,
                                                    const RegClause* root)
{
    uint32_t emit = 0;
    while (word) {
        const int j = (__ffs(word) - 1) >> 1;
        const uint32_t ps = (word >> (2 * j)) & 3;
        word &= ~(3u << (2 * j));
        if (ps == WIDE_BOTH) {
            ++emit;
            continue;
        }
        const uint2 raw = __ldg(reinterpret_cast<const uint2*>(root + w * 16 + j));
        const uint32_t kinds = (raw.x >> 8) & 0xff;
        const uint32_t k = ps == WIDE_A ? (kinds & 3) : ((kinds >> 2) & 3);
        const uint32_t src = ps == WIDE_A ? (raw.y & 0xffff) : (raw.y >> 16);
        emit += !(k == OPND_REG && src == (raw.x >> 16));
    }
    return emit;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane)
{
    for (int sh = 1; sh < 32; sh <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, v, sh);
        if (lane >= sh) v += t;
    }
    return v;
}

/// Linear-scan register allocation of a pruned tape, in place (one thread):
/// a backward pass marks each operand's last use, a forward pass gives every
/// result the lowest free register (X, Y and Z keep registers 0-2 while they
/// are still to be read).  On straight-line code this uses as many registers
/// as values are live at once, which is at most the unpruned tape's count;
/// the leaf kernel then fits the register file of most leaf tapes in shared
/// memory.  Values are unchanged: only storage moves.
static __device__ __noinline__ TapeRef renumber_tape(uint2* raw_t, TapeRef tr,
                                                     uint8_t* lastuse,
                                                     uint16_t* regmap,
                                                     uint32_t* mask,
                                                     uint32_t* status)
{
    const uint32_t nm = (tr.nregs + 31) / 32;
    const uint32_t rk = tr.root >> 16, rr = tr.root & 0xffff;
    for (uint32_t w = 0; w < nm; ++w) mask[w] = 0;   // live-after bits
    if (rk == OPND_REG) mask[rr >> 5] |= 1u << (rr & 31);
    for (int64_t c = static_cast<int64_t>(tr.len) - 1; c >= 0; --c) {
        const uint2 raw = raw_t[c];
        const uint32_t o = raw.x >> 16, kinds = (raw.x >> 8) & 0xff;
        const uint32_t a = raw.y & 0xffff, b = raw.y >> 16;
        mask[o >> 5] &= ~(1u << (o & 31));
        uint8_t f = 0;
        if ((kinds & 3) == OPND_REG) {
            if (!(mask[a >> 5] & (1u << (a & 31)))) f |= 1;
            mask[a >> 5] |= 1u << (a & 31);
        }
        if (dev_is_binary(raw.x & 0xff) && ((kinds >> 2) & 3) == OPND_REG) {
            if (!(mask[b >> 5] & (1u << (b & 31)))) f |= 2;
            mask[b >> 5] |= 1u << (b & 31);
        }
        lastuse[c] = f;
    }
    // X, Y, Z start in registers 0-2; those not read by the tape are free.
    const uint32_t xyz_live = mask[0] & 7u;
    constexpr uint32_t kWords = (kMaxTapeRegs + 31) / 32;
    for (uint32_t w = 0; w < kWords; ++w) mask[w] = ~0u;   // free bits
    if (kMaxTapeRegs % 32) mask[kWords - 1] = (1u << (kMaxTapeRegs % 32)) - 1;
    mask[0] &= ~xyz_live;
    for (uint32_t r = 0; r < 3; ++r) regmap[r] = static_cast<uint16_t>(r);
    uint32_t hi = 3;
    for (uint32_t c = 0; c < tr.len; ++c) {
        uint2 raw = raw_t[c];
        const uint32_t o = raw.x >> 16, kinds = (raw.x >> 8) & 0xff;
        const bool binary = dev_is_binary(raw.x & 0xff);
        uint32_t a = raw.y & 0xffff, b = raw.y >> 16;
        const uint8_t f = lastuse[c];
        if ((kinds & 3) == OPND_REG) a = regmap[a];
        if (binary && ((kinds >> 2) & 3) == OPND_REG) b = regmap[b];
        if (f & 1) mask[a >> 5] |= 1u << (a & 31);
        if (f & 2) mask[b >> 5] |= 1u << (b & 31);
        uint32_t r = 0xffffffffu;
        for (uint32_t w = 0; w < kWords; ++w) {
            if (mask[w]) {
                r = w * 32 + __ffs(mask[w]) - 1;
                break;
            }
        }
        if (r >= kMaxTapeRegs) {   // more live values than registers: cannot happen
            atomicOr(status, ST_REGS);
            return tr;
        }
        mask[r >> 5] &= ~(1u << (r & 31));
        regmap[o] = static_cast<uint16_t>(r);
        hi = max(hi, r + 1);
        raw.x = (raw.x & 0xffffu) | (r << 16);
        raw.y = a | (b << 16);
        raw_t[c] = raw;
    }
    const uint32_t root = rk == OPND_REG ? regmap[rr] : rr;
    return {tr.off, tr.len, hi, root | (rk << 16)};
}

__global__ void __launch_bounds__(256)
k_interval_wide(WideArgs A, int d)
{
    extern __shared__ __align__(16) unsigned char wsm[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + warp;
    WideSmem* SM = reinterpret_cast<WideSmem*>(wsm) + warp;
    const Octree& o = A.o;
    const LevelView& lv = o.lv[d];
    const DevTape& bt = A.bt;
    const uint32_t n = A.n;
    const uint32_t nw = (n + 15) / 16;
    const uint32_t nw1 = (nw + 31) / 32;
    float2* gS = A.S + static_cast<size_t>(gw) * (n + 3);
    uint8_t* gSN = A.SN + static_cast<size_t>(gw) * (n + 3);
    uint8_t* gP = A.pst + static_cast<size_t>(gw) * n;
    uint8_t* gL = A.live + static_cast<size_t>(gw) * n;
    uint32_t* gN = A.newpos + static_cast<size_t>(gw) * n;
    uint32_t* st2 = A.st2 + static_cast<size_t>(gw) * nw;
    uint32_t* l1 = A.l1 + static_cast<size_t>(gw) * nw1;
    uint32_t* wl = A.wl + static_cast<size_t>(gw) * nw;
    const unsigned full = 0xffffffffu;
    const uint32_t lt_mask = (1u << lane) - 1;

    while (true) {
        uint32_t i = 0;
        if (lane == 0) i = atomicAdd(A.next_cell, 1u);
        i = __shfl_sync(full, i, 0);
        if (i >= lv.n_cells) break;
        ListRef P;
        TapeRef T;
        if (d == 0) {
            P = A.root_list;
            T = root_tape_ref(bt);
        } else {
            P = lv.group_list[i >> 3];
            T = lv.group_tape[i >> 3];
        }
        const uint4* PL = reinterpret_cast<const uint4*>(A.in_lists + P.off);
        const bool small = P.len <= kWideSmemSlots;
        float2* S = small ? SM->S : gS;
        uint8_t* SN = small ? SM->SN : gSN;
        uint8_t* pst = small ? SM->pst : gP;
        uint8_t* live = small ? SM->live : gL;
        uint32_t* newpos = small ? SM->newpos : gN;
        if (lane < 3) {
            double blo[3], bhi[3];
            cell_bounds(o, d, lv.coords[i], blo, bhi);
            const Iv v = iv_make(static_cast<float>(blo[lane]), static_cast<float>(bhi[lane]));
            S[lane] = make_float2(v.lo, v.hi);
            SN[lane] = v.nan;
        }
        for (uint32_t k = lane; k < P.len; k += 32) live[k] = 0;
        __syncwarp();

        // Forward pass, level by level (entries are sorted by level, so a
        // chunk of 32 spans few levels; the warp steps through them).
        const uint32_t nchunks = (P.len + 31) / 32;
        bool changed = false;
        for (uint32_t ch = 0; ch < nchunks; ++ch) {
            const uint32_t k = ch * 32 + lane;
            const bool valid = k < P.len;
            const uint4 e = valid ? PL[k] : make_uint4(0, 0, 0, 0);
            const uint32_t lev = valid ? (e.x >> kWideLevelShift) : 0xffffffffu;
            const int last = static_cast<int>(min(31u, P.len - 1 - ch * 32));
            uint32_t l = __shfl_sync(full, lev, 0);
            const uint32_t lmax = __shfl_sync(full, lev, last);
            while (true) {
                if (lev == l) changed |= wide_forward(e, k, bt.cpool, S, SN, pst);
                __syncwarp();
                if (l == lmax) break;
                const uint32_t m = __ballot_sync(full, valid && lev > l);
                l = __shfl_sync(full, lev, __ffs(m) - 1);
            }
        }
        changed = __any_sync(full, changed);
        const Iv root = wide_fetch(bt.root_kind, P.root, S, SN, bt.cpool);
        const uint8_t state = iv_state(root);
        if (lane == 0) {
            lv.type[i] = state == ST_EMPTY ? CELL_EMPTY
                       : state == ST_FILLED ? CELL_FILLED : CELL_BRANCH;
        }
        if (state != ST_AMBIGUOUS) continue;

        if (root.nan || !changed) {
            // NaN-unsafe or nothing decided: the children keep this tape
            // (dc_tree.inl:107-111).  Its list moves to the next arena.
            uint32_t off = 0;
            if (A.write_lists) {
                unsigned long long o64 = 0;
                if (lane == 0) o64 = atomicAdd(A.out_top, static_cast<unsigned long long>(P.len));
                o64 = __shfl_sync(full, o64, 0);
                if (o64 + P.len <= A.out_cap) {
                    off = static_cast<uint32_t>(o64);
                    uint4* out = reinterpret_cast<uint4*>(A.out_lists + off);
                    for (uint32_t k = lane; k < P.len; k += 32) out[k] = PL[k];
                } else if (lane == 0) {
                    atomicOr(A.status, ST_LIST_OVERFLOW);
                }
            }
            if (lane == 0) {
                lv.cell_list[i] = {off, P.len, P.root, 0u};
                lv.cell_tape[i] = T;
            }
            continue;
        }

        // Backward liveness pass, levels in decreasing order.
        if (lane == 0 && bt.root_kind == OPND_REG && P.root >= 3) live[P.root - 3] = 1;
        __syncwarp();
        for (int ch = static_cast<int>(nchunks) - 1; ch >= 0; --ch) {
            const uint32_t k = ch * 32 + lane;
            const bool valid = k < P.len;
            const uint4 e = valid ? PL[k] : make_uint4(0, 0, 0, 0);
            const uint32_t lev = valid ? (e.x >> kWideLevelShift) : 0u;
            const int last = static_cast<int>(min(31u, P.len - 1 - ch * 32));
            const uint32_t lmin = __shfl_sync(full, lev, 0);
            uint32_t l = __shfl_sync(full, lev, last);
            while (true) {
                if (valid && lev == l && live[k]) wide_mark(e, pst[k], live);
                __syncwarp();
                if (l == lmin) break;
                const uint32_t m = __ballot_sync(full, valid && lev < l);
                l = __shfl_sync(full, lev, 31 - __clz(m));
            }
        }

        // Child positions of the live entries, and their 2-bit states by
        // clause index (for the register tape, which is in clause order).
        uint32_t cnt = 0;
        for (uint32_t ch = 0; ch < nchunks; ++ch) {
            const uint32_t k = ch * 32 + lane;
            const bool lv_ = k < P.len && live[k];
            const uint32_t m = __ballot_sync(full, lv_);
            if (lv_) {
                newpos[k] = cnt + __popc(m & lt_mask);
                const uint32_t c = PL[k].w;
                atomicOr(st2 + (c >> 4), static_cast<uint32_t>(pst[k]) << (2 * (c & 15)));
                atomicOr(l1 + (c >> 9), 1u << ((c >> 4) & 31));
            }
            cnt += __popc(m);
        }
        __syncwarp();
        const uint32_t new_root = (bt.root_kind == OPND_REG && P.root >= 3)
                                      ? newpos[P.root - 3] + 3 : P.root;
        uint32_t loff = 0;
        if (A.write_lists) {
            unsigned long long o64 = 0;
            if (lane == 0) o64 = atomicAdd(A.out_top, static_cast<unsigned long long>(cnt));
            o64 = __shfl_sync(full, o64, 0);
            const bool ok = o64 + cnt <= A.out_cap;
            if (!ok && lane == 0) atomicOr(A.status, ST_LIST_OVERFLOW);
            if (ok) {
                loff = static_cast<uint32_t>(o64);
                uint4* out = reinterpret_cast<uint4*>(A.out_lists + loff);
                for (uint32_t k = lane; k < P.len; k += 32) {
                    if (!live[k]) continue;
                    uint4 e = PL[k];
                    const uint32_t ps = pst[k];
                    const uint32_t kinds = (e.x >> 8) & 0xf;
                    const bool binary = dev_is_binary(e.x & 0xff);
                    if (ps == WIDE_B) e.y = 0;
                    else if ((kinds & 3) == OPND_REG && e.y >= 3) e.y = newpos[e.y - 3] + 3;
                    if (ps == WIDE_A) e.z = 0;
                    else if (binary && ((kinds >> 2) & 3) == OPND_REG && e.z >= 3) {
                        e.z = newpos[e.z - 3] + 3;
                    }
                    e.x = (e.x & ~(3u << 12)) | (ps << 12);
                    out[newpos[k]] = e;
                }
            }
        }

        // Register tape for this cell: the live clauses in clause order, with
        // decided min/max clauses as copies (dropped when the copy is onto
        // the same register).  First the non-zero state words, in order.
        uint32_t nwl = 0;
        for (uint32_t j0 = 0; j0 < nw1; j0 += 32) {
            const uint32_t j = j0 + lane;
            uint32_t bits = 0;
            if (j < nw1) {
                bits = l1[j];
                l1[j] = 0;
            }
            const uint32_t c_ = __popc(bits);
            const uint32_t incl = warp_incl_scan(c_, lane);
            uint32_t at = nwl + incl - c_;
            while (bits) {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1;
                wl[at++] = j * 32 + b;
            }
            nwl += __shfl_sync(full, incl, 31);
        }
        __syncwarp();
        uint32_t emit = 0;
        for (uint32_t k0 = 0; k0 < nwl; k0 += 32) {
            const uint32_t k = k0 + lane;
            uint32_t e_ = 0;
            if (k < nwl) {
                const uint32_t w = wl[k];
                e_ = wide_word_emits(st2[w], w, bt.clauses);
            }
            emit += __reduce_add_sync(full, e_);
        }
        unsigned long long a64 = 0;
        if (lane == 0) a64 = atomicAdd(A.arena_top, static_cast<unsigned long long>(emit));
        a64 = __shfl_sync(full, a64, 0);
        const bool aok = a64 + emit <= A.arena_cap;
        if (!aok && lane == 0) atomicOr(A.status, ST_ARENA_OVERFLOW);
        uint32_t pos = static_cast<uint32_t>(a64);
        for (uint32_t k0 = 0; k0 < nwl; k0 += 32) {
            const uint32_t k = k0 + lane;
            uint32_t word = 0, w = 0, e_ = 0;
            if (k < nwl) {
                w = wl[k];
                word = st2[w];
                e_ = wide_word_emits(word, w, bt.clauses);
                st2[w] = 0;
            }
            const uint32_t incl = warp_incl_scan(e_, lane);
            uint32_t at = pos + incl - e_;
            if (aok) {
                while (word) {
                    const int j = (__ffs(word) - 1) >> 1;
                    const uint32_t ps = (word >> (2 * j)) & 3;
                    word &= ~(3u << (2 * j));
                    const uint2 raw = __ldg(reinterpret_cast<const uint2*>(bt.clauses + w * 16 + j));
                    if (ps == WIDE_BOTH) {
                        *reinterpret_cast<uint2*>(A.arena + at++) = raw;
                        continue;
                    }
                    const uint32_t kinds = (raw.x >> 8) & 0xff;
                    const uint32_t kk = ps == WIDE_A ? (kinds & 3) : ((kinds >> 2) & 3);
                    const uint32_t src = ps == WIDE_A ? (raw.y & 0xffff) : (raw.y >> 16);
                    const uint32_t ro = raw.x >> 16;
                    if (kk == OPND_REG && src == ro) continue;
                    RegClause cc;
                    cc.op = OP_COPY;
                    cc.kinds = static_cast<uint8_t>(kk);
                    cc.out = static_cast<uint16_t>(ro);
                    cc.a = static_cast<uint16_t>(src);
                    cc.b = 0;
                    A.arena[at++] = cc;
                }
            }
            pos += __shfl_sync(full, incl, 31);
        }
        __syncwarp();
        TapeRef out_t = T;
        if (aok) {
            out_t = {static_cast<uint32_t>(a64), emit, bt.n_regs,
                     static_cast<uint32_t>(bt.root) | (static_cast<uint32_t>(bt.root_kind) << 16)};
            if (emit <= kRenumberMax) {
                // Short tapes get compact registers: staged through the
                // warp's shared slot area (free again at this point).
                uint2* buf = reinterpret_cast<uint2*>(SM->S);
                uint2* dst = reinterpret_cast<uint2*>(A.arena + a64);
                for (uint32_t k = lane; k < emit; k += 32) buf[k] = dst[k];
                __syncwarp();
                if (lane == 0) {
                    out_t = renumber_tape(buf, out_t, SM->live, SM->regmap, SM->mask, A.status);
                }
                __syncwarp();
                for (uint32_t k = lane; k < emit; k += 32) dst[k] = buf[k];
                out_t.nregs = __shfl_sync(full, out_t.nregs, 0);
                out_t.root = __shfl_sync(full, out_t.root, 0);
            }
        }
        if (lane == 0) {
            lv.cell_list[i] = {loff, cnt, new_root, 0u};
            lv.cell_tape[i] = out_t;
        }
        __syncwarp();
    }
}

// Top levels: one block per cell.  The first levels have few cells with
// long lists (the unpruned tape at depth 0), so all warps of a block work on
// one cell: a wave of kBlockThreads consecutive entries at a time, stepping
// through the levels the wave spans with a block barrier per level.  Same
// results as k_interval_wide (lists, register tapes); tapes are not
// renumbered (they are long at these depths).

constexpr int kBlockThreads = 512;
constexpr int kBlockWarps = kBlockThreads / 32;

/// Exclusive prefix over the block of one count per thread, and the total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* warp_tot,
                                                    uint32_t& total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t incl = warp_incl_scan(v, lane);
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    uint32_t before = 0;
    total = 0;
    for (int w = 0; w < kBlockWarps; ++w) {
        const uint32_t t = warp_tot[w];
        if (w < warp) before += t;
        total += t;
    }
    __syncthreads();
    return before + incl - v;
}

__global__ void __launch_bounds__(kBlockThreads)
k_interval_block(WideArgs A, int d)
{
    __shared__ uint32_t warp_tot[kBlockWarps];
    __shared__ unsigned long long bcast;
    __shared__ uint32_t cell;
    const int tid = threadIdx.x;
    const Octree& o = A.o;
    const LevelView& lv = o.lv[d];
    const DevTape& bt = A.bt;
    const uint32_t n = A.n;
    const uint32_t nw = (n + 15) / 16;
    const size_t slot = blockIdx.x;
    float2* S = A.S + slot * (n + 3);
    uint8_t* SN = A.SN + slot * (n + 3);
    uint8_t* pst = A.pst + slot * n;
    uint8_t* live = A.live + slot * n;
    uint32_t* newpos = A.newpos + slot * n;
    uint32_t* st2 = A.st2 + slot * nw;

    while (true) {
        if (tid == 0) cell = atomicAdd(A.next_cell, 1u);
        __syncthreads();
        const uint32_t i = cell;
        __syncthreads();
        if (i >= lv.n_cells) break;
        ListRef P;
        TapeRef T;
        if (d == 0) {
            P = A.root_list;
            T = root_tape_ref(bt);
        } else {
            P = lv.group_list[i >> 3];
            T = lv.group_tape[i >> 3];
        }
        const uint4* PL = reinterpret_cast<const uint4*>(A.in_lists + P.off);
        if (tid < 3) {
            double blo[3], bhi[3];
            cell_bounds(o, d, lv.coords[i], blo, bhi);
            const Iv v = iv_make(static_cast<float>(blo[tid]), static_cast<float>(bhi[tid]));
            S[tid] = make_float2(v.lo, v.hi);
            SN[tid] = v.nan;
        }
        for (uint32_t k = tid; k < P.len; k += kBlockThreads) live[k] = 0;
        __syncthreads();

        // Forward pass: waves of consecutive entries, levels in order.
        const uint32_t nwaves = (P.len + kBlockThreads - 1) / kBlockThreads;
        bool changed = false;
        for (uint32_t w = 0; w < nwaves; ++w) {
            const uint32_t b0 = w * kBlockThreads;
            const uint32_t k = b0 + tid;
            const bool valid = k < P.len;
            const uint4 e = valid ? PL[k] : make_uint4(0, 0, 0, 0);
            const uint32_t lev = valid ? (e.x >> kWideLevelShift) : 0xffffffffu;
            const uint32_t lf = PL[b0].x >> kWideLevelShift;
            const uint32_t ll = PL[min(b0 + kBlockThreads, P.len) - 1].x >> kWideLevelShift;
            for (uint32_t l = lf; l <= ll; ++l) {
                if (lev == l) changed |= wide_forward(e, k, bt.cpool, S, SN, pst);
                __syncthreads();
            }
        }
        changed = __syncthreads_or(changed) != 0;
        const Iv root = wide_fetch(bt.root_kind, P.root, S, SN, bt.cpool);
        const uint8_t state = iv_state(root);
        if (tid == 0) {
            lv.type[i] = state == ST_EMPTY ? CELL_EMPTY
                       : state == ST_FILLED ? CELL_FILLED : CELL_BRANCH;
        }
        if (state != ST_AMBIGUOUS) continue;

        if (root.nan || !changed) {
            // The children keep this tape; its list moves to the next arena.
            uint32_t off = 0;
            if (A.write_lists) {
                if (tid == 0) bcast = atomicAdd(A.out_top, static_cast<unsigned long long>(P.len));
                __syncthreads();
                const unsigned long long o64 = bcast;
                __syncthreads();
                if (o64 + P.len <= A.out_cap) {
                    off = static_cast<uint32_t>(o64);
                    uint4* out = reinterpret_cast<uint4*>(A.out_lists + off);
                    for (uint32_t k = tid; k < P.len; k += kBlockThreads) out[k] = PL[k];
                } else if (tid == 0) {
                    atomicOr(A.status, ST_LIST_OVERFLOW);
                }
            }
            if (tid == 0) {
                lv.cell_list[i] = {off, P.len, P.root, 0u};
                lv.cell_tape[i] = T;
            }
            continue;
        }

        // Backward liveness pass: waves in reverse, levels decreasing.
        if (tid == 0 && bt.root_kind == OPND_REG && P.root >= 3) live[P.root - 3] = 1;
        __syncthreads();
        for (int w = static_cast<int>(nwaves) - 1; w >= 0; --w) {
            const uint32_t b0 = w * kBlockThreads;
            const uint32_t k = b0 + tid;
            const bool valid = k < P.len;
            const uint4 e = valid ? PL[k] : make_uint4(0, 0, 0, 0);
            const uint32_t lev = valid ? (e.x >> kWideLevelShift) : 0xffffffffu;
            const uint32_t lf = PL[b0].x >> kWideLevelShift;
            const uint32_t ll = PL[min(b0 + kBlockThreads, P.len) - 1].x >> kWideLevelShift;
            for (uint32_t l = ll + 1; l-- > lf;) {
                if (lev == l && live[k]) wide_mark(e, pst[k], live);
                __syncthreads();
            }
        }

        // Child positions of the live entries and their 2-bit states.
        uint32_t cnt = 0;
        for (uint32_t w = 0; w < nwaves; ++w) {
            const uint32_t k = w * kBlockThreads + tid;
            const bool lv_ = k < P.len && live[k];
            uint32_t tot = 0;
            const uint32_t before = block_excl_scan(lv_ ? 1u : 0u, warp_tot, tot);
            if (lv_) {
                newpos[k] = cnt + before;
                const uint32_t c = PL[k].w;
                atomicOr(st2 + (c >> 4), static_cast<uint32_t>(pst[k]) << (2 * (c & 15)));
            }
            cnt += tot;
        }
        __syncthreads();
        const uint32_t new_root = (bt.root_kind == OPND_REG && P.root >= 3)
                                      ? newpos[P.root - 3] + 3 : P.root;
        uint32_t loff = 0;
        if (A.write_lists) {
            if (tid == 0) bcast = atomicAdd(A.out_top, static_cast<unsigned long long>(cnt));
            __syncthreads();
            const unsigned long long o64 = bcast;
            __syncthreads();
            const bool ok = o64 + cnt <= A.out_cap;
            if (!ok && tid == 0) atomicOr(A.status, ST_LIST_OVERFLOW);
            if (ok) {
                loff = static_cast<uint32_t>(o64);
                uint4* out = reinterpret_cast<uint4*>(A.out_lists + loff);
                for (uint32_t k = tid; k < P.len; k += kBlockThreads) {
                    if (!live[k]) continue;
                    uint4 e = PL[k];
                    const uint32_t ps = pst[k];
                    const uint32_t kinds = (e.x >> 8) & 0xf;
                    const bool binary = dev_is_binary(e.x & 0xff);
                    if (ps == WIDE_B) e.y = 0;
                    else if ((kinds & 3) == OPND_REG && e.y >= 3) e.y = newpos[e.y - 3] + 3;
                    if (ps == WIDE_A) e.z = 0;
                    else if (binary && ((kinds >> 2) & 3) == OPND_REG && e.z >= 3) {
                        e.z = newpos[e.z - 3] + 3;
                    }
                    e.x = (e.x & ~(3u << 12)) | (ps << 12);
                    out[newpos[k]] = e;
                }
            }
        }

        // Register tape: live clauses in clause order (dense over the state
        // words, which hold the whole tape at these depths).
        uint32_t emit = 0;
        for (uint32_t w = tid; w < nw; w += kBlockThreads) emit += wide_word_emits(st2[w], w, bt.clauses);
        uint32_t etot = 0;
        block_excl_scan(emit, warp_tot, etot);
        if (tid == 0) bcast = atomicAdd(A.arena_top, static_cast<unsigned long long>(etot));
        __syncthreads();
        const unsigned long long a64 = bcast;
        __syncthreads();
        const bool aok = a64 + etot <= A.arena_cap;
        if (!aok && tid == 0) atomicOr(A.status, ST_ARENA_OVERFLOW);
        uint32_t pos = static_cast<uint32_t>(a64);
        const uint32_t nwwaves = (nw + kBlockThreads - 1) / kBlockThreads;
        for (uint32_t ww = 0; ww < nwwaves; ++ww) {
            const uint32_t w = ww * kBlockThreads + tid;
            uint32_t word = 0, e_ = 0;
            if (w < nw) {
                word = st2[w];
                e_ = wide_word_emits(word, w, bt.clauses);
                st2[w] = 0;
            }
            uint32_t tot = 0;
            uint32_t at = pos + block_excl_scan(e_, warp_tot, tot);
            if (aok) {
                while (word) {
                    const int j = (__ffs(word) - 1) >> 1;
                    const uint32_t ps = (word >> (2 * j)) & 3;
                    word &= ~(3u << (2 * j));
                    const uint2 raw = __ldg(reinterpret_cast<const uint2*>(bt.clauses + w * 16 + j));
                    if (ps == WIDE_BOTH) {
                        *reinterpret_cast<uint2*>(A.arena + at++) = raw;
                        continue;
                    }
                    const uint32_t kinds = (raw.x >> 8) & 0xff;
                    const uint32_t kk = ps == WIDE_A ? (kinds & 3) : ((kinds >> 2) & 3);
                    const uint32_t src = ps == WIDE_A ? (raw.y & 0xffff) : (raw.y >> 16);
                    const uint32_t ro = raw.x >> 16;
                    if (kk == OPND_REG && src == ro) continue;
                    RegClause cc;
                    cc.op = OP_COPY;
                    cc.kinds = static_cast<uint8_t>(kk);
                    cc.out = static_cast<uint16_t>(ro);
                    cc.a = static_cast<uint16_t>(src);
                    cc.b = 0;
                    A.arena[at++] = cc;
                }
            }
            pos += tot;
        }
        if (tid == 0) {
            lv.cell_list[i] = {loff, cnt, new_root, 0u};
            lv.cell_tape[i] = aok ? TapeRef{static_cast<uint32_t>(a64), etot, bt.n_regs,
                                             static_cast<uint32_t>(bt.root) |
                                                 (static_cast<uint32_t>(bt.root_kind) << 16)}
                                  : T;
        }
        __syncthreads();
    }
}

// Deep levels: one warp per sibling group, one lane per cell.  The eight
// cells share their parent's register tape, so lanes 0-7 walk the same
// clause stream (no divergence) with the interval register file in shared
// memory, as IntervalEvaluator does, and prune with a backward liveness pass
// over registers (Tape::push, tape.cpp:23-160).  Used once cells are many
// and tapes short, where the per-cell overheads of the level-ordered form
// dominate; it writes register tapes only.

struct GroupArgs {
    Octree o;
    DevTape bt;
    RegClause* arena;
    unsigned long long* arena_top;
    uint64_t arena_cap;
    uint8_t* dec;                  // [warps][8][dec_cap] min/max decisions
    uint32_t dec_cap;
    uint8_t* lastuse;              // [warps][8][kRenumberMax] renumbering flags
    uint32_t nregs_max;            // register file size (this depth's largest group tape)
    uint32_t* status;
    uint32_t* next_group;          // work counter (zero at launch)
};

__host__ __device__ inline size_t group_smem_per_warp(uint32_t nregs_max)
{
    // L, H (float), regmap (u16) per register and lane; masks; N (u8).
    const size_t b = static_cast<size_t>(nregs_max) * 8 * (4 + 4 + 2) + 8 * 13 * 4 +
                     static_cast<size_t>(nregs_max) * 8;
    return (b + 15) / 16 * 16;
}

__global__ void __launch_bounds__(128)
k_interval_group(GroupArgs A, int d)
{
    extern __shared__ __align__(16) unsigned char gsm[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const uint32_t nr = A.nregs_max;
    unsigned char* base = gsm + group_smem_per_warp(nr) * warp;
    float* Lo = reinterpret_cast<float*>(base);
    float* Hi = Lo + nr * 8;
    uint16_t* RM = reinterpret_cast<uint16_t*>(Hi + nr * 8) + lane * nr;
    uint32_t* MK = reinterpret_cast<uint32_t*>(reinterpret_cast<uint16_t*>(Hi + nr * 8) + nr * 8) +
                   lane * 13;
    uint8_t* Nn = reinterpret_cast<uint8_t*>(reinterpret_cast<uint32_t*>(
                      reinterpret_cast<uint16_t*>(Hi + nr * 8) + nr * 8) + 8 * 13);
    const uint32_t gw = blockIdx.x * wpb + warp;
    uint8_t* dec = A.dec + (static_cast<size_t>(gw) * 8 + (lane & 7)) * A.dec_cap;
    uint8_t* lastuse = A.lastuse + (static_cast<size_t>(gw) * 8 + (lane & 7)) * kRenumberMax;
    const Octree& o = A.o;
    const LevelView& lv = o.lv[d];
    const DevTape& bt = A.bt;
    auto fetch = [&](uint32_t kind, uint32_t idx) -> Iv {
        if (kind == OPND_REG) return {Lo[idx * 8 + lane], Hi[idx * 8 + lane], Nn[idx * 8 + lane] != 0};
        const float v = __ldg(bt.cpool + idx);
        return iv_make(v, v);
    };

    while (true) {
        uint32_t g = 0;
        if (lane == 0) g = atomicAdd(A.next_group, 1u);
        g = __shfl_sync(0xffffffffu, g, 0);
        if (g >= lv.n_groups) break;
        if (lane >= 8) continue;
        const uint32_t i = 8 * g + lane;
        const TapeRef T = lv.group_tape[g];
        const RegClause* cl = A.arena + T.off;
        const uint32_t rk = T.root >> 16, rr = T.root & 0xffff;

        double blo[3], bhi[3];
        cell_bounds(o, d, lv.coords[i], blo, bhi);
        for (int a = 0; a < 3; ++a) {
            const Iv v = iv_make(static_cast<float>(blo[a]), static_cast<float>(bhi[a]));
            Lo[a * 8 + lane] = v.lo;
            Hi[a * 8 + lane] = v.hi;
            Nn[a * 8 + lane] = v.nan;
        }
        // Forward pass, recording the push decision of every min/max
        // (IntervalEvaluator::push, eval_interval.cpp:116-167).
        bool changed = false;
        uint32_t ch = 0;
        for (uint32_t c = 0; c < T.len; ++c) {
            const uint2 raw = __ldg(reinterpret_cast<const uint2*>(cl + c));
            const uint8_t o_ = raw.x & 0xff;
            const uint32_t kinds = (raw.x >> 8) & 0xff;
            const uint32_t ro = raw.x >> 16;
            const Iv a = fetch(kinds & 3, raw.y & 0xffff);
            const Iv b = fetch((kinds >> 2) & 3, raw.y >> 16);
            const Iv r = iv_apply(o_, a, b);
            if (o_ == op::MIN || o_ == op::MAX) {
                uint8_t keep = 0;   // 0 both, 1 a, 2 b
                if (a.lo > b.hi) keep = (o_ == op::MAX) ? 1 : 2;
                else if (b.lo > a.hi) keep = (o_ == op::MAX) ? 2 : 1;
                changed |= keep != 0;
                if (ch < A.dec_cap) dec[ch] = keep;
                ++ch;
            }
            Lo[ro * 8 + lane] = r.lo;
            Hi[ro * 8 + lane] = r.hi;
            Nn[ro * 8 + lane] = r.nan;
        }
        const Iv root = fetch(rk, rr);
        const uint8_t state = iv_state(root);
        lv.type[i] = state == ST_EMPTY ? CELL_EMPTY
                   : state == ST_FILLED ? CELL_FILLED : CELL_BRANCH;
        if (state != ST_AMBIGUOUS) continue;
        if (ch > A.dec_cap) {   // cannot happen: dec_cap is the unpruned tape's count
            atomicOr(A.status, ST_REGS);
            lv.cell_tape[i] = T;
            continue;
        }
        // NaN-unsafe results keep the unpruned tape (dc_tree.inl:107-111).
        if (root.nan || !changed) {
            lv.cell_tape[i] = T;
            continue;
        }
        // Backward liveness pass over registers: count, then allocate and
        // write the kept clauses from the back.
        uint32_t kept = 0;
        TapeRef out = T;
        for (int pass = 0; pass < 2; ++pass) {
            for (uint32_t r = 0; r < T.nregs; ++r) Nn[r * 8 + lane] = 0;
            if (rk == OPND_REG) Nn[rr * 8 + lane] = 1;
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
            for (int64_t c = static_cast<int64_t>(T.len) - 1; c >= 0; --c) {
                const uint2 raw = __ldg(reinterpret_cast<const uint2*>(cl + c));
                const uint8_t o_ = raw.x & 0xff;
                const uint32_t kinds = (raw.x >> 8) & 0xff;
                const uint32_t ro = raw.x >> 16;
                uint8_t keep = 0;
                if (o_ == op::MIN || o_ == op::MAX) keep = dec[--chi];
                if (!Nn[ro * 8 + lane]) continue;
                Nn[ro * 8 + lane] = 0;
                uint2 outc = raw;
                bool emit = true;
                if (keep) {
                    const uint32_t k = keep == 1 ? (kinds & 3) : ((kinds >> 2) & 3);
                    const uint32_t src = keep == 1 ? (raw.y & 0xffff) : (raw.y >> 16);
                    if (k == OPND_REG) {
                        Nn[src * 8 + lane] = 1;
                        emit = src != ro;
                    }
                    outc.x = OP_COPY | (k << 8) | (ro << 16);
                    outc.y = src;
                } else {
                    if ((kinds & 3) == OPND_REG) Nn[(raw.y & 0xffff) * 8 + lane] = 1;
                    if (dev_is_binary(o_) && ((kinds >> 2) & 3) == OPND_REG) {
                        Nn[(raw.y >> 16) * 8 + lane] = 1;
                    }
                }
                if (!emit) continue;
                if (pass == 0) {
                    ++kept;
                } else {
                    *reinterpret_cast<uint2*>(A.arena + off + (--pos)) = outc;
                }
            }
            if (pass == 1) {
                out = {static_cast<uint32_t>(off), kept, T.nregs, T.root};
                if (kept <= kRenumberMax) {
                    out = renumber_tape(reinterpret_cast<uint2*>(A.arena + off), out, lastuse,
                                        RM, MK, A.status);
                }
            }
        }
        lv.cell_tape[i] = out;
    }
}

////////////////////////////////////////////////////////////////////////////////
// 2. Leaves: one warp per group of eight sibling cells


struct EdgeSlot {
    double t0[3], t1[3];   // current search bracket: inside, outside
    float g0[4], g1[4];    // gradient + value at t0 / t1
    uint8_t amb[2];        // tied min/max at t0 / t1
};

/// Per-warp state kept in shared memory (small: occupancy is set by it).
struct LeafWarpShared {
    int8_t slot_of[54];    // lattice edge -> slot, -1 if not crossing
    uint8_t st[27];        // corner states (CELL_EMPTY / CELL_FILLED)
    uint8_t nslots;
    int32_t rec[8];
};

/// Per-warp state kept in global memory (L1-cached): edge brackets, the
/// gradients at their final ends and the feature evaluator's scratch, one
/// slice per resident warp.
struct LeafWarpScratch {
    FeatureScratch fs;
    EdgeSlot e[54];
};

/// A crossing lattice edge's QEF, handed from the leaf kernel to the rank
/// and vertex kernels.
struct EdgeRec {
    double t0[3], t1[3];   // final search bracket: inside end, outside end
    Qef q;
    uint8_t exists;
    uint8_t rank;
};

/// Where a leaf group's edge records start, and which lattice edge has
/// which (-1: none).
struct GroupEdges {
    uint32_t base;          // 0xffffffff: the records did not fit
    uint8_t n_edges;
    int8_t slot_of[54];
};

/// The interpreters' register file (one float4 per register and lane): in
/// the block's dynamic shared memory at byte offset `soff` (S = true: the
/// compiler then emits shared-memory loads and stores, and knows they cannot
/// alias anything else), or in global memory at `g` (tapes with too many
/// registers).
template <bool S>
__device__ __forceinline__ float4* regfile4(uint32_t soff, float* g)
{
    if (S) {
        extern __shared__ __align__(16) unsigned char rf_smem[];
        return reinterpret_cast<float4*>(rf_smem + soff);
    }
    return reinterpret_cast<float4*>(g);
}

/// The warp's decoded-clause buffer (kLeafOps LeafOps) at byte offset `off`
/// of the block's dynamic shared memory.
__device__ __forceinline__ LeafOp* leaf_ops(uint32_t off)
{
    extern __shared__ __align__(16) unsigned char rf_smem[];
    return reinterpret_cast<LeafOp*>(rf_smem + off);
}

/// dv_value on four points (a float4 per operand), the value rules of
/// dev_point.cuh; the rare opcodes out of line.
__device__ __forceinline__ float4 dv_value4f(uint8_t o, const float4& a, const float4& b)
{
#define LFB_EACH2(F) make_float4(F(a.x, b.x), F(a.y, b.y), F(a.z, b.z), F(a.w, b.w))
#define LFB_EACH1(F) make_float4(F(a.x), F(a.y), F(a.z), F(a.w))
    switch (o) {
        case op::ADD: return LFB_EACH2(f_add);
        case op::MUL: return LFB_EACH2(f_mul);
        case op::MIN: return LFB_EACH2(sc_min);
        case op::MAX: return LFB_EACH2(sc_max);
        case op::SUB: return LFB_EACH2(f_sub);
        case op::SQUARE: return LFB_EACH1(f_square);
        case op::SQRT: return LFB_EACH1(f_sqrt);
        case op::NEG: return LFB_EACH1(f_neg);
        case op::ABS: return LFB_EACH1(f_abs);
        case op::CONST_VAR:
        case OP_COPY: return a;
        default: return leaf_generic4(o, a, b);
    }
#undef LFB_EACH1
#undef LFB_EACH2
}

/// Values of the tape at four points per lane (point k of this lane in
/// component k), streaming the tape's clauses (one clause fetched ahead) with
/// the register file as one float4 per register and lane.  With ties
/// (a run-time flag, so that one copy of the loop serves corners and edge
/// search), bit k of *amb reports a min / max with equal arguments at point
/// k (ArrayEvaluator::getAmbiguous, eval_array.cpp:197-217).
template <bool S>
static __device__ __noinline__ float4 warp_value4(const float* __restrict__ cpool,
                                                  uint32_t root_kind, uint32_t root,
                                                  const RegClause* __restrict__ cl, uint32_t len,
                                                  uint32_t soff, float* Rg, int lane, float4 x,
                                                  float4 y, float4 z, bool ties, uint32_t* amb)
{
    float4* R = regfile4<S>(soff, Rg) + lane;
    R[0] = x;
    R[32] = y;
    R[64] = z;
    uint32_t t = 0;
    uint2 next = len ? __ldg(reinterpret_cast<const uint2*>(cl)) : make_uint2(0, 0);
#pragma unroll 1
    for (uint32_t c = 0; c < len; ++c) {
        const uint2 raw = next;
        if (c + 1 < len) next = __ldg(reinterpret_cast<const uint2*>(cl + c + 1));
        const uint8_t o = raw.x & 0xff;
        const uint32_t kinds = (raw.x >> 8) & 0xff;
        const uint32_t ra = raw.y & 0xffff, rb = raw.y >> 16, ro = raw.x >> 16;
        const float4 a = (kinds & 3) == OPND_REG ? R[ra * 32] : splat4(__ldg(cpool + ra));
        const float4 b = ((kinds >> 2) & 3) == OPND_REG ? R[rb * 32] : splat4(__ldg(cpool + rb));
        if (ties && (o == op::MIN || o == op::MAX)) t |= tie4(a, b);
        R[ro * 32] = dv_value4f(o, a, b);
    }
    *amb = t;
    if (root_kind == OPND_REG) return R[root * 32];
    return splat4(__ldg(cpool + root));
}

/// Value and gradient of the tape at one point per lane, plus, for most
/// points, FeatureEvaluator's feature list (eval_feature.cpp:171-372)
/// without building it.  Every register is either plain (one feature: its
/// gradient, no epsilons) or tainted (anything else).  A tied min/max of two
/// plain features is settled as the general feature path settles it
/// (Feature::push and operator<, feature.cpp:50-72, 247-284): a gradient
/// difference of zero length keeps the first argument; otherwise the two
/// candidates (each gradient with the normalised difference, or its
/// negation, as epsilon) are sorted and, when their gradients agree to
/// within 1e-10 (squared), collapse to the first, epsilons dropped.  Any
/// other tie taints the result; a min/max without a tie passes on the chosen
/// side, taint included; all other clauses are tainted when an operand is.
/// Values are always exact.  *plain says the root is untainted: its single
/// feature is then the returned gradient.  *ambig reports any tie
/// (ArrayEvaluator::getAmbiguous).  Tapes with more than 64 registers report
/// every tie as not plain.
template <bool S>
static __device__ __noinline__ D4 leaf_deriv(const float* __restrict__ cpool, uint32_t root_kind,
                                             uint32_t root, uint32_t n_regs,
                                             const RegClause* __restrict__ cl, uint32_t len,
                                             uint32_t soff, float* Rg, uint32_t ops_off, int lane,
                                             float x, float y, float z, bool* ambig, bool* plain,
                                             bool predecoded)
{
    float4* R = regfile4<S>(soff, Rg) + lane;
    LeafOp* ops = leaf_ops(ops_off);
    R[0] = make_float4(x, 1.0f, 0.0f, 0.0f);
    R[32] = make_float4(y, 0.0f, 1.0f, 0.0f);
    R[64] = make_float4(z, 0.0f, 0.0f, 1.0f);
    const bool trackable = n_regs <= 64;
    uint64_t taint = 0;
    bool amb = false, lost = false;
    if (len <= kLeafOps && predecoded) {
        if (len) leaf_run_deriv(ops, len, R, taint, amb, lost, trackable);
    } else {
        LeafRaw raw = leaf_fetch(cl, len, 0, lane);
        for (uint32_t c0 = 0; c0 < len; c0 += kLeafOps) {
            __syncwarp();
            const uint32_t n = leaf_decode_chunk(ops, raw, len, c0, cpool, lane);
            raw = leaf_fetch(cl, len, c0 + kLeafOps, lane);
            leaf_run_deriv(ops, n, R, taint, amb, lost, trackable);
        }
        __syncwarp();
    }
    *ambig = amb;
    *plain = !lost && !(root_kind == OPND_REG && ((taint >> (root & 63)) & 1));
    if (root_kind == OPND_REG) return d4_of(R[root * 32]);
    return {__ldg(cpool + root), 0.0f, 0.0f, 0.0f};
}

constexpr size_t kLeafSmallBytes = (sizeof(LeafWarpShared) + 15) / 16 * 16;
constexpr uint32_t kLeafSmemRegs = 16;   // shared-memory register file per warp

struct LeafArgs {
    Octree o;
    DevTape bt;
    const RegClause* arena;
    LeafRec* recs;
    uint32_t* rec_top;
    uint32_t rec_cap;
    uint32_t* status;
    unsigned long long* evals;
    LeafWarpScratch* scratch;   // gridDim.x * warps-per-block slices
    float* rd;                  // per warp: n_regs x 4 x 32 floats (long tapes)
    uint32_t smem_regs;         // registers of the shared-memory register file
    uint32_t* next_group;       // work counter (zero at launch)
    const uint32_t* order;      // processing order of the groups (or null)
    unsigned long long* prof;   // debug: 8 per group (cycles by section, feature calls, E)
    float* featws;              // per warp: n_regs x kRegBlock floats of feature lists
    EdgeRec* edges;             // crossing-edge QEFs of all groups
    unsigned long long* edge_top;
    uint32_t edge_cap;
    GroupEdges* group_edges;    // one per group
    uint32_t* rec_group;        // per leaf record: group * 8 + cell
    uint32_t* next_group2;      // work counter of k_leaf_qef (zero at launch)
};

__global__ void __launch_bounds__(256, 3)
k_leaf_groups(LeafArgs A, uint32_t n_groups)
{
    extern __shared__ __align__(16) unsigned char lsmem[];
    // The edge search's sample fractions j / 15, divided once per block
    // (the same correctly rounded quotients as dividing at every sample).
    __shared__ double frac_tab[16];
    if (threadIdx.x < 16) frac_tab[threadIdx.x] = threadIdx.x / (16 - 1.0);
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    LeafWarpShared* S = reinterpret_cast<LeafWarpShared*>(lsmem) + warp;
    // Register file of the tape interpreters (n_regs x 4 x 32 floats): in
    // shared memory when the group's tape uses
    // at most A.smem_regs registers (leaf tapes are renumbered compactly, so
    // nearly all do), else in a per-warp slice of global memory.
    float* Rs = reinterpret_cast<float*>(lsmem + kLeafSmallBytes * wpb) +
                static_cast<size_t>(warp) * A.smem_regs * 128;
    float* Rgl = A.rd + (static_cast<size_t>(blockIdx.x) * wpb + warp) * A.bt.n_regs * 128;
    // Decoded clauses of the group's tape (leaf_interp.cuh), after the
    // register files.
    const uint32_t ops_off = static_cast<uint32_t>(kLeafSmallBytes * wpb +
                                                   static_cast<size_t>(wpb) * A.smem_regs * 128 * 4 +
                                                   static_cast<size_t>(warp) * kLeafOps * sizeof(LeafOp));
    LeafWarpScratch* W = A.scratch + static_cast<size_t>(blockIdx.x) * wpb + warp;
    uint64_t my_evals = 0, my_devals = 0;
    // Persistent warps take the next group from a shared counter (group
    // costs vary by orders of magnitude with the tape length).
    while (true) {
    uint32_t g = 0;
    if (lane == 0) g = atomicAdd(A.next_group, 1u);
    g = __shfl_sync(0xffffffffu, g, 0);
    if (g >= n_groups) break;
    if (A.order) g = A.order[g];
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
        tr = root_tape_ref(A.bt);
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
    const long long t_group = clock64();
    unsigned long long feat_cycles = 0, feat_calls = 0;
    const DevTape tb = with_tape(A.bt, tr);
    const bool rs = tb.n_regs <= A.smem_regs;
    float* R = rs ? Rs : Rgl;
    const uint32_t rsoff = static_cast<uint32_t>(reinterpret_cast<unsigned char*>(Rs) - lsmem);
#define RF_CALL(fn, ...) (rs ? fn<true>(__VA_ARGS__) : fn<false>(__VA_ARGS__))
#define RF_VALUE4(...) (rs ? warp_value4<true>(__VA_ARGS__) : warp_value4<false>(__VA_ARGS__))
    // Tapes that fit the buffer are decoded once for the whole group.
    __syncwarp();
    const FeatCtx fc{A.featws + (static_cast<size_t>(blockIdx.x) * wpb + warp) *
                                    A.bt.n_regs * kRegBlock,
                     &W->fs, A.status};

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
    {
        uint32_t amb4 = 0;
        const float4 v4 = RF_VALUE4(tb.cpool, tb.root_kind, tb.root, cl, tr.len, rsoff, R,
                                    lane, splat4(px), splat4(py), splat4(pz), true, &amb4);
        cv = v4.x;
        camb = (amb4 & 1) != 0;
        const uint32_t act = __ballot_sync(0xffffffffu, lane < npts);
        if (lane == 0) my_evals += static_cast<uint64_t>(__popc(act)) * tr.len;
    }
    uint8_t cst = CELL_EMPTY;
    bool need_d = false, need_f = false;
    if (lane < npts) {
        if (cv > 0 || cv != cv) cst = CELL_EMPTY;
        else if (cv < 0) cst = CELL_FILLED;
        else if (!camb) need_d = true;
        else need_f = true;
    }
    if (__any_sync(0xffffffffu, need_d || need_f)) {
        bool amb = false, plain = false;
        const D4 d = RF_CALL(leaf_deriv, tb.cpool, tb.root_kind, tb.root, tb.n_regs, cl,
                             tr.len, rsoff, R, ops_off, lane, px, py, pz, &amb, &plain, false);
        const uint32_t act = __ballot_sync(0xffffffffu, need_d || need_f);
        if (lane == 0) my_devals += static_cast<uint64_t>(__popc(act)) * tr.len;
        if (need_d) {
            cst = (d.dx != 0 || d.dy != 0 || d.dz != 0) ? CELL_FILLED : CELL_EMPTY;
        }
        if (need_f && plain) {
            // FeatureEvaluator::isInside with one feature at a zero value.
            const float g[3] = {d.dx, d.dy, d.dz};
            cst = sqrtf(fdot(g, g)) > 0 ? CELL_FILLED : CELL_EMPTY;
            need_f = false;
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
            const long long t0 = clock64();
            const bool inside = dev_is_inside(fc, tb, cl, tr.len, qx, qy, qz, lane);
            feat_cycles += clock64() - t0;
            ++feat_calls;
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

    const long long t_crossing = clock64();
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
            EdgeSlot& es = W->e[first_slot + before];
            const bool f0 = S->st[p0] == CELL_FILLED;
            double a[3], b[3];
            pt_pos(f0 ? p0 : p1, a);
            pt_pos(f0 ? p1 : p0, b);
            for (int k = 0; k < 3; ++k) { es.t0[k] = a[k]; es.t1[k] = b[k]; }
        }
        __syncwarp();
        if (lane == 0) S->nslots = static_cast<uint8_t>(first_slot + __popc(m));
        __syncwarp();
    }
    const int E = S->nslots;

    // --- edge search: 4 rounds of 16 points (dc_tree.inl:326-410) -------
    // Each round samples an edge's bracket [t0, t1] at 16 evenly spaced
    // points j = 0..15 and keeps [s(j-1), s(j)] around the first sample j >= 1
    // that is outside; failing that, the last one, unless it is an inside
    // zero.  s(0) = t0 is never tested, and s(15) = t1 is the previous
    // round's outside end (round 1: the corner known to be outside), which is
    // never an inside zero, so the outcome is "first outside j in 1..14,
    // else 15": only 14 samples per edge are evaluated.  One pass holds nine
    // edges (126 of the 4 x 32 sample slots): slot p = 32k + lane of
    // sub-batch k is sample 1 + p % 14 of edge base + p / 14.  Most groups
    // have nine crossing edges, one pass per round.
    auto sample = [&](int slot, int j, double q[3]) {
        const double frac = frac_tab[j];
        const EdgeSlot& es = W->e[slot];
        for (int k = 0; k < 3; ++k) q[k] = es.t0[k] * (1 - frac) + es.t1[k] * frac;
    };
    constexpr int kEdgesPerPass = 9, kSamples = 14;
    for (int round = 0; round < 4; ++round) {
        for (int base = 0; base < E; base += kEdgesPerPass) {
            float qx[4] = {0, 0, 0, 0}, qy[4] = {0, 0, 0, 0}, qz[4] = {0, 0, 0, 0};
            bool act[4];
            int n_act = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int p = 32 * k + lane;
                const int slot = base + p / kSamples;
                act[k] = p < kEdgesPerPass * kSamples && slot < E;
                if (act[k]) {
                    double q[3];
                    sample(slot, 1 + p % kSamples, q);
                    qx[k] = static_cast<float>(q[0]);
                    qy[k] = static_cast<float>(q[1]);
                    qz[k] = static_cast<float>(q[2]);
                    ++n_act;
                }
            }
            uint32_t unused = 0;
            const float4 v4 = RF_VALUE4(tb.cpool, tb.root_kind, tb.root, cl, tr.len,
                                        rsoff, R, lane,
                                        make_float4(qx[0], qx[1], qx[2], qx[3]),
                                        make_float4(qy[0], qy[1], qy[2], qy[3]),
                                        make_float4(qz[0], qz[1], qz[2], qz[3]), false, &unused);
            my_evals += static_cast<uint64_t>(__reduce_add_sync(0xffffffffu, n_act)) * tr.len;
            const float vs[4] = {v4.x, v4.y, v4.z, v4.w};
            uint32_t term[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const float v = vs[k];
                // A sample exactly on the surface is resolved with
                // FeatureEvaluator::isInside: for a point without tied
                // min/max that is "gradient is non-zero" (one feature),
                // otherwise the full feature search.
                const bool zero = act[k] && v == 0;
                bool inside = true;
                if (__any_sync(0xffffffffu, zero)) {
                    bool amb = false, plain = false;
                    const D4 dg = RF_CALL(leaf_deriv, tb.cpool, tb.root_kind, tb.root,
                                          tb.n_regs, cl, tr.len, rsoff, R, ops_off, lane,
                                          qx[k], qy[k], qz[k], &amb, &plain, false);
                    const uint32_t zact = __ballot_sync(0xffffffffu, zero);
                    if (lane == 0) my_devals += static_cast<uint64_t>(__popc(zact)) * tr.len;
                    amb = amb && !plain;   // a settled tie leaves one plain feature
                    if (zero && !amb) {
                        const float g[3] = {dg.dx, dg.dy, dg.dz};
                        inside = sqrtf(fdot(g, g)) > 0;
                    }
                    uint32_t full = __ballot_sync(0xffffffffu, zero && amb);
                    while (full) {
                        const int src = __ffs(full) - 1;
                        full &= full - 1;
                        const float zx = __shfl_sync(0xffffffffu, qx[k], src);
                        const float zy = __shfl_sync(0xffffffffu, qy[k], src);
                        const float zz = __shfl_sync(0xffffffffu, qz[k], src);
                        const long long t0 = clock64();
                        const bool in = dev_is_inside(fc, tb, cl, tr.len, zx, zy, zz, lane);
                        feat_cycles += clock64() - t0;
                        ++feat_calls;
                        if (lane == src) inside = in;
                    }
                }
                term[k] = __ballot_sync(0xffffffffu, act[k] && (v > 0 || (v == 0 && !inside)));
            }
            // New brackets, one lane per edge, from the old ones.
            if (lane < kEdgesPerPass && base + lane < E) {
                const int p0 = kSamples * lane;
                const int w0 = p0 >> 5, sh = p0 & 31;
                uint32_t lo_w = 0, hi_w = 0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (k == w0) lo_w = term[k];
                    if (k == w0 + 1) hi_w = term[k];
                }
                const uint64_t bits = ((static_cast<uint64_t>(hi_w) << 32) | lo_w) >> sh;
                const uint32_t t = static_cast<uint32_t>(bits) & ((1u << kSamples) - 1);
                const int pick = t ? __ffs(t) : 15;   // sample index of the outside end
                const int s_ = base + lane;
                double nt0[3], nt1[3];
                sample(s_, pick - 1, nt0);
                sample(s_, pick, nt1);
                EdgeSlot& es = W->e[s_];
                for (int c = 0; c < 3; ++c) { es.t0[c] = nt0[c]; es.t1[c] = nt1[c]; }
            }
            __syncwarp();
        }
    }

    const long long t_gradients = clock64();
    const long long t_vertices = t_gradients;
    // --- hand the final brackets to k_leaf_qef, the lattice edge map and
    //     the records to the vertex kernel ---------------------------------
    {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(A.edge_top, static_cast<unsigned long long>(E));
        base = __shfl_sync(0xffffffffu, base, 0);
        const bool fits = base + E <= A.edge_cap;
        GroupEdges& ge = A.group_edges[single ? 0 : g];
        if (!fits) {
            if (lane == 0) {
                atomicOr(A.status, ST_EDGE_OVERFLOW);
                ge.base = 0xffffffffu;
                ge.n_edges = 0;
            }
        } else {
            for (int s_ = lane; s_ < E; s_ += 32) {
                EdgeRec& r = A.edges[base + s_];
                for (int k = 0; k < 3; ++k) {
                    r.t0[k] = W->e[s_].t0[k];
                    r.t1[k] = W->e[s_].t1[k];
                }
            }
            if (lane == 0) {
                ge.base = static_cast<uint32_t>(base);
                ge.n_edges = static_cast<uint8_t>(E);
            }
            for (int k = lane; k < n_lat_edges; k += 32) ge.slot_of[k] = S->slot_of[k];
            if (lane < ncell && S->rec[lane] >= 0) {
                A.rec_group[S->rec[lane]] = (single ? 0u : g * 8u) + static_cast<uint32_t>(lane);
            }
        }
    }
    (void)base_coords;
    if (A.prof && lane == 0) {
        const long long t_end = clock64();
        unsigned long long* P = A.prof + 8ull * g;
        P[0] = t_end - t_group;
        P[1] = feat_cycles;
        P[2] = feat_calls;
        P[3] = E;
        P[4] = t_crossing - t_group;      // corners, classification
        P[5] = t_gradients - t_crossing;  // crossing edges, edge search
        P[6] = t_vertices - t_gradients;  // gradients, QEF pushes
        P[7] = t_end - t_vertices;        // edge records
    }
    }   // groups
#undef RF_CALL
#undef RF_VALUE4
    if (lane == 0) {
        atomicAdd(A.evals, static_cast<unsigned long long>(my_evals));
        atomicAdd(A.evals + 1, static_cast<unsigned long long>(my_devals));
    }
}

/// Gradients at the two ends of every crossing edge's final bracket and the
/// edge's QEF (dc_tree.inl:412-471): one warp per leaf group (the group's
/// tape), one bracket end per lane, then each lane pushes whole edges
/// (inside end first).  Points where a min / max is tied use every feature
/// gradient instead (eval_feature.cpp:125-169).  A launch of its own, so
/// that the derivative interpreter does not share the instruction cache
/// with the value interpreter of the edge search.
__global__ void __launch_bounds__(256, 3)
k_leaf_qef(LeafArgs A, uint32_t n_groups)
{
    extern __shared__ __align__(16) unsigned char lsmem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    float* Rs = reinterpret_cast<float*>(lsmem + kLeafSmallBytes * wpb) +
                static_cast<size_t>(warp) * A.smem_regs * 128;
    float* Rgl = A.rd + (static_cast<size_t>(blockIdx.x) * wpb + warp) * A.bt.n_regs * 128;
    const uint32_t ops_off = static_cast<uint32_t>(kLeafSmallBytes * wpb +
                                                   static_cast<size_t>(wpb) * A.smem_regs * 128 * 4 +
                                                   static_cast<size_t>(warp) * kLeafOps * sizeof(LeafOp));
    LeafWarpScratch* W = A.scratch + static_cast<size_t>(blockIdx.x) * wpb + warp;
    const FeatCtx fc{A.featws + (static_cast<size_t>(blockIdx.x) * wpb + warp) *
                                    A.bt.n_regs * kRegBlock,
                     &W->fs, A.status};
    uint64_t my_devals = 0;
    const Octree& o = A.o;
    const int Ld = o.levels;
    const bool single = (Ld == 0);
    while (true) {
        uint32_t g = 0;
        if (lane == 0) g = atomicAdd(A.next_group2, 1u);
        g = __shfl_sync(0xffffffffu, g, 0);
        if (g >= n_groups) break;
        if (A.order) g = A.order[g];
        const GroupEdges& ge = A.group_edges[single ? 0 : g];
        const uint32_t gbase = ge.base;
        const int E = ge.n_edges;
        if (gbase == 0xffffffffu || E == 0) continue;
        const TapeRef tr = single ? root_tape_ref(A.bt) : o.lv[Ld].group_tape[g];
        const RegClause* cl = A.arena + tr.off;
        const DevTape tb = with_tape(A.bt, tr);
        const bool rs = tb.n_regs <= A.smem_regs;
        float* R = rs ? Rs : Rgl;
        const uint32_t rsoff = static_cast<uint32_t>(reinterpret_cast<unsigned char*>(Rs) - lsmem);
        __syncwarp();
        if (tr.len <= kLeafOps) {
            leaf_decode_chunk(leaf_ops(ops_off), leaf_fetch(cl, tr.len, 0, lane), tr.len, 0,
                              tb.cpool, lane);
        }
        EdgeRec* er = A.edges + gbase;
        for (int base = 0; base < 2 * E; base += 32) {
            const int p = base + lane;
            const bool active = p < 2 * E;
            double q[3] = {0, 0, 0};
            if (active) {
                const EdgeRec& e = er[p >> 1];
                for (int k = 0; k < 3; ++k) q[k] = (p & 1) ? e.t1[k] : e.t0[k];
            }
            bool amb = false, plain = false;
            const D4 d = rs ? leaf_deriv<true>(tb.cpool, tb.root_kind, tb.root, tb.n_regs, cl,
                                               tr.len, rsoff, R, ops_off, lane,
                                               static_cast<float>(q[0]), static_cast<float>(q[1]),
                                               static_cast<float>(q[2]), &amb, &plain, true)
                            : leaf_deriv<false>(tb.cpool, tb.root_kind, tb.root, tb.n_regs, cl,
                                                tr.len, rsoff, R, ops_off, lane,
                                                static_cast<float>(q[0]), static_cast<float>(q[1]),
                                                static_cast<float>(q[2]), &amb, &plain, true);
            const uint32_t gact = __ballot_sync(0xffffffffu, active);
            if (lane == 0) my_devals += static_cast<uint64_t>(__popc(gact)) * tr.len;
            amb = amb && !plain;   // a settled tie leaves one plain feature
            if (active) {
                EdgeSlot& es = W->e[p >> 1];
                float* gg = (p & 1) ? es.g1 : es.g0;
                gg[0] = d.dx; gg[1] = d.dy; gg[2] = d.dz; gg[3] = d.v;
                es.amb[p & 1] = amb;
            }
        }
        __syncwarp();
        const uint32_t any_amb = __ballot_sync(0xffffffffu, [&] {
            bool a = false;
            for (int s_ = lane; s_ < E; s_ += 32) a |= W->e[s_].amb[0] || W->e[s_].amb[1];
            return a;
        }());
        if (!any_amb) {
            for (int s_ = lane; s_ < E; s_ += 32) {
                const EdgeSlot& es = W->e[s_];
                EdgeRec& r = er[s_];
                Qef qf;
                qef_zero(qf);
                for (int side = 0; side < 2; ++side) {
                    const float* gg = side ? es.g1 : es.g0;
                    const double* pos = side ? r.t1 : r.t0;
                    const double gd[3] = {gg[0], gg[1], gg[2]};
                    qef_push(qf, pos, gd, static_cast<double>(gg[3]));
                }
                r.q = qf;
                r.exists = 1;
                r.rank = 0;
            }
        } else {
            for (int s_ = lane; s_ < E; s_ += 32) {
                qef_zero(er[s_].q);
                er[s_].exists = 0;
                er[s_].rank = 0;
            }
            __syncwarp();
            for (int s_ = 0; s_ < E; ++s_) {
                const EdgeSlot& es = W->e[s_];
                EdgeRec& r = er[s_];
                for (int side = 0; side < 2; ++side) {
                    const float* gg = side ? es.g1 : es.g0;
                    const double* pos = side ? r.t1 : r.t0;
                    if (es.amb[side]) {
                        dev_push_features(fc, tb, cl, tr.len, pos, static_cast<double>(gg[3]),
                                          &r.q, &r.exists, lane);
                    } else if (lane == 0) {
                        const double gd[3] = {gg[0], gg[1], gg[2]};
                        qef_push(r.q, pos, gd, static_cast<double>(gg[3]));
                        r.exists = 1;
                    }
                    __syncwarp();
                }
            }
        }
        __syncwarp();
    }
    if (lane == 0) atomicAdd(A.evals + 1, static_cast<unsigned long long>(my_devals));
}

/// Intersection::get_rank (intersection.hpp:67-88) of every crossing edge's
/// QEF, one thread per edge.
__global__ void __launch_bounds__(128)
k_edge_rank(EdgeRec* edges, const unsigned long long* edge_top, uint32_t cap)
{
    const uint64_t n = min(static_cast<unsigned long long>(cap), *edge_top);
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        edges[i].rank = static_cast<uint8_t>(qef_rank(edges[i].q));
    }
}

/// Per-patch vertices of the leaf records (dc_tree.inl:474-549), one thread
/// per record: the patch's crossing edges found through the group's lattice
/// edge map, the mass point over the edges of highest rank, the summed QEF
/// and DCTree::findVertex.  `single`: the root cell is the only leaf (a
/// 2 x 2 x 2 lattice instead of the 3 x 3 x 3 of a sibling group).
__global__ void __launch_bounds__(128)
k_leaf_vertices(LeafRec* recs, const uint32_t* rec_top, uint32_t rec_cap,
                const uint32_t* rec_group, const GroupEdges* group_edges, uint32_t n_groups,
                const EdgeRec* edges, uint32_t edge_cap, int single)
{
    const uint32_t n_recs = min(rec_cap, *rec_top);
    const int n = single ? 2 : 3;
    const int seg = n - 1;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n_recs;
         r += gridDim.x * blockDim.x) {
        const uint32_t gi = rec_group[r];
        // records of groups whose edges did not fit have none (the mesh is
        // rendered again with more room)
        if (gi == 0xffffffffu || (gi >> 3) >= n_groups) continue;
        const int cell = static_cast<int>(gi & 7);
        const GroupEdges& ge = group_edges[gi >> 3];
        if (ge.base == 0xffffffffu || ge.base + ge.n_edges > edge_cap) continue;
        LeafRec& L = recs[r];
        const uint8_t mask = L.corner_mask;
        auto lat_pt = [&](int corner) {
            const int cx = cell & 1, cy = (cell >> 1) & 1, cz = (cell >> 2) & 1;
            return (cx + (corner & 1)) + n * ((cy + ((corner >> 1) & 1)) +
                                              n * (cz + ((corner >> 2) & 1)));
        };
        const int np = c_tab.npatch[mask];
        for (int patch = 0; patch < np; ++patch) {
            const int ne = c_tab.nedge[mask][patch];
            int slots[12];
            for (int k = 0; k < ne; ++k) {
                const int ca = c_tab.v[mask][patch][k][0];
                const int cb = c_tab.v[mask][patch][k][1];
                // lattice edge between the two corners of this cell
                const int pa = lat_pt(ca), pb = lat_pt(cb);
                const int lo_p = pa < pb ? pa : pb;
                const int diff = (pa < pb ? pb - pa : pa - pb);
                const int ax = diff == 1 ? 0 : diff == n ? 1 : 2;
                const int c0 = lo_p % n, c1 = (lo_p / n) % n, c2 = lo_p / (n * n);
                int le;
                if (ax == 0) le = c0 + seg * (c1 + n * c2);
                else if (ax == 1) le = c1 + seg * (c0 + n * c2);
                else le = c2 + seg * (c0 + n * c1);
                le += ax * seg * n * n;
                const int sl = ge.slot_of[le];
                slots[k] = sl < 0 ? -1 : static_cast<int>(ge.base) + sl;
            }
            int max_rank = 0;
            for (int k = 0; k < ne; ++k) {
                if (slots[k] >= 0 && edges[slots[k]].exists && edges[slots[k]].rank > max_rank) {
                    max_rank = edges[slots[k]].rank;
                }
            }
            Qef q;
            qef_zero(q);
            for (int k = 0; k < ne; ++k) {
                if (slots[k] < 0 || !edges[slots[k]].exists) continue;
                const EdgeRec& es = edges[slots[k]];
                if (es.rank == max_rank) {
                    q.mass[0] += es.q.mass[0] / es.q.mass[3];
                    q.mass[1] += es.q.mass[1] / es.q.mass[3];
                    q.mass[2] += es.q.mass[2] / es.q.mass[3];
                    q.mass[3] += 1.0;
                }
            }
            for (int k = 0; k < ne; ++k) {
                if (slots[k] < 0 || !edges[slots[k]].exists) continue;
                qef_add(q, edges[slots[k]].q);
            }
            double v[3];
            int rank = 0;
            qef_vertex(q, v, &rank);
            for (int k = 0; k < 3; ++k) L.vert[patch][k] = v[k];
            if (patch == np - 1) {
                for (int k = 0; k < 4; ++k) L.mass[k] = q.mass[k];
                for (int k = 0; k < 6; ++k) L.ata[k] = q.ata[k];
                for (int k = 0; k < 3; ++k) L.atb[k] = q.atb[k];
                L.btb = q.btb;
                L.rank = static_cast<uint8_t>(rank);
            }
        }
    }
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
    // (Tape::getBase, tape.cpp:188-209); the unpruned tape otherwise.  Any
    // tape valid at the point gives the same value, so when this cell
    // contains the vertex, the shortest one is taken instead: that of the
    // deepest cell below it that contains the vertex and was ambiguous when
    // its interval was evaluated (so has a pruned tape).
    const float vf[3] = {static_cast<float>(v[0]), static_cast<float>(v[1]),
                         static_cast<float>(v[2])};
    auto contains = [&](int dd, uint32_t ii) {
        double blo[3], bhi[3];
        cell_bounds(o, dd, o.lv[dd].coords[ii], blo, bhi);
        bool in = true;
        for (int a = 0; a < 3; ++a) {
            in &= vf[a] >= static_cast<float>(blo[a]) && vf[a] <= static_cast<float>(bhi[a]);
        }
        return in;
    };
    TapeRef tr = root_tape_ref(A.bt);
    if (contains(d, i)) {
        int dd = d;
        uint32_t ii = i;
        while (dd + 1 < o.levels) {
            const int32_t k = o.lv[dd].child_group[ii];
            if (k < 0) break;
            bool found = false;
            for (uint32_t j = 0; j < 8 && !found; ++j) {
                const uint32_t c = 8 * static_cast<uint32_t>(k) + j;
                if (o.lv[dd + 1].child_group[c] >= 0 && contains(dd + 1, c)) {
                    ii = c;
                    found = true;
                }
            }
            if (!found) break;
            ++dd;
        }
        tr = o.lv[dd].cell_tape[ii];
    } else {
        int dd = d;
        uint32_t ii = i;
        while (dd > 0) {
            ii = o.lv[dd].group_parent[ii >> 3];
            --dd;
            if (contains(dd, ii)) {
                tr = o.lv[dd].cell_tape[ii];
                break;
            }
        }
    }
    const float value = thread_value(with_tape(A.bt, tr), A.arena + tr.off, tr.len, csmem, tid, B,
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

/// Sort keys for the leaf groups: tape length (longest first), so that the
/// persistent leaf kernel starts the expensive groups early.
__global__ void k_leaf_order_keys(const TapeRef* group_tape, uint32_t n,
                                  uint32_t* keys, uint32_t* vals)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = group_tape[i].len;
    vals[i] = i;
}

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
/// group's parent, tapes and child coordinates.
__global__ void k_build_groups(Octree o, int d, const uint32_t* scan, uint32_t* nregs_next)
{
    const LevelView& lv = o.lv[d];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool branch = i < lv.n_cells && lv.type[i] == CELL_BRANCH;
    // largest register count of the next depth's group tapes (sizes the
    // group-mode interval kernel's shared memory for that depth)
    const uint32_t nr = branch ? lv.cell_tape[i].nregs : 0u;
    const uint32_t wmax = __reduce_max_sync(0xffffffffu, nr);
    if ((threadIdx.x & 31) == 0 && wmax) atomicMax(nregs_next, wmax);
    if (i >= lv.n_cells) return;
    if (!branch) {
        lv.child_group[i] = -1;
        return;
    }
    const uint32_t g = scan[i];
    lv.child_group[i] = static_cast<int32_t>(g);
    LevelView& nv = o.lv[d + 1];
    nv.group_parent[g] = i;
    nv.group_tape[g] = lv.cell_tape[i];
    nv.group_list[g] = lv.cell_list[i];
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

// Binary STL records (mesh.cpp:177-193): per triangle a zero normal, its
// three vertices and a zero attribute word, 50 bytes, little-endian like
// the host.  50-byte records are only 2-byte aligned, so a block packs its
// kStlBlock records in shared memory as 16-bit words and writes them out as
// one contiguous run of words.
constexpr uint32_t kStlBlock = 128;
constexpr uint32_t kStlWords = 25;

__global__ void __launch_bounds__(kStlBlock)
k_pack_stl(const float* __restrict__ verts, const uint32_t* __restrict__ tris, uint32_t n,
           uint16_t* __restrict__ out)
{
    __shared__ uint16_t rec[kStlBlock * kStlWords];
    const uint32_t first = blockIdx.x * kStlBlock;
    const uint32_t i = first + threadIdx.x;
    uint16_t* r = rec + threadIdx.x * kStlWords;
    if (i < n) {
        for (int k = 0; k < 6; ++k) r[k] = 0;
        for (int v = 0; v < 3; ++v) {
            const uint32_t id = tris[3 * static_cast<size_t>(i) + v];
            for (int a = 0; a < 3; ++a) {
                const uint32_t bits = __float_as_uint(verts[3 * static_cast<size_t>(id) + a]);
                r[6 + 6 * v + 2 * a] = static_cast<uint16_t>(bits & 0xffff);
                r[6 + 6 * v + 2 * a + 1] = static_cast<uint16_t>(bits >> 16);
            }
        }
        r[24] = 0;
    }
    __syncthreads();
    const uint32_t m = min(kStlBlock, n - first);
    uint16_t* dst = out + static_cast<size_t>(first) * kStlWords;
    for (uint32_t k = threadIdx.x; k < m * kStlWords; k += kStlBlock) dst[k] = rec[k];
}

// libfive_mesh_coords' index list (libfive.cpp:375-388): a, b, c, -1 per
// triangle.
__global__ void k_pack_coords(const uint32_t* __restrict__ tris, uint32_t n, int4* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const size_t t = 3 * static_cast<size_t>(i);
        out[i] = make_int4(static_cast<int>(tris[t]), static_cast<int>(tris[t + 1]),
                           static_cast<int>(tris[t + 2]), -1);
    }
}

}  // namespace lfb

////////////////////////////////////////////////////////////////////////////////
// Host driver

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <vector>

#include "mesher.hpp"

namespace lfb {

namespace {

/// What one mesh in flight owns on the host side: grow-only device buffers
/// keyed by purpose, the stream its work runs on and download()'s
/// page-locked staging buffer.  A context serves one mesh at a time (its
/// mutex) and keeps its buffers from call to call.
/// Freed scratch the device's memory pool keeps across synchronisations
/// (for the next mesh of any context) before it returns memory to the driver.
constexpr uint64_t kPoolKeepBytes = uint64_t(32) << 30;

struct Workspace {
    std::mutex mu;
    cudaStream_t s = 0;
    std::map<int, DevBuf> bufs;
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    // Leaf edge records per leaf group (grows when a mesh needs more; the
    // mesh is then rendered again).
    uint32_t edges_per_group = 16;
    bool retry = false;

    template <class T>
    T* get(int key, size_t count)
    {
        DevBuf& b = bufs[key];
        if (!b.ordered) {
            // scratch lives in the device's memory pool, allocated in this
            // context's stream order
            b.ordered = true;
            b.stream = s;
        }
        if (!b.reserve(std::max<size_t>(count, 1) * sizeof(T))) return nullptr;
        return b.as<T>();
    }
};

/// The context of single-mesh calls: work on the legacy default stream, as
/// callers that time those calls with events on that stream expect.
Workspace& default_workspace()
{
    static Workspace* w = new Workspace;   // never destroyed: see pinned_pool()
    return *w;
}

/// Context k of the concurrent batch path, created on first use with its
/// own non-blocking stream (so that batched meshes overlap each other and
/// never wait on unrelated default-stream work).
struct StreamPool {
    std::mutex mu;
    std::vector<Workspace*> pool;
};

StreamPool& stream_pool()
{
    static StreamPool* p = new StreamPool;   // never destroyed, like the contexts
    return *p;
}

Workspace* stream_workspace(unsigned k)
{
    auto& sp = stream_pool();
    std::lock_guard<std::mutex> lock(sp.mu);
    auto& pool = sp.pool;
    while (pool.size() <= k) {
        auto* w = new Workspace;
        if (!cuda_ok(cudaStreamCreateWithFlags(&w->s, cudaStreamNonBlocking), "stream")) {
            delete w;
            return nullptr;
        }
        pool.push_back(w);
    }
    return pool[k];
}

enum BufKey {
    K_ARENA = 1, K_STATUS, K_COUNTERS, K_RECS, K_FLAGS, K_SCAN,
    K_CUBTMP, K_TASK_A, K_TASK_B, K_TRIS, K_USED, K_VSCAN, K_VERTS, K_FEAT,
    K_LIST_A, K_LIST_B, K_WIDE_S, K_WIDE_SN, K_WIDE_P, K_WIDE_LIVE, K_WIDE_NEW,
    K_WIDE_ST2, K_WIDE_L1, K_WIDE_WL, K_LEAF_RD, K_ORDER_K0, K_ORDER_K1,
    K_ORDER_V0, K_ORDER_V1, K_SORTTMP, K_PROF, K_GDEC, K_GLAST, K_FEATWS,
    K_EDGES, K_GEDGES, K_RECGROUP, K_NREGS, K_STL, K_COORDS,
    K_LEVEL = 100,
};

bool upload_tables()
{
    static std::mutex mu;
    static bool ready = false;
    std::lock_guard<std::mutex> lock(mu);
    if (ready) return true;
    static DcTables t;
    build_dc_tables(t);
    if (!cuda_ok(cudaMemcpyToSymbol(c_tab, &t, sizeof(t)), "dc tables")) return false;
    ready = true;
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

/// Cells per level up to which a whole block works on each cell
/// (kBlockModeCells; LFB_BLOCK_MODE_CELLS overrides it, for the parity tests).
uint32_t block_mode_cells()
{
    static const long v = [] {
        const char* e = std::getenv("LFB_BLOCK_MODE_CELLS");
        return e ? std::max(0L, std::atol(e)) : static_cast<long>(kBlockModeCells);
    }();
    return static_cast<uint32_t>(v);
}

/// Cells per level from which the interval stage switches to group mode
/// (kGroupModeCells; the LFB_GROUP_MODE_CELLS environment variable overrides
/// it, which the parity tests use to run both modes on small shapes).
uint32_t group_mode_cells()
{
    static const uint32_t v = [] {
        const char* e = std::getenv("LFB_GROUP_MODE_CELLS");
        return e ? static_cast<uint32_t>(std::max(1L, std::atol(e))) : kGroupModeCells;
    }();
    return v;
}

bool debug_levels()
{
    static const bool on = [] {
        const char* e = std::getenv("LFB_DEBUG_LEVELS");
        return e && e[0] == '1';
    }();
    return on;
}

template <class T>
bool exclusive_scan(Workspace& ws, const T* in, T* out, uint32_t n, cudaStream_t s)
{
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, n, s);
    void* t = ws.get<unsigned char>(K_CUBTMP, tmp);
    if (!t) return false;
    return cuda_ok(cub::DeviceScan::ExclusiveSum(t, tmp, in, out, n, s), "scan");
}

}  // namespace

namespace {

/// Page-locked host blocks for mesh arrays, recycled: a mesh freed by
/// libfive_mesh_delete gives its blocks back for the next one, so a render
/// loop pins memory once and every download is a single direct copy.
struct PinnedPool {
    std::mutex mu;
    std::multimap<size_t, void*> free_blocks;   // capacity -> block
    std::map<void*, size_t> owned;              // every pool block
    size_t free_bytes = 0;
    size_t owned_bytes = 0;
    static constexpr size_t kKeepBytes = size_t(1) << 30;   // cached when free
    // Page-locked memory in use or cached at most; beyond it (many large
    // meshes alive at once) blocks are pageable, since pinning is slow and
    // takes memory from the rest of the host.
    static constexpr size_t kMaxOwned = size_t(4) << 30;
};

PinnedPool& pinned_pool()
{
    static PinnedPool* p = new PinnedPool;   // never destroyed: meshes may outlive statics
    return *p;
}

}  // namespace

void* host_alloc(size_t bytes)
{
    constexpr size_t kGrain = size_t(2) << 20;
    const size_t n = std::max<size_t>((bytes + kGrain - 1) / kGrain * kGrain, kGrain);
    auto& P = pinned_pool();
    {
        std::lock_guard<std::mutex> lock(P.mu);
        auto it = P.free_blocks.lower_bound(n);
        if (it != P.free_blocks.end() && it->first <= 2 * n) {
            void* blk = it->second;
            P.free_bytes -= it->first;
            P.free_blocks.erase(it);
            return blk;
        }
    }
    {
        std::lock_guard<std::mutex> lock(P.mu);
        if (P.owned_bytes + n > PinnedPool::kMaxOwned) {
            return std::aligned_alloc(kGrain, n);   // pageable; same interface
        }
        P.owned_bytes += n;   // reserved before the (slow) pinning call
    }
    void* blk = nullptr;
    if (cudaMallocHost(&blk, n) != cudaSuccess || !blk) {
        cudaGetLastError();
        std::lock_guard<std::mutex> lock(P.mu);
        P.owned_bytes -= n;
        return std::aligned_alloc(kGrain, n);   // pageable fallback; same interface
    }
    std::lock_guard<std::mutex> lock(P.mu);
    P.owned[blk] = n;
    return blk;
}

void host_free(void* p)
{
    if (!p) return;
    auto& P = pinned_pool();
    std::lock_guard<std::mutex> lock(P.mu);
    auto it = P.owned.find(p);
    if (it == P.owned.end()) {
        std::free(p);
        return;
    }
    P.free_blocks.emplace(it->second, p);
    P.free_bytes += it->second;
    // Keep at most kKeepBytes of idle blocks, largest first out.
    while (P.free_bytes > PinnedPool::kKeepBytes && !P.free_blocks.empty()) {
        auto last = std::prev(P.free_blocks.end());
        P.free_bytes -= last->first;
        P.owned_bytes -= last->first;
        P.owned.erase(last->second);
        cudaFreeHost(last->second);
        P.free_blocks.erase(last);
    }
}

MeshOut::~MeshOut()
{
    host_free(verts);
    host_free(tris);
    host_free(coords);
}

libfive_mesh* MeshOut::release()
{
    auto m = new libfive_mesh;
    m->verts = verts;
    m->tris = tris;
    m->vert_count = vert_count;
    m->tri_count = tri_count;
    verts = nullptr;
    tris = nullptr;
    return m;
}

namespace {

/// Device -> pageable host copy: one transfer into a pinned staging buffer
/// (grow-only, kept between calls), then a host copy split over a few
/// threads (a single thread's memcpy is the slow part of a mesh download).
bool download(Workspace& ws, void* dst, const void* src, size_t bytes, cudaStream_t s)
{
    if (bytes == 0) return true;
    bool page_locked = false;
    {
        auto& P = pinned_pool();
        std::lock_guard<std::mutex> lock(P.mu);
        page_locked = P.owned.count(dst) != 0;
    }
    if (page_locked) {
        // Page-locked destination: one direct transfer.
        return cuda_ok(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), "download") &&
               cuda_ok(cudaStreamSynchronize(s), "download");
    }
    void*& pinned = ws.pinned;
    if (bytes > ws.pinned_bytes) {
        if (pinned) cudaFreeHost(pinned);
        pinned = nullptr;
        ws.pinned_bytes = 0;
        const size_t want = std::max<size_t>(bytes + bytes / 4, size_t(8) << 20);
        if (!cuda_ok(cudaMallocHost(&pinned, want), "pinned staging")) return false;
        ws.pinned_bytes = want;
    }
    if (!cuda_ok(cudaMemcpyAsync(pinned, src, bytes, cudaMemcpyDeviceToHost, s), "download") ||
        !cuda_ok(cudaStreamSynchronize(s), "download")) {
        return false;
    }
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t n_threads = std::min<size_t>(std::min<unsigned>(hw, 8u),
                                              std::max<size_t>(1, bytes >> 22));
    const size_t part = (bytes + n_threads - 1) / n_threads;
    auto copy = [&](size_t t) {
        const size_t lo = t * part, hi = std::min(bytes, lo + part);
        if (lo < hi) {
            std::memcpy(static_cast<char*>(dst) + lo, static_cast<const char*>(pinned) + lo,
                        hi - lo);
        }
    };
    std::vector<std::thread> pool;
    for (size_t t = 1; t < n_threads; ++t) pool.emplace_back(copy, t);
    copy(0);
    for (auto& th : pool) th.join();
    return true;
}

}  // namespace

namespace {

/// Stage-timing events, destroyed on every way out of a render.
struct StageEvents {
    cudaEvent_t ev[5] = {};
    bool on = false;
    void create()
    {
        for (auto& e : ev) cudaEventCreate(&e);
        on = true;
    }
    ~StageEvents()
    {
        if (on) {
            for (auto& e : ev) cudaEventDestroy(e);
        }
    }
};

/// Writes the STL file of a mesh whose vertices and triangles (indices from
/// 1, vertex 0 the placeholder) are on the device: header and count, then
/// the records, packed on the device kStlChunk triangles at a time into two
/// alternating device buffers and copied into two page-locked halves, so
/// that the file write of one chunk overlaps the packing and copy of the
/// next.
int stream_stl(Workspace& ws, const char* path, const float* verts, const uint32_t* tris,
               uint32_t n_tri, cudaStream_t s, uint64_t& n_launch)
{
    constexpr uint32_t kStlChunk = 1u << 20;
    const uint32_t chunk = std::min<uint32_t>(kStlChunk, std::max<uint32_t>(n_tri, 1));
    const size_t chunk_bytes = static_cast<size_t>(chunk) * 2 * kStlWords;
    uint16_t* dev = ws.get<uint16_t>(K_STL, 2 * chunk_bytes / 2);
    if (!dev) return LFB_E_CUDA;
    if (2 * chunk_bytes > ws.pinned_bytes) {
        if (ws.pinned) cudaFreeHost(ws.pinned);
        ws.pinned = nullptr;
        ws.pinned_bytes = 0;
        if (!cuda_ok(cudaMallocHost(&ws.pinned, 2 * chunk_bytes), "pinned staging")) {
            return LFB_E_CUDA;
        }
        ws.pinned_bytes = 2 * chunk_bytes;
    }
    std::FILE* f = stl_begin(path, n_tri);
    if (!f) return set_error(LFB_E_INVALID, std::string("could not open ") + path);
    cudaEvent_t done[2];
    if (!cuda_ok(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming), "event") ||
        !cuda_ok(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming), "event")) {
        std::fclose(f);
        return LFB_E_CUDA;
    }
    int rc = 0;
    const uint32_t n_chunks = (n_tri + chunk - 1) / chunk;
    for (uint32_t k = 0; k <= n_chunks && rc == 0; ++k) {
        if (k < n_chunks) {
            const uint32_t first = k * chunk;
            const uint32_t m = std::min(chunk, n_tri - first);
            uint16_t* d = dev + (k & 1) * (chunk_bytes / 2);
            char* h = static_cast<char*>(ws.pinned) + (k & 1) * chunk_bytes;
            k_pack_stl<<<(m + kStlBlock - 1) / kStlBlock, kStlBlock, 0, s>>>(
                verts, tris + 3 * static_cast<size_t>(first), m, d);
            ++n_launch;
            if (!cuda_ok(cudaGetLastError(), "STL kernel") ||
                !cuda_ok(cudaMemcpyAsync(h, d, static_cast<size_t>(m) * 50,
                                         cudaMemcpyDeviceToHost, s), "download") ||
                !cuda_ok(cudaEventRecord(done[k & 1], s), "event")) {
                rc = LFB_E_CUDA;
            }
        }
        if (rc == 0 && k > 0) {
            // the previous chunk: wait for its copy, then write it
            const uint32_t p = k - 1;
            const char* h = static_cast<const char*>(ws.pinned) + (p & 1) * chunk_bytes;
            const size_t bytes = static_cast<size_t>(std::min(chunk, n_tri - p * chunk)) * 50;
            if (!cuda_ok(cudaEventSynchronize(done[p & 1]), "download")) {
                rc = LFB_E_CUDA;
            } else if (std::fwrite(h, 1, bytes, f) != bytes) {
                rc = set_error(LFB_E_INVALID, std::string("could not write ") + path);
            }
        }
    }
    cudaStreamSynchronize(s);
    cudaEventDestroy(done[0]);
    cudaEventDestroy(done[1]);
    if (std::fclose(f) != 0 && rc == 0) {
        rc = set_error(LFB_E_INVALID, std::string("could not write ") + path);
    }
    return rc;
}

/// One mesh in the context `ws` (held by the caller), on its stream; one
/// attempt (render_in retries when a capacity estimate was too small).
int render_once(Workspace& ws, GpuTape& g, const libfive_region3& R, double min_feature,
                double max_err, MeshOut& out, lfb_mesh_stats* stats,
                const volatile int32_t* cancel, bool first_attempt)
{
    if (!upload_tables()) return LFB_E_CUDA;
    cudaStream_t s = ws.s;
    // Cancellation (BRepSettings::cancel, polled by WorkerPool::run,
    // worker_pool.inl:105, and the dual walk, dual.hpp:315): checked at
    // every point where the host waits for the stream anyway.
    auto cancelled = [&] {
        if (cancel && *cancel) {
            cudaStreamSynchronize(s);
            set_error(LFB_E_CANCELLED, "mesh cancelled");
            return true;
        }
        return false;
    };
    if (cancelled()) return LFB_E_CANCELLED;
    const bool small = debug_hooks().small_capacity.load() != 0;
    if (small) {
        // test hook: start from empty buffers and minimal capacities
        cudaStreamSynchronize(s);
        ws.bufs.clear();
        if (first_attempt) ws.edges_per_group = 1;
    }
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
    unsigned long long* counters = ws.get<unsigned long long>(K_COUNTERS, 10);
    if (!status || !counters) return LFB_E_CUDA;
    cudaMemsetAsync(status, 0, sizeof(uint32_t), s);
    cudaMemsetAsync(counters, 0, 10 * sizeof(unsigned long long), s);
    unsigned long long* edge_top = counters + 8;
    unsigned long long* arena_top = counters + 1;
    uint32_t* rec_top = reinterpret_cast<uint32_t*>(counters + 2);
    unsigned long long* evals = counters + 3;
    unsigned long long* list_top = counters + 5;
    if (!g.ensure_wide()) return LFB_E_UNSUPPORTED;

    // Register-tape arena: the unpruned tape first, pruned tapes appended
    // (every depth's tapes stay: the collapse pass evaluates points with
    // them).  It keeps its size from call to call.
    auto cap_of = [&](int key, size_t elem) {
        return static_cast<uint64_t>(ws.bufs[key].bytes / elem);
    };
    RegClause* arena = ws.get<RegClause>(
        K_ARENA, std::max<uint64_t>(cap_of(K_ARENA, sizeof(RegClause)),
                                    small ? bt.n + 64
                                          : std::max<size_t>(bt.n * 64 + (1u << 20), 1u << 22)));
    if (!arena) return LFB_E_CUDA;
    uint64_t arena_cap = cap_of(K_ARENA, sizeof(RegClause));
    if (bt.n && !cuda_ok(cudaMemcpyAsync(arena, bt.clauses, bt.n * sizeof(RegClause),
                                         cudaMemcpyDeviceToDevice, s), "arena")) {
        return LFB_E_CUDA;
    }
    unsigned long long top_host = bt.n;
    cudaMemcpyAsync(arena_top, &top_host, sizeof(top_host), cudaMemcpyHostToDevice, s);

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
        lv.cell_list = ws.get<ListRef>(k + 7, n_cells);
        lv.group_list = ws.get<ListRef>(k + 8, n_groups);
        if (!lv.coords || !lv.type || !lv.rec || !lv.child_group || !lv.cell_tape ||
            !lv.group_parent || !lv.group_tape || !lv.cell_list || !lv.group_list) {
            return false;
        }
        cudaMemsetAsync(lv.rec, 0xff, n_cells * sizeof(int32_t), s);
        return true;
    };
    // Level 0: the root cell.
    if (!alloc_level(0, 1, 0)) return LFB_E_CUDA;
    k_init_root<<<1, 1, 0, s>>>(o);
    if (L == 0) {
        // No interval pass: the root is evaluated as a leaf right away.
        cudaMemsetAsync(o.lv[0].type, CELL_BRANCH, 1, s);
    }

    // Stage timing with CUDA events on the pipeline's stream (only when the
    // caller asks for statistics).
    StageEvents events;
    cudaEvent_t* ev = events.ev;
    if (stats) {
        events.create();
        cudaEventRecord(ev[0], s);
    }
    uint64_t n_launch = 1;   // k_init_root
    uint64_t cells_evaluated = 0;

    // Per-warp global scratch of the interval kernel (see WideArgs).
    const uint64_t n = bt.n;
    const uint64_t nw16 = (n + 15) / 16;
    const uint64_t nw1 = (nw16 + 31) / 32;
    const uint64_t per_warp = 9 * (n + 3) + 6 * n + 8 * nw16 + 4 * nw1;
    const uint64_t max_warps = static_cast<uint64_t>(device_sm_count()) * 32;
    const uint64_t budget_warps = std::max<uint64_t>(8, (768ull << 20) / std::max<uint64_t>(per_warp, 1));
    const uint32_t scratch_warps =
        static_cast<uint32_t>(std::min(max_warps, budget_warps) / 8 * 8);
    float2* wS = ws.get<float2>(K_WIDE_S, scratch_warps * (n + 3));
    uint8_t* wSN = ws.get<uint8_t>(K_WIDE_SN, scratch_warps * (n + 3));
    uint8_t* wP = ws.get<uint8_t>(K_WIDE_P, scratch_warps * n);
    uint8_t* wLive = ws.get<uint8_t>(K_WIDE_LIVE, scratch_warps * n);
    uint32_t* wNew = ws.get<uint32_t>(K_WIDE_NEW, scratch_warps * n);
    uint32_t* wSt2 = ws.get<uint32_t>(K_WIDE_ST2, scratch_warps * nw16);
    uint32_t* wL1 = ws.get<uint32_t>(K_WIDE_L1, scratch_warps * nw1);
    uint32_t* wWl = ws.get<uint32_t>(K_WIDE_WL, scratch_warps * nw16);
    if (!wS || !wSN || !wP || !wLive || !wNew || !wSt2 || !wL1 || !wWl) return LFB_E_CUDA;
    if (L > 0) {
        cudaMemsetAsync(wSt2, 0, scratch_warps * nw16 * 4, s);
        cudaMemsetAsync(wL1, 0, scratch_warps * nw1 * 4, s);
    }
    const size_t wide_smem = sizeof(WideSmem) * 8;
    if (!raise_smem_limit(reinterpret_cast<const void*>(k_interval_wide), wide_smem)) {
        return LFB_E_CUDA;
    }
    // Two list arenas, one per parity of depth: depth d reads the lists of
    // its groups from one and writes its children's lists to the other.
    const int list_key[2] = {K_LIST_A, K_LIST_B};
    for (int k = 0; k < 2; ++k) {
        if (!ws.get<WideEntry>(list_key[k], std::max<uint64_t>(cap_of(list_key[k], sizeof(WideEntry)),
                                                                small ? 64 : 4 * n + 1024))) {
            return LFB_E_CUDA;
        }
    }

    // Deep levels (many cells, short tapes) switch to one warp per sibling
    // group over register tapes; every level below stays in that mode.
    const uint32_t group_warps = static_cast<uint32_t>(device_sm_count()) * 32;
    const uint32_t gdec_cap = std::max<uint32_t>(bt.n_choices, 1);
    uint8_t* gdec = ws.get<uint8_t>(K_GDEC, static_cast<size_t>(group_warps) * 8 * gdec_cap);
    uint8_t* glast = ws.get<uint8_t>(K_GLAST, static_cast<size_t>(group_warps) * 8 * kRenumberMax);
    // per depth: the largest register count of its group tapes
    uint32_t* level_nregs = ws.get<uint32_t>(K_NREGS, kMaxLevels + 2);
    if (!gdec || !glast || !level_nregs) return LFB_E_CUDA;
    cudaMemsetAsync(level_nregs, 0, (kMaxLevels + 2) * sizeof(uint32_t), s);
    bool group_mode = false;

    for (int d = 0; d < L; ++d) {
        if (cancelled()) return LFB_E_CANCELLED;
        LevelView& lv = o.lv[d];
        cells_evaluated += lv.n_cells;
        const auto t_level = std::chrono::steady_clock::now();
        unsigned long long arena_before = 0;
        uint32_t nregs_d = bt.n_regs;
        cudaMemcpyAsync(&arena_before, arena_top, sizeof(arena_before), cudaMemcpyDeviceToHost, s);
        if (d > 0) {
            cudaMemcpyAsync(&nregs_d, level_nregs + d, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        }
        if (!cuda_ok(cudaStreamSynchronize(s), "interval stage")) return LFB_E_CUDA;
        // The group-mode register file holds this depth's largest tape (the
        // pruned tapes of deep levels need far fewer registers than the
        // unpruned tape, so more warps fit on an SM).
        nregs_d = std::min<uint32_t>(std::max<uint32_t>(nregs_d, 3), bt.n_regs);
        const size_t group_smem = group_smem_per_warp(nregs_d) * 4;
        group_mode = group_mode || (d > 0 && lv.n_cells >= group_mode_cells() &&
                                    group_smem <= 200 * 1024);
        if (group_mode && group_smem > 48 * 1024 &&
            !raise_smem_limit(reinterpret_cast<const void*>(k_interval_group), group_smem)) {
            return LFB_E_CUDA;
        }
        const bool write_lists = d + 1 < L && !group_mode;
        const int out_key = list_key[(d + 1) & 1];
        for (int attempt = 0; attempt < 4; ++attempt) {
            WideArgs W;
            W.o = o;
            W.bt = bt;
            W.n = bt.n;
            W.in_lists = d == 0 ? g.d_wide : ws.bufs[list_key[d & 1]].as<WideEntry>();
            W.root_list = {0u, bt.n, g.wide_root, 0u};
            W.out_lists = ws.bufs[out_key].as<WideEntry>();
            W.out_top = list_top;
            W.out_cap = cap_of(out_key, sizeof(WideEntry));
            W.write_lists = write_lists ? 1 : 0;
            W.arena = arena;
            W.arena_top = arena_top;
            W.arena_cap = arena_cap;
            W.S = wS;
            W.SN = wSN;
            W.pst = wP;
            W.live = wLive;
            W.newpos = wNew;
            W.st2 = wSt2;
            W.l1 = wL1;
            W.wl = wWl;
            W.status = status;
            W.next_cell = reinterpret_cast<uint32_t*>(counters + 6);
            cudaMemsetAsync(W.next_cell, 0, sizeof(uint32_t), s);
            cudaMemsetAsync(list_top, 0, sizeof(unsigned long long), s);
            if (group_mode) {
                GroupArgs G{o, bt, arena, arena_top, arena_cap, gdec, gdec_cap, glast,
                            nregs_d, status, W.next_cell};
                const uint32_t blocks = std::min<uint32_t>(group_warps / 4, (lv.n_groups + 3) / 4);
                k_interval_group<<<std::max<uint32_t>(blocks, 1), 128, group_smem, s>>>(G, d);
            } else if (lv.n_cells <= block_mode_cells()) {
                const uint32_t blocks = std::min<uint32_t>(
                    std::min<uint32_t>(scratch_warps, device_sm_count() * 2), lv.n_cells);
                k_interval_block<<<std::max<uint32_t>(blocks, 1), kBlockThreads, 0, s>>>(W, d);
            } else {
                const uint32_t warps = std::min<uint32_t>(scratch_warps, (lv.n_cells + 7) / 8 * 8);
                k_interval_wide<<<warps / 8, 256, wide_smem, s>>>(W, d);
            }
            ++n_launch;
            if (!cuda_ok(cudaGetLastError(), "interval kernel")) return LFB_E_CUDA;
            uint32_t st = 0;
            unsigned long long tops[2] = {0, 0};
            cudaMemcpyAsync(&st, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
            cudaMemcpyAsync(&tops[0], arena_top, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
            cudaMemcpyAsync(&tops[1], list_top, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
            if (!cuda_ok(cudaStreamSynchronize(s), "interval kernel")) return LFB_E_CUDA;
            if (st & ST_REGS) {
                return set_error(LFB_E_UNSUPPORTED, "tape register renumbering failed");
            }
            if (!(st & (ST_ARENA_OVERFLOW | ST_LIST_OVERFLOW))) break;
            if (attempt == 3) return set_error(LFB_E_CAPACITY, "tape arena overflow");
            // The counters kept counting past the capacity: grow to what this
            // depth needs and run it again.
            if (st & ST_LIST_OVERFLOW) {
                // The output arena holds nothing yet: no copy needed.
                if (!ws.get<WideEntry>(out_key, tops[1] + tops[1] / 4 + 1024)) return LFB_E_CUDA;
            }
            if (st & ST_ARENA_OVERFLOW) {
                // The arena keeps its contents (the tapes of the levels
                // above): a larger buffer in the same stream order, the
                // used part copied over, the old one freed after the copy.
                const uint64_t new_cap = tops[0] + tops[0] / 4 + (1u << 20);
                DevBuf& b = ws.bufs[K_ARENA];
                RegClause* bigger = nullptr;
                const cudaError_t e =
                    b.ordered ? cudaMallocAsync(reinterpret_cast<void**>(&bigger),
                                                new_cap * sizeof(RegClause), b.stream)
                              : cudaMalloc(&bigger, new_cap * sizeof(RegClause));
                if (e == cudaErrorMemoryAllocation) note_device_oom();
                if (!cuda_ok(e, "arena grow")) return LFB_E_CUDA;
                cudaMemcpyAsync(bigger, arena, arena_before * sizeof(RegClause),
                                cudaMemcpyDeviceToDevice, s);
                if (b.ordered) {
                    cudaFreeAsync(b.ptr, b.stream);
                } else {
                    cudaStreamSynchronize(s);
                    cudaFree(b.ptr);
                }
                b.ptr = bigger;
                b.bytes = new_cap * sizeof(RegClause);
                arena = bigger;
                arena_cap = new_cap;
            }
            cudaMemcpyAsync(arena_top, &arena_before, sizeof(arena_before), cudaMemcpyHostToDevice, s);
            cudaMemsetAsync(status, 0, sizeof(uint32_t), s);
        }

        if (debug_levels()) {
            unsigned long long top_now = 0, lt = 0;
            cudaMemcpyAsync(&top_now, arena_top, sizeof(top_now), cudaMemcpyDeviceToHost, s);
            cudaMemcpyAsync(&lt, list_top, sizeof(lt), cudaMemcpyDeviceToHost, s);
            cudaStreamSynchronize(s);
            const double ms = std::chrono::duration<double, std::milli>(
                std::chrono::steady_clock::now() - t_level).count();
            std::fprintf(stderr, "[lfb] depth %d: %u cells, arena %llu clauses, lists %llu, %.3f ms\n",
                         d, lv.n_cells, top_now, lt, ms);
        }
        // Compact the branch cells into the groups of depth d + 1.
        uint32_t* flags = ws.get<uint32_t>(K_FLAGS, lv.n_cells + 1);
        uint32_t* scan = ws.get<uint32_t>(K_SCAN, lv.n_cells + 1);
        if (!flags || !scan) return LFB_E_CUDA;
        k_branch_flags<<<(lv.n_cells + 255) / 256, 256, 0, s>>>(lv.type, lv.n_cells, flags);
        cudaMemsetAsync(flags + lv.n_cells, 0, sizeof(uint32_t), s);
        if (!exclusive_scan(ws, flags, scan, lv.n_cells + 1, s)) return LFB_E_CUDA;
        uint32_t n_groups = 0;
        cudaMemcpyAsync(&n_groups, scan + lv.n_cells, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if (!cuda_ok(cudaStreamSynchronize(s), "scan")) return LFB_E_CUDA;
        if (static_cast<uint64_t>(n_groups) * 8 >= (1u << 27)) {
            return set_error(LFB_E_CAPACITY, "more than 2^27 cells on one octree level");
        }
        if (!alloc_level(d + 1, n_groups * 8, n_groups)) return LFB_E_CUDA;
        k_build_groups<<<(lv.n_cells + 255) / 256, 256, 0, s>>>(o, d, scan, level_nregs + d + 1);
        n_launch += 2;   // k_branch_flags + k_build_groups
        if (n_groups == 0) {
            // Nothing ambiguous below this depth: no leaves, no faces.
            o.levels = L;
            for (int dd = d + 1; dd <= L; ++dd) {
                if (!alloc_level(dd, 0, 0)) return LFB_E_CUDA;
            }
            break;
        }
    }

    if (cancelled()) return LFB_E_CANCELLED;
    if (stats) cudaEventRecord(ev[1], s);
    // Leaves.
    const uint32_t n_leaf_groups = (L == 0) ? 1 : o.lv[L].n_groups;
    const size_t rec_cap = static_cast<size_t>(n_leaf_groups) * 8 + cells_evaluated + 16;
    LeafRec* recs = ws.get<LeafRec>(K_RECS, rec_cap);
    if (!recs) return LFB_E_CUDA;
    if (n_leaf_groups) {
        // Shared memory per warp: the small lattice state and a register
        // file of smem_regs x 4 x 32 floats; groups whose tape needs more
        // registers use global memory instead.
        const int wpb = 8;
        const uint32_t smem_regs = std::min<uint32_t>(bt.n_regs, kLeafSmemRegs);
        if (debug_levels() && L > 0) {
            std::vector<TapeRef> gt(n_leaf_groups);
            cudaMemcpyAsync(gt.data(), o.lv[L].group_tape, n_leaf_groups * sizeof(TapeRef),
                            cudaMemcpyDeviceToHost, s);
            cudaStreamSynchronize(s);
            std::map<uint32_t, uint64_t> hist, lhist;
            uint64_t len_sum = 0;
            for (const TapeRef& t : gt) {
                ++hist[t.nregs];
                len_sum += t.len;
                uint32_t b = 0;
                while ((1u << (b + 1)) <= t.len) ++b;
                lhist[b] += t.len;
            }
            std::fprintf(stderr, "[lfb] leaf tape clauses by log2(length):");
            for (const auto& h : lhist) {
                std::fprintf(stderr, " %u:%llu", h.first, static_cast<unsigned long long>(h.second));
            }
            std::fprintf(stderr, "\n");
            std::fprintf(stderr, "[lfb] leaf groups %u, mean tape %.1f, registers:",
                         n_leaf_groups, static_cast<double>(len_sum) / std::max<uint32_t>(n_leaf_groups, 1));
            for (const auto& h : hist) {
                std::fprintf(stderr, " %u:%llu", h.first, static_cast<unsigned long long>(h.second));
            }
            std::fprintf(stderr, "\n");
        }
        const size_t per_warp = kLeafSmallBytes + static_cast<size_t>(smem_regs) * 128 * 4 +
                                kLeafOps * sizeof(LeafOp);
        const size_t smem = per_warp * wpb;
        if (smem > 220 * 1024) {
            return set_error(LFB_E_UNSUPPORTED, "tape register file too large for the leaf kernel");
        }
        if (!raise_smem_limit(reinterpret_cast<const void*>(k_leaf_groups), smem)) {
            return LFB_E_CUDA;
        }
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_leaf_groups, 32 * wpb, smem);
        per_sm = std::max(per_sm, 1);
        const uint32_t want = (n_leaf_groups + wpb - 1) / wpb;
        const uint32_t grid = std::min<uint32_t>(want, static_cast<uint32_t>(device_sm_count() * per_sm));
        LeafWarpScratch* scratch = ws.get<LeafWarpScratch>(K_FEAT, static_cast<size_t>(grid) * wpb);
        if (!scratch) return LFB_E_CUDA;
        float* rd = ws.get<float>(K_LEAF_RD, static_cast<size_t>(grid) * wpb * bt.n_regs * 128);
        if (!rd) return LFB_E_CUDA;
        uint32_t* next_group = reinterpret_cast<uint32_t*>(counters + 7);
        cudaMemsetAsync(next_group, 0, sizeof(uint32_t), s);
        // Longest tapes first.
        const uint32_t* order = nullptr;
        if (L > 0 && n_leaf_groups > 1) {
            uint32_t* k0 = ws.get<uint32_t>(K_ORDER_K0, n_leaf_groups);
            uint32_t* k1 = ws.get<uint32_t>(K_ORDER_K1, n_leaf_groups);
            uint32_t* v0 = ws.get<uint32_t>(K_ORDER_V0, n_leaf_groups);
            uint32_t* v1 = ws.get<uint32_t>(K_ORDER_V1, n_leaf_groups);
            if (!k0 || !k1 || !v0 || !v1) return LFB_E_CUDA;
            k_leaf_order_keys<<<(n_leaf_groups + 255) / 256, 256, 0, s>>>(
                o.lv[L].group_tape, n_leaf_groups, k0, v0);
            ++n_launch;
            size_t tmp = 0;
            cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, k0, k1, v0, v1,
                                                      static_cast<int>(n_leaf_groups), 0, 32, s);
            void* t = ws.get<unsigned char>(K_SORTTMP, tmp);
            if (!t || !cuda_ok(cub::DeviceRadixSort::SortPairsDescending(
                                   t, tmp, k0, k1, v0, v1, static_cast<int>(n_leaf_groups), 0,
                                   32, s), "leaf order")) {
                return LFB_E_CUDA;
            }
            order = v1;
        }
        unsigned long long* prof = nullptr;
        if (debug_levels()) prof = ws.get<unsigned long long>(K_PROF, 8ull * n_leaf_groups);
        float* featws = ws.get<float>(K_FEATWS, static_cast<size_t>(grid) * wpb * bt.n_regs *
                                                    kRegBlock);
        if (!featws) return LFB_E_CUDA;
        const uint64_t edge_cap64 = static_cast<uint64_t>(n_leaf_groups) * ws.edges_per_group +
                                    (small ? 0 : 1024);
        const uint32_t edge_cap = static_cast<uint32_t>(std::min<uint64_t>(edge_cap64, 1u << 31));
        EdgeRec* edges = ws.get<EdgeRec>(K_EDGES, edge_cap);
        GroupEdges* gedges = ws.get<GroupEdges>(K_GEDGES, n_leaf_groups);
        uint32_t* rec_group = ws.get<uint32_t>(K_RECGROUP, rec_cap);
        if (!edges || !gedges || !rec_group) return LFB_E_CUDA;
        cudaMemsetAsync(rec_group, 0xff, rec_cap * sizeof(uint32_t), s);
        LeafArgs A{o, bt, arena, recs, rec_top, static_cast<uint32_t>(rec_cap), status,
                   evals, scratch, rd, smem_regs, next_group, order, prof, featws,
                   edges, edge_top, edge_cap, gedges, rec_group,
                   reinterpret_cast<uint32_t*>(counters + 9)};
        k_leaf_groups<<<grid, 32 * wpb, smem, s>>>(A, n_leaf_groups);
        if (!cuda_ok(cudaGetLastError(), "leaf kernel")) return LFB_E_CUDA;
        if (!raise_smem_limit(reinterpret_cast<const void*>(k_leaf_qef), smem)) {
            return LFB_E_CUDA;
        }
        k_leaf_qef<<<grid, 32 * wpb, smem, s>>>(A, n_leaf_groups);
        ++n_launch;
        if (!cuda_ok(cudaGetLastError(), "leaf QEF kernel")) return LFB_E_CUDA;
        // Edge ranks, then the records' vertices: one thread per edge / record.
        const uint32_t sms = static_cast<uint32_t>(device_sm_count());
        k_edge_rank<<<std::min<uint32_t>(sms * 16, (edge_cap + 127) / 128), 128, 0, s>>>(
            edges, edge_top, edge_cap);
        k_leaf_vertices<<<std::min<uint32_t>(sms * 16, static_cast<uint32_t>((rec_cap + 127) / 128)),
                          128, 0, s>>>(recs, rec_top, static_cast<uint32_t>(rec_cap), rec_group,
                                       gedges, n_leaf_groups, edges, edge_cap, L == 0 ? 1 : 0);
        n_launch += 2;
        if (!cuda_ok(cudaGetLastError(), "leaf vertex kernels")) return LFB_E_CUDA;
        if (prof) {
            std::vector<unsigned long long> pf(8ull * n_leaf_groups);
            std::vector<TapeRef> gt(n_leaf_groups);
            cudaMemcpyAsync(pf.data(), prof, pf.size() * 8, cudaMemcpyDeviceToHost, s);
            if (L > 0) {
                cudaMemcpyAsync(gt.data(), o.lv[L].group_tape, n_leaf_groups * sizeof(TapeRef),
                                cudaMemcpyDeviceToHost, s);
            }
            cudaStreamSynchronize(s);
            std::vector<uint32_t> idx(n_leaf_groups);
            for (uint32_t k = 0; k < n_leaf_groups; ++k) idx[k] = k;
            std::sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return pf[8 * a] > pf[8 * b]; });
            unsigned long long sec[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (uint32_t k = 0; k < n_leaf_groups; ++k) {
                for (int q = 0; q < 8; ++q) sec[q] += pf[8 * k + q];
            }
            {
                std::map<uint32_t, uint64_t> eh;
                for (uint32_t k = 0; k < n_leaf_groups; ++k) ++eh[static_cast<uint32_t>(pf[8 * k + 3])];
                std::fprintf(stderr, "[lfb] crossing edges per group:");
                for (const auto& h : eh) {
                    std::fprintf(stderr, " %u:%llu", h.first, static_cast<unsigned long long>(h.second));
                }
                std::fprintf(stderr, "\n");
            }
            std::fprintf(stderr, "[lfb] leaf cycles total %llu: corners %llu, edge search %llu, "
                         "gradients+QEF %llu, vertices %llu; features %llu in %llu calls\n",
                         sec[0], sec[4], sec[5], sec[6], sec[7], sec[1], sec[2]);
            for (uint32_t k = 0; k < std::min<uint32_t>(12, n_leaf_groups); ++k) {
                const uint32_t gg = idx[k];
                std::fprintf(stderr, "[lfb]   group %u: %llu cycles, features %llu cycles / %llu calls, E %llu, tape %u regs %u\n",
                             gg, pf[8 * gg], pf[8 * gg + 1], pf[8 * gg + 2], pf[8 * gg + 3],
                             L > 0 ? gt[gg].len : bt.n, L > 0 ? gt[gg].nregs : bt.n_regs);
            }
        }
        ++n_launch;
    }
    if (cancelled()) return LFB_E_CANCELLED;
    if (stats) cudaEventRecord(ev[2], s);

    // Bottom-up collapse.
    {
        CollapseArgs C{o, bt, arena, recs, rec_top, static_cast<uint32_t>(rec_cap), status,
                       max_err};
        int block = 128;
        while (block > 32 && static_cast<size_t>(bt.n_regs) * block * 4 > 96 * 1024) block /= 2;
        const size_t smem = static_cast<size_t>(bt.n_regs) * block * 4;
        if (smem > 48 * 1024) {
            if (!raise_smem_limit(reinterpret_cast<const void*>(k_collapse_level), smem)) {
                return LFB_E_CUDA;
            }
        }
        for (int d = L - 1; d >= 0; --d) {
            const uint32_t n = o.lv[d].n_cells;
            if (!n) continue;
            const auto t_c = std::chrono::steady_clock::now();
            k_collapse_level<<<(n + block - 1) / block, block, smem, s>>>(C, d);
            ++n_launch;
            if (debug_levels()) {
                cudaStreamSynchronize(s);
                std::fprintf(stderr, "[lfb] collapse depth %d: %u cells, %.3f ms\n", d, n,
                             std::chrono::duration<double, std::milli>(
                                 std::chrono::steady_clock::now() - t_c).count());
            }
        }
        if (!cuda_ok(cudaGetLastError(), "collapse kernel")) return LFB_E_CUDA;
    }

    if (stats) cudaEventRecord(ev[3], s);
    uint32_t st = 0, n_recs = 0;
    cudaMemcpyAsync(&st, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&n_recs, rec_top, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (!cuda_ok(cudaStreamSynchronize(s), "leaf/collapse")) return LFB_E_CUDA;
    if (st & ST_RECORD_OVERFLOW) return set_error(LFB_E_CAPACITY, "leaf record overflow");
    if (st & ST_EDGE_OVERFLOW) {
        // more crossing edges than records were reserved for: grow, and the
        // caller renders the mesh again
        unsigned long long need = 0;
        cudaMemcpyAsync(&need, edge_top, sizeof(need), cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        const uint32_t groups = std::max<uint32_t>(n_leaf_groups, 1);
        ws.edges_per_group = static_cast<uint32_t>(std::min<unsigned long long>(
            54, need / groups + 2));
        ws.retry = true;
        return set_error(LFB_E_CAPACITY, "leaf edge records overflowed");
    }
    if (st & ST_FEATURE_OVERFLOW) {
        std::string why;
        if (st & ST_FEAT_EPS) {
            why += " (more than " + std::to_string(kMaxEps) + " epsilon directions in a feature)";
        }
        if (st & ST_FEAT_LIST) {
            why += " (more than " + std::to_string(kMaxFeat) + " features in a clause)";
        }
        if (st & ST_FEAT_TMP) {
            why += " (more than " + std::to_string(kTmpFeat) + " candidate features in a clause)";
        }
        return set_error(LFB_E_CAPACITY,
                         "feature list overflow at a non-smooth sample point" + why);
    }

    // Dual walk.
    host_free(out.verts);
    host_free(out.tris);
    out.verts = static_cast<libfive_vec3*>(host_alloc(sizeof(libfive_vec3)));
    out.tris = nullptr;
    out.vert_count = 1;
    out.tri_count = 0;
    if (!out.verts) return set_error(LFB_E_CAPACITY, "host allocation failed");
    out.verts[0] = {0.0f, 0.0f, 0.0f};
    uint8_t root_type = 0;
    cudaMemcpyAsync(&root_type, o.lv[0].type, 1, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    const uint32_t n_keys = n_recs * 4;
    bool stl_written = false;
    if (root_type == CELL_BRANCH && n_recs) {
        size_t task_cap = small ? 1024 : std::max<size_t>(1u << 16, static_cast<size_t>(n_recs) * 24);
        size_t tri_cap = small ? 1024 : std::max<size_t>(1u << 16, static_cast<size_t>(n_recs) * 16);
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
                if (cancelled()) return LFB_E_CANCELLED;
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
            if (!exclusive_scan(ws, flags, vscan, n_keys + 1, s)) return LFB_E_CUDA;
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
            if (out.format == MeshFormat::Stl) {
                // records packed on the device, streamed to the file
                out.tri_count = n_tri;
                const int rc = stream_stl(ws, out.stl_path, verts, tris, n_tri, s, n_launch);
                if (rc) return rc;
                stl_written = true;
                break;
            }
            host_free(out.verts);
            out.verts = static_cast<libfive_vec3*>(
                host_alloc((static_cast<size_t>(n_verts) + 1) * sizeof(libfive_vec3)));
            if (!out.verts) return set_error(LFB_E_CAPACITY, "host allocation failed");
            out.vert_count = n_verts + 1;
            out.tri_count = n_tri;
            if (!download(ws, out.verts, verts, out.vert_count * sizeof(libfive_vec3), s)) {
                return LFB_E_CUDA;
            }
            if (out.format == MeshFormat::Coords) {
                int4* c = ws.get<int4>(K_COORDS, std::max<uint32_t>(n_tri, 1));
                host_free(out.coords);
                out.coords = static_cast<int32_t*>(host_alloc(static_cast<size_t>(n_tri) * 16));
                if (!c) return LFB_E_CUDA;
                if (!out.coords && n_tri) return set_error(LFB_E_CAPACITY, "host allocation failed");
                if (n_tri) {
                    k_pack_coords<<<(n_tri + 255) / 256, 256, 0, s>>>(tris, n_tri, c);
                    ++n_launch;
                    if (!download(ws, out.coords, c, static_cast<size_t>(n_tri) * 16, s)) {
                        return LFB_E_CUDA;
                    }
                }
                break;
            }
            out.tris = static_cast<libfive_tri*>(
                host_alloc(static_cast<size_t>(n_tri) * sizeof(libfive_tri)));
            if (!out.tris) return set_error(LFB_E_CAPACITY, "host allocation failed");
            if (!download(ws, out.tris, tris, static_cast<size_t>(n_tri) * sizeof(libfive_tri), s)) {
                return LFB_E_CUDA;
            }
            break;
        }
    }

    if (out.format == MeshFormat::Stl && !stl_written) {
        // no surface: the file holds the header and a zero count
        std::FILE* f = stl_begin(out.stl_path, 0);
        if (!f) return set_error(LFB_E_INVALID, std::string("could not open ") + out.stl_path);
        const bool ok = std::ferror(f) == 0;
        if (std::fclose(f) != 0 || !ok) {
            return set_error(LFB_E_INVALID, std::string("could not write ") + out.stl_path);
        }
    }
    note_launches(n_launch);
    if (stats) {
        cudaEventRecord(ev[4], s);
        cudaEventSynchronize(ev[4]);
        unsigned long long ce[2] = {0, 0};
        cudaMemcpyAsync(ce, evals, sizeof(ce), cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        stats->levels = static_cast<uint32_t>(L);
        stats->cells_evaluated = cells_evaluated;
        stats->leaf_groups = n_leaf_groups;
        stats->leaves_ambiguous = n_recs;
        stats->clause_evals = ce[0];
        stats->clause_evals_grad = ce[1];
        stats->triangles = out.tri_count;
        stats->vertices = out.vert_count - 1;
        stats->kernel_launches = n_launch;
        float ms[4];
        for (int k = 0; k < 4; ++k) cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]);
        stats->ms_interval = ms[0];
        stats->ms_leaf = ms[1];
        stats->ms_collapse = ms[2];
        stats->ms_dual = ms[3];
        stats->ms_total = std::chrono::duration<double, std::milli>(
                              std::chrono::steady_clock::now() - t_start).count();
    }
    return 0;
}

}  // namespace

/// One mesh in the context `ws`, rendered again (up to twice) when an
/// attempt reports that a capacity estimate was too small.
int render_in(Workspace& ws, GpuTape& g, const libfive_region3& R, double min_feature,
              double max_err, MeshOut& out, lfb_mesh_stats* stats,
              const volatile int32_t* cancel)
{
    int rc = 0;
    for (int attempt = 0; attempt < 3; ++attempt) {
        ws.retry = false;
        rc = render_once(ws, g, R, min_feature, max_err, out, stats, cancel, attempt == 0);
        if (rc == 0 || !ws.retry) break;
        clear_error();
    }
    return rc;
}

int render_dc_mesh(GpuTape& g, const libfive_region3& R, double min_feature,
                   double max_err, MeshOut& out, lfb_mesh_stats* stats,
                   const volatile int32_t* cancel)
{
    if (!require_device()) return LFB_E_CUDA;
    keep_pool_memory(kPoolKeepBytes);
    Workspace& ws = default_workspace();
    std::lock_guard<std::mutex> lock(ws.mu);
    take_device_oom();
    int rc = render_in(ws, g, R, min_feature, max_err, out, stats, cancel);
    if (rc == LFB_E_CUDA && take_device_oom()) {
        // The device ran out of memory: idle batch contexts give their
        // scratch back, this context starts from empty buffers, and the
        // mesh is rendered once more.
        cudaStreamSynchronize(ws.s);
        cudaGetLastError();
        {
            auto& sp = stream_pool();
            std::lock_guard<std::mutex> plock(sp.mu);
            for (Workspace* w : sp.pool) {
                std::unique_lock<std::mutex> wl(w->mu, std::try_to_lock);
                if (wl.owns_lock()) w->bufs.clear();
            }
        }
        ws.bufs.clear();
        clear_error();
        rc = render_in(ws, g, R, min_feature, max_err, out, stats, cancel);
    }
    return rc;
}

int render_dc_meshes(MeshJob* jobs, size_t n, unsigned workers)
{
    if (!require_device()) return LFB_E_CUDA;
    keep_pool_memory(kPoolKeepBytes);
    if (n == 0) return 0;
    for (size_t i = 0; i < n; ++i) {
        if (!jobs[i].g) return set_error(LFB_E_INVALID, "null tape in a mesh batch");
    }
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "device")) return LFB_E_CUDA;

    // Longest first, so that the last meshes to start are short ones.
    std::vector<double> cost(n);
    for (size_t i = 0; i < n; ++i) {
        const MeshJob& j = jobs[i];
        const double lo[3] = {j.R.X.lower, j.R.Y.lower, j.R.Z.lower};
        const double hi[3] = {j.R.X.upper, j.R.Y.upper, j.R.Z.upper};
        const int L = std::min(level_from_resolution(lo, hi, j.min_feature), 30);
        cost[i] = static_cast<double>(j.g->reg.clauses.size() + 1) * std::ldexp(1.0, 2 * L);
    }
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t a, size_t b) { return cost[a] > cost[b]; });

    workers = std::max(1u, std::min<unsigned>(workers, static_cast<unsigned>(
                                                           std::min<size_t>(n, 16))));
    // Large meshes (tape length x 4^depth above kBigCost) fill the GPU on
    // their own and need the most scratch memory: worker 0 renders them one
    // after another while the other workers render the small ones side by
    // side; worker 0 joins them when the large ones are done.
    constexpr double kBigCost = 2e9;
    std::vector<size_t> big, small;
    for (size_t i : order) (cost[i] >= kBigCost && workers > 1 ? big : small).push_back(i);
    std::atomic<size_t> next_big{0}, next_small{0};
    auto run_queue = [&](Workspace* ws, const std::vector<size_t>& q, std::atomic<size_t>& next) {
        for (;;) {
            const size_t i = next.fetch_add(1);
            if (i >= q.size()) break;
            MeshJob& j = jobs[q[i]];
            clear_error();
            j.rc = render_in(*ws, *j.g, j.R, j.min_feature, j.max_err, j.out,
                             j.want_stats ? &j.stats : nullptr, j.cancel);
            if (j.rc != 0) last_error(&j.err);
        }
    };
    auto work = [&](unsigned k) {
        cudaSetDevice(dev);
        Workspace* ws = stream_workspace(k);
        if (!ws) return;
        std::lock_guard<std::mutex> lock(ws->mu);
        if (k == 0) run_queue(ws, big, next_big);
        run_queue(ws, small, next_small);
    };
    std::vector<std::thread> pool;
    for (unsigned k = 1; k < workers; ++k) pool.emplace_back(work, k);
    work(0);
    for (auto& t : pool) t.join();

    // A mesh that ran out of device memory while others were in flight is
    // rendered again alone, after the other contexts (and the single-call
    // context, when idle) have given their buffers back.
    std::vector<size_t> retry;
    for (size_t i = 0; i < n; ++i) {
        if (jobs[i].rc == LFB_E_CUDA && jobs[i].err.find("out of memory") != std::string::npos) {
            retry.push_back(i);
        }
    }
    if (!retry.empty()) {
        cudaDeviceSynchronize();
        cudaGetLastError();
        for (unsigned k = 1; k < workers; ++k) {
            Workspace* w = stream_workspace(k);
            std::lock_guard<std::mutex> lock(w->mu);
            w->bufs.clear();
        }
        {
            Workspace& d = default_workspace();
            std::unique_lock<std::mutex> lock(d.mu, std::try_to_lock);
            if (lock.owns_lock()) d.bufs.clear();
        }
        Workspace* w = stream_workspace(0);
        std::lock_guard<std::mutex> lock(w->mu);
        for (size_t i : retry) {
            MeshJob& j = jobs[i];
            clear_error();
            j.err.clear();
            j.rc = render_in(*w, *j.g, j.R, j.min_feature, j.max_err, j.out,
                             j.want_stats ? &j.stats : nullptr, j.cancel);
            if (j.rc != 0) last_error(&j.err);
        }
    }

    clear_error();
    for (size_t i = 0; i < n; ++i) {
        const MeshJob& j = jobs[i];
        if (j.rc == 1) return set_error(LFB_E_CUDA, "no stream context for a mesh batch");
        if (j.rc != 0) return set_error(j.rc, j.err);
    }
    return 0;
}

}  // namespace lfb
