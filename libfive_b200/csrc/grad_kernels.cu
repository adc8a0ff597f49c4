// Gradients with respect to free variables and point coordinates.
//
//  * k_jacobian: JacobianEvaluator::gradient (eval_jacobian.cpp:49-115) in
//    its own forward mode.  One thread per (point, three variables): X, Y, Z
//    carry zero tangents, variable k0 + c carries a unit tangent in slot c,
//    and CONST_VAR clears tangents (clear_vars).  Each output is the same
//    sequence of float operations as the reference's per-variable column.
//  * k_grad_forward / k_grad_backward: reverse mode (the reference has none).
//    The forward pass stores the clauses' local partials (the forward
//    derivative rules of DerivArrayEvaluator, eval_deriv_array.cpp:119-256,
//    applied to unit tangents, so min / max / abs pick the same branch),
//    except those fixed by the opcode (partial_kind); the
//    backward pass walks the register tape from the end, one adjoint per
//    register, and sends variable adjoints to a warp-reduced atomic sum.
#include <cfloat>
#include <mutex>
#include <vector>

#include "eval_api.hpp"
#include "eval_kernels.cuh"
#include "jit.hpp"
#include "libfive_b200.h"

namespace lfb {

namespace {

__device__ __forceinline__ D4 jac_fetch(uint8_t kind, uint16_t idx, const float* R,
                                        int tid, int B, const float* __restrict__ cp,
                                        uint32_t n_const, uint32_t k0)
{
    if (kind == OPND_REG) {
        const float* r = R + idx * 4 * B + tid;
        return {r[0], r[B], r[2 * B], r[3 * B]};
    }
    const float v = __ldg(cp + idx);
    if (kind == OPND_VAR) {
        const uint32_t k = idx - n_const;
        return {v, k == k0 ? 1.0f : 0.0f, k == k0 + 1 ? 1.0f : 0.0f, k == k0 + 2 ? 1.0f : 0.0f};
    }
    return {v, 0.0f, 0.0f, 0.0f};
}

__global__ void __launch_bounds__(128)
k_jacobian(DevTape t, uint32_t n, uint32_t n_vars, const float* __restrict__ X,
           const float* __restrict__ Y, const float* __restrict__ Z, float* __restrict__ out)
{
    extern __shared__ float smem[];
    const int B = blockDim.x;
    const int tid = threadIdx.x;
    const uint32_t ntrip = (n_vars + 2) / 3;
    const uint64_t items = static_cast<uint64_t>(n) * ntrip;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * B;
    float* R = smem;
    for (uint64_t it = static_cast<uint64_t>(blockIdx.x) * B + tid; it - tid < items;
         it += stride) {
        const bool ok = it < items;
        const uint32_t i = ok ? static_cast<uint32_t>(it / ntrip) : 0u;
        const uint32_t k0 = ok ? static_cast<uint32_t>(it % ntrip) * 3 : 0u;
        const float p[3] = {ok ? X[i] : 0.0f, ok ? Y[i] : 0.0f, ok ? Z[i] : 0.0f};
        for (int a = 0; a < 3; ++a) {
            float* r = R + a * 4 * B + tid;
            r[0] = p[a];
            r[B] = 0.0f;
            r[2 * B] = 0.0f;
            r[3 * B] = 0.0f;
        }
        for (uint32_t c = 0; c < t.n; ++c) {
            const uint2 raw = __ldg(reinterpret_cast<const uint2*>(t.clauses + c));
            const uint8_t o = raw.x & 0xff;
            const uint8_t kinds = (raw.x >> 8) & 0xff;
            const D4 a = jac_fetch(kinds & 3, raw.y & 0xffff, R, tid, B, t.cpool, t.n_const, k0);
            const D4 b = jac_fetch((kinds >> 2) & 3, raw.y >> 16, R, tid, B, t.cpool, t.n_const, k0);
            const D4 d = dv_deriv(o, a, b, true);
            float* r = R + (raw.x >> 16) * 4 * B + tid;
            r[0] = d.v; r[B] = d.dx; r[2 * B] = d.dy; r[3 * B] = d.dz;
        }
        if (ok) {
            const D4 d = jac_fetch(t.root_kind, t.root, R, tid, B, t.cpool, t.n_const, k0);
            float* row = out + static_cast<size_t>(i) * n_vars;
            row[k0] = d.dx;
            if (k0 + 1 < n_vars) row[k0 + 1] = d.dy;
            if (k0 + 2 < n_vars) row[k0 + 2] = d.dz;
        }
    }
}

/// How a clause's local partials (d out / d a, d out / d b for unit
/// tangents) reach the backward pass: PK_CONST ones are fixed by the opcode
/// (ADD, SUB, NEG, CONST_VAR, COPY: exactly 1 or -1), PK_CHOICE (MIN, MAX)
/// store d out / d a (0 or 1; the other is its complement), PK_ONE (other
/// unary ops) store d out / d a, PK_TWO (other binary ops) store both.
/// Slots are numbered per tape; a point's partials take n_pslot floats.
enum : uint32_t { PK_CONST = 0, PK_CHOICE = 1, PK_ONE = 2, PK_TWO = 3 };

uint32_t partial_kind(uint8_t o)
{
    switch (o) {
        case op::ADD: case op::SUB: case op::NEG: case op::CONST_VAR: case OP_COPY:
            return PK_CONST;
        case op::MIN: case op::MAX:
            return PK_CHOICE;
        default:
            return op::arity(o) == 2 ? PK_TWO : PK_ONE;
    }
}

__device__ __forceinline__ float2 const_partials(uint8_t o)
{
    switch (o) {
        case op::ADD: return make_float2(1.0f, 1.0f);
        case op::SUB: return make_float2(1.0f, -1.0f);
        case op::NEG: return make_float2(-1.0f, 0.0f);
        default: return make_float2(1.0f, 0.0f);   // CONST_VAR, COPY
    }
}

__device__ __forceinline__ float gv_fetch(uint8_t kind, uint16_t idx, const float* R, int tid,
                                          int B, const float* __restrict__ cp)
{
    return kind == OPND_REG ? R[idx * B + tid] : __ldg(cp + idx);
}

/// Value and local partials (d out / d a, d out / d b) of one clause: the
/// results of dv_deriv for unit tangents (a = (1, 0), b = (0, 1)), bit for
/// bit, computed directly for the common opcodes (one transcendental call
/// instead of two for EXP, one division instead of three for LOG / SQRT /
/// RECIP / DIV) and through dv_deriv_all for the rest.
__device__ __forceinline__ void dv_partials(uint8_t o, float av, float bv, float* v, float* pa,
                                            float* pb)
{
    switch (o) {
        case op::ADD: *v = __fadd_rn(av, bv); *pa = 1.0f; *pb = 1.0f; return;
        case op::SUB: *v = __fsub_rn(av, bv); *pa = 1.0f; *pb = -1.0f; return;
        case op::MUL:
            *v = __fmul_rn(av, bv);
            *pa = __fadd_rn(__fmul_rn(0.0f, av), __fmul_rn(1.0f, bv));
            *pb = __fadd_rn(__fmul_rn(1.0f, av), __fmul_rn(0.0f, bv));
            return;
        case op::MIN:
            *v = sc_min(av, bv);
            *pa = av < bv ? 1.0f : 0.0f;
            *pb = av < bv ? 0.0f : 1.0f;
            return;
        case op::MAX:
            *v = sc_max(av, bv);
            *pa = av < bv ? 0.0f : 1.0f;
            *pb = av < bv ? 1.0f : 0.0f;
            return;
        case op::SQUARE: *v = __fmul_rn(av, av); *pa = __fmul_rn(av, 2.0f); *pb = 0.0f; return;
        case op::NEG: *v = -av; *pa = -1.0f; *pb = 0.0f; return;
        case op::ABS: *v = fabsf(av); *pa = av > 0 ? 1.0f : -1.0f; *pb = 0.0f; return;
        case op::SQRT: {
            const float ov = __fsqrt_rn(av);
            *v = ov;
            *pa = av < 0 ? 0.0f : __fdiv_rn(1.0f, __fmul_rn(2.0f, ov));
            *pb = 0.0f;
            return;
        }
        case op::LOG: *v = logf(av); *pa = __fdiv_rn(1.0f, av); *pb = 0.0f; return;
        case op::EXP: {
            const float e = expf(av);
            *v = e;
            *pa = __fmul_rn(1.0f, e);
            *pb = 0.0f;
            return;
        }
        case op::RECIP:
            *v = __fdiv_rn(1.0f, av);
            *pa = __fdiv_rn(1.0f, -__fmul_rn(av, av));
            *pb = 0.0f;
            return;
        case op::DIV: {
            const float den = __fmul_rn(bv, bv);
            *v = __fdiv_rn(av, bv);
            *pa = __fdiv_rn(__fsub_rn(__fmul_rn(1.0f, bv), __fmul_rn(0.0f, av)), den);
            *pb = __fdiv_rn(__fsub_rn(__fmul_rn(0.0f, bv), __fmul_rn(1.0f, av)), den);
            return;
        }
        default: {
            const D4 d = dv_deriv_all(o, D4{av, 1.0f, 0.0f, 0.0f}, D4{bv, 0.0f, 1.0f, 0.0f},
                                      false);
            *v = d.v;
            *pa = d.dx;
            *pb = d.dy;
        }
    }
}

/// Forward pass of the reverse mode, PTS points per thread (points
/// base + k * blockDim.x): value of every clause, and the local partials
/// its kind keeps, at P[slot * m + i] (and slot + 1 for PK_TWO).  Register r
/// of point k lives at R[(r * PTS + k) * blockDim.x + tid].
template <int PTS>
__global__ void __launch_bounds__(128)
k_grad_forward(DevTape t, const uint32_t* __restrict__ pslot, uint32_t m,
               const float* __restrict__ X, const float* __restrict__ Y,
               const float* __restrict__ Z, float* __restrict__ P, float* __restrict__ f)
{
    extern __shared__ float smem[];
    const int B = blockDim.x;
    const int tid = threadIdx.x;
    float* R = smem;
    uint32_t idx[PTS];
    bool ok[PTS];
#pragma unroll
    for (int k = 0; k < PTS; ++k) {
        idx[k] = (blockIdx.x * PTS + k) * B + tid;
        ok[k] = idx[k] < m;
        R[(0 * PTS + k) * B + tid] = ok[k] ? X[idx[k]] : 0.0f;
        R[(1 * PTS + k) * B + tid] = ok[k] ? Y[idx[k]] : 0.0f;
        R[(2 * PTS + k) * B + tid] = ok[k] ? Z[idx[k]] : 0.0f;
    }
    for (uint32_t c = 0; c < t.n; ++c) {
        const uint2 raw = __ldg(reinterpret_cast<const uint2*>(t.clauses + c));
        const uint8_t o = raw.x & 0xff;
        const uint8_t kinds = (raw.x >> 8) & 0xff;
        const uint32_t ra = raw.y & 0xffff, rb = raw.y >> 16, ro = raw.x >> 16;
        const uint32_t ps = __ldg(pslot + c);
        const uint32_t kind = ps >> 28, slot = ps & 0x0fffffffu;
        const bool ra_reg = (kinds & 3) == OPND_REG, rb_reg = ((kinds >> 2) & 3) == OPND_REG;
        const float ca = ra_reg ? 0.0f : __ldg(t.cpool + ra);
        const float cb = rb_reg ? 0.0f : __ldg(t.cpool + rb);
#pragma unroll
        for (int k = 0; k < PTS; ++k) {
            const float av = ra_reg ? R[(ra * PTS + k) * B + tid] : ca;
            const float bv = rb_reg ? R[(rb * PTS + k) * B + tid] : cb;
            float v, pa, pb;
            dv_partials(o, av, bv, &v, &pa, &pb);
            R[(ro * PTS + k) * B + tid] = v;
            if (ok[k] && kind != PK_CONST) {
                P[static_cast<size_t>(slot) * m + idx[k]] = pa;
                if (kind == PK_TWO) P[static_cast<size_t>(slot + 1) * m + idx[k]] = pb;
            }
        }
    }
    if (f) {
#pragma unroll
        for (int k = 0; k < PTS; ++k) {
            if (ok[k]) {
                f[idx[k]] = t.root_kind == OPND_REG ? R[(t.root * PTS + k) * B + tid]
                                                    : __ldg(t.cpool + t.root);
            }
        }
    }
}

__device__ __forceinline__ float warp_sum(float v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

/// Backward pass: adjoints per register from the root (seeded with s_i) to
/// the start; X, Y, Z adjoints are registers 0-2 at the end.  With
/// block_const_var, CONST_VAR stops the adjoint (variable gradients, as
/// clear_vars does in the forward Jacobian); otherwise it passes through
/// (point gradients, as in DerivArrayEvaluator).  Variable adjoints are
/// summed over the warp, then (SV) over the block in shared memory, and
/// reach gvars with one atomic add per variable and block; without SV
/// (too many variables for shared memory) each warp adds to gvars.
template <bool SV, int PTS>
__global__ void __launch_bounds__(128)
k_grad_backward(DevTape t, const uint32_t* __restrict__ pslot, uint32_t m,
                const float* __restrict__ P,
                const float* __restrict__ seed, float* __restrict__ gx,
                float* __restrict__ gy, float* __restrict__ gz, float* __restrict__ gvars,
                int block_const_var)
{
    extern __shared__ float smem[];
    const int B = blockDim.x;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    uint32_t idx[PTS];
    bool ok[PTS];
#pragma unroll
    for (int k = 0; k < PTS; ++k) {
        idx[k] = (blockIdx.x * PTS + k) * B + tid;
        ok[k] = idx[k] < m;
    }
    // adjoint of register r, point k: A[(r * PTS + k) * B + tid]
    float* A = smem;
    float* Gv = smem + t.n_regs * PTS * B;
    const uint32_t n_vars = t.n_cpool - t.n_const;
    if (SV && gvars) {
        for (uint32_t k = tid; k < n_vars; k += B) Gv[k] = 0.0f;
        __syncthreads();
    }
    auto add_var = [&](uint32_t k, float g) {
        const float w = warp_sum(g);
        if (lane == 0 && w != 0.0f) atomicAdd((SV ? Gv : gvars) + k, w);
    };
    for (uint32_t r = 0; r < t.n_regs * PTS; ++r) A[r * B + tid] = 0.0f;
    float s0[PTS];
#pragma unroll
    for (int k = 0; k < PTS; ++k) s0[k] = ok[k] ? (seed ? seed[idx[k]] : 1.0f) : 0.0f;
    if (t.root_kind == OPND_REG) {
#pragma unroll
        for (int k = 0; k < PTS; ++k) A[(t.root * PTS + k) * B + tid] = s0[k];
    } else if (t.root_kind == OPND_VAR && gvars) {
        float g = 0.0f;
#pragma unroll
        for (int k = 0; k < PTS; ++k) g += s0[k];
        add_var(t.root - t.n_const, g);
    }
    for (int64_t c = static_cast<int64_t>(t.n) - 1; c >= 0; --c) {
        const uint2 raw = __ldg(reinterpret_cast<const uint2*>(t.clauses + c));
        const uint8_t o = raw.x & 0xff;
        const uint8_t kinds = (raw.x >> 8) & 0xff;
        const uint32_t ro = raw.x >> 16, ra = raw.y & 0xffff, rb = raw.y >> 16;
        const uint32_t ps = __ldg(pslot + c);
        const uint32_t kind = ps >> 28, slot = ps & 0x0fffffffu;
        const uint8_t ka = kinds & 3, kb = (kinds >> 2) & 3;
        const bool binary = dev_is_binary(o);
        const bool blocked = block_const_var && o == op::CONST_VAR;
        float va = 0.0f, vb = 0.0f;   // variable adjoints of this clause, summed over points
#pragma unroll
        for (int k = 0; k < PTS; ++k) {
            float* ao = A + (ro * PTS + k) * B + tid;
            const float adj = *ao;
            *ao = 0.0f;
            float2 pd = make_float2(0.0f, 0.0f);
            if (kind == PK_CONST) {
                pd = const_partials(o);
            } else if (ok[k]) {
                const float p0 = P[static_cast<size_t>(slot) * m + idx[k]];
                pd = kind == PK_TWO ? make_float2(p0, P[static_cast<size_t>(slot + 1) * m + idx[k]])
                   : kind == PK_CHOICE ? make_float2(p0, 1.0f - p0)
                                       : make_float2(p0, 0.0f);
            }
            if (blocked) pd = make_float2(0.0f, 0.0f);
            // register adjoints accumulate with one fused multiply-add per
            // operand, as the compiled backward kernels do
            if (ka == OPND_REG) {
                float* aa = A + (ra * PTS + k) * B + tid;
                *aa = __fmaf_rn(adj, pd.x, *aa);
            } else {
                va += adj * pd.x;
            }
            if (binary) {
                if (kb == OPND_REG) {
                    float* ab = A + (rb * PTS + k) * B + tid;
                    *ab = __fmaf_rn(adj, pd.y, *ab);
                } else {
                    vb += adj * pd.y;
                }
            }
        }
        if (gvars) {
            if (ka == OPND_VAR) add_var(ra - t.n_const, va);
            if (binary && kb == OPND_VAR) add_var(rb - t.n_const, vb);
        }
    }
#pragma unroll
    for (int k = 0; k < PTS; ++k) {
        if (ok[k]) {
            if (gx) gx[idx[k]] = A[(0 * PTS + k) * B + tid];
            if (gy) gy[idx[k]] = A[(1 * PTS + k) * B + tid];
            if (gz) gz[idx[k]] = A[(2 * PTS + k) * B + tid];
        }
    }
    if (SV && gvars) {
        __syncthreads();
        for (uint32_t k = tid; k < n_vars; k += B) {
            if (Gv[k] != 0.0f) atomicAdd(gvars + k, Gv[k]);
        }
    }
}

/// The tape's partial-slot table (partial_kind), uploaded on first use.
bool ensure_pslots(GpuTape& g)
{
    std::lock_guard<std::mutex> lock(g.mu);
    if (g.pslot_ready) return true;
    std::vector<uint32_t> ps(std::max<size_t>(g.reg.clauses.size(), 1), 0);
    uint32_t next = 0;
    for (size_t c = 0; c < g.reg.clauses.size(); ++c) {
        const uint32_t kind = partial_kind(g.reg.clauses[c].op);
        ps[c] = next | (kind << 28);
        next += kind == PK_CONST ? 0 : kind == PK_TWO ? 2 : 1;
    }
    if (next >= (1u << 28)) {
        set_error(LFB_E_UNSUPPORTED, "tape too long for the reverse mode");
        return false;
    }
    if (!cuda_ok(cudaMalloc(&g.d_pslot, ps.size() * sizeof(uint32_t)), "partial slots") ||
        !cuda_ok(cudaMemcpy(g.d_pslot, ps.data(), ps.size() * sizeof(uint32_t),
                            cudaMemcpyHostToDevice), "partial slots")) {
        return false;
    }
    g.h_pslot = std::move(ps);
    g.n_pslot = next;
    g.pslot_ready = true;
    return true;
}

bool tape_has_const_var(const GpuTape& g)
{
    for (const RegClause& c : g.reg.clauses) {
        if (c.op == op::CONST_VAR) return true;
    }
    return false;
}

/// Device buffers of a call on host data (grow-only, reused).
struct GradStaging {
    DevBuf in, out, partials;
};

GradStaging& grad_staging()
{
    static GradStaging s;
    return s;
}

constexpr int kBlock = 128;

bool set_smem(const void* fn, size_t bytes)
{
    return raise_smem_limit(fn, bytes);
}

int jacobian_device(GpuTape& g, uint64_t n, const float* x, const float* y, const float* z,
                    float* out, cudaStream_t s)
{
    const DevTape t = g.dev();
    const uint32_t nv = g.reg.n_vars;
    if (nv == 0 || n == 0) return 0;
    const size_t smem = static_cast<size_t>(t.n_regs) * kBlock * 4 * sizeof(float);
    if (smem > 200 * 1024) return set_error(LFB_E_UNSUPPORTED, "tape needs too many registers");
    if (!set_smem(reinterpret_cast<const void*>(k_jacobian), smem)) return LFB_E_CUDA;
    const uint64_t kChunk = uint64_t(1) << 22;   // points per launch
    for (uint64_t off = 0; off < n; off += kChunk) {
        const uint32_t m = static_cast<uint32_t>(std::min(kChunk, n - off));
        const uint64_t items = static_cast<uint64_t>(m) * ((nv + 2) / 3);
        const uint64_t blocks = std::min<uint64_t>((items + kBlock - 1) / kBlock,
                                                   static_cast<uint64_t>(device_sm_count()) * 64);
        k_jacobian<<<static_cast<unsigned>(blocks), kBlock, smem, s>>>(
            t, m, nv, x + off, y + off, z + off, out + off * nv);
        if (!cuda_ok(cudaGetLastError(), "jacobian kernel")) return LFB_E_CUDA;
        note_launches(1);
    }
    return 0;
}

int grad_device(GpuTape& g, uint64_t n, const float* x, const float* y, const float* z,
                const float* seed, float* f, float* gx, float* gy, float* gz, float* gvars,
                cudaStream_t s)
{
    const DevTape t = g.dev();
    if (n == 0) return 0;
    // Two points per thread in both passes: registers / adjoints of both
    // points in shared memory, plus (when they fit) the block's variable
    // adjoints.
    constexpr int kPts = 2;
    const size_t smem = static_cast<size_t>(t.n_regs) * kBlock * kPts * sizeof(float);
    if (smem > 200 * 1024) return set_error(LFB_E_UNSUPPORTED, "tape needs too many registers");
    const size_t smem_sv = smem + static_cast<size_t>(t.n_cpool - t.n_const) * sizeof(float);
    const bool sv = smem_sv <= 200 * 1024;
    if (!set_smem(reinterpret_cast<const void*>(k_grad_forward<kPts>), smem) ||
        !set_smem(reinterpret_cast<const void*>(k_grad_backward<false, kPts>), smem) ||
        (sv && !set_smem(reinterpret_cast<const void*>(k_grad_backward<true, kPts>), smem_sv))) {
        return LFB_E_CUDA;
    }
    // Checkpointed reverse mode when the tape compiles: per point it stores
    // only the registers each tape segment reads from earlier segments, and
    // the backward kernel recomputes the segment from them (jit.cpp).
    if (const uint32_t ckf = jit_ckpt_prepare(g)) {
        const uint64_t per_point = 4ull * ckf;
        const uint64_t cchunk = std::max<uint64_t>(kBlock, std::min<uint64_t>(
            (4ull << 30) / per_point / kBlock * kBlock, uint64_t(1) << 22));
        auto& cst = grad_staging();
        if (!cst.partials.reserve(std::min(cchunk, n) * per_point)) return LFB_E_CUDA;
        float* C = cst.partials.as<float>();
        const bool has_cv = tape_has_const_var(g);
        const bool want_xyz = gx || gy || gz;
        for (uint64_t off = 0; off < n; off += cchunk) {
            const uint32_t m = static_cast<uint32_t>(std::min(cchunk, n - off));
            if (!jit_ckpt_forward(g, m, x + off, y + off, z + off, C, f ? f + off : nullptr, s)) {
                return set_error(LFB_E_CUDA, "checkpointed gradient kernel launch failed");
            }
            const float* sd = seed ? seed + off : nullptr;
            float* ox = gx ? gx + off : nullptr;
            float* oy = gy ? gy + off : nullptr;
            float* oz = gz ? gz + off : nullptr;
            bool ok = true;
            if (!has_cv) {
                if (want_xyz || gvars) {
                    ok = jit_ckpt_backward(g, m, C, sd, ox, oy, oz, gvars, 0, s);
                }
            } else {
                // CONST_VAR passes point gradients but blocks variable ones.
                if (want_xyz) ok = jit_ckpt_backward(g, m, C, sd, ox, oy, oz, nullptr, 0, s);
                if (gvars && ok) {
                    ok = jit_ckpt_backward(g, m, C, sd, nullptr, nullptr, nullptr, gvars, 1, s);
                }
            }
            if (!ok) return set_error(LFB_E_CUDA, "checkpointed gradient kernel launch failed");
            if (!cuda_ok(cudaGetLastError(), "gradient kernels")) return LFB_E_CUDA;
        }
        return 0;
    }
    if (!ensure_pslots(g)) return LFB_E_CUDA;
    const uint32_t* pslot = g.d_pslot;
    // Partials take 4 bytes per slot and point: points per launch so that
    // they stay within 4 GiB (enough points to fill the GPU for tapes of
    // tens of thousands of clauses).
    const uint64_t per_point = std::max<uint64_t>(4ull * g.n_pslot, 4);
    const uint64_t chunk = std::max<uint64_t>(kBlock, std::min<uint64_t>(
        (4ull << 30) / per_point / kBlock * kBlock, uint64_t(1) << 22));
    auto& st = grad_staging();
    if (!st.partials.reserve(std::min(chunk, n) * per_point)) return LFB_E_CUDA;
    float* P = st.partials.as<float>();
    const bool has_cv = tape_has_const_var(g);
    const bool want_xyz = gx || gy || gz;
    auto backward = [&](uint32_t m, unsigned blocks, const float* sd, uint64_t off, bool xyz,
                        float* gv, int block_cv) {
        float* ox = xyz && gx ? gx + off : nullptr;
        float* oy = xyz && gy ? gy + off : nullptr;
        float* oz = xyz && gz ? gz + off : nullptr;
        if (gv && sv) {
            k_grad_backward<true, kPts><<<blocks, kBlock, smem_sv, s>>>(
                t, pslot, m, P, sd, ox, oy, oz, gv, block_cv);
        } else {
            k_grad_backward<false, kPts><<<blocks, kBlock, smem, s>>>(
                t, pslot, m, P, sd, ox, oy, oz, gv, block_cv);
        }
        note_launches(1);
    };
    // The tape's compiled reverse-mode kernels (jit.cpp) when it has them,
    // else the interpreters; both do the same arithmetic.
    const uint32_t* hs = g.h_pslot.data();
    const bool jit = jit_partials(g, hs, 0, x, y, z, P, f, s) &&
                     jit_backward(g, hs, 0, P, seed, gx, gy, gz, gvars, 0, s);
    auto backward_any = [&](uint32_t m, unsigned blocks, const float* sd, uint64_t off, bool xyz,
                            float* gv, int block_cv) {
        if (jit) {
            return jit_backward(g, hs, m, P, sd, xyz && gx ? gx + off : nullptr,
                                xyz && gy ? gy + off : nullptr, xyz && gz ? gz + off : nullptr,
                                gv, block_cv, s);
        }
        backward(m, blocks, sd, off, xyz, gv, block_cv);
        return true;
    };
    for (uint64_t off = 0; off < n; off += chunk) {
        const uint32_t m = static_cast<uint32_t>(std::min(chunk, n - off));
        const unsigned blocks = (m + kBlock * kPts - 1) / (kBlock * kPts);
        if (jit) {
            if (!jit_partials(g, hs, m, x + off, y + off, z + off, P, f ? f + off : nullptr, s)) {
                return set_error(LFB_E_CUDA, "compiled gradient kernel launch failed");
            }
        } else {
            k_grad_forward<kPts><<<blocks, kBlock, smem, s>>>(t, pslot, m, x + off, y + off,
                                                              z + off, P, f ? f + off : nullptr);
            note_launches(1);
        }
        const float* sd = seed ? seed + off : nullptr;
        bool ok = true;
        if (!has_cv) {
            if (want_xyz || gvars) ok = backward_any(m, blocks, sd, off, true, gvars, 0);
        } else {
            // CONST_VAR passes point gradients but blocks variable ones.
            if (want_xyz) ok = backward_any(m, blocks, sd, off, true, nullptr, 0);
            if (gvars && ok) ok = backward_any(m, blocks, sd, off, false, gvars, 1);
        }
        if (!ok) return set_error(LFB_E_CUDA, "compiled gradient kernel launch failed");
        if (!cuda_ok(cudaGetLastError(), "gradient kernels")) return LFB_E_CUDA;
    }
    return 0;
}

}  // namespace

int eval_jacobian(GpuTape& g, uint64_t n, const float* x, const float* y, const float* z,
                  float* out, cudaStream_t s, bool device)
{
    if (!require_device()) return LFB_E_CUDA;
    if (!x || !y || !z || (!out && g.reg.n_vars)) {
        return set_error(LFB_E_INVALID, "lfb_eval_jacobian: null argument");
    }
    std::lock_guard<std::mutex> lock(global_mutex());
    if (device) return jacobian_device(g, n, x, y, z, out, s);
    if (n == 0 || g.reg.n_vars == 0) return 0;
    auto& st = grad_staging();
    const size_t nv = g.reg.n_vars;
    if (!st.in.reserve(n * 3 * sizeof(float)) || !st.out.reserve(n * nv * sizeof(float))) {
        return LFB_E_CUDA;
    }
    float* d = st.in.as<float>();
    const size_t b = n * sizeof(float);
    cudaStream_t s0 = 0;
    if (!cuda_ok(cudaMemcpyAsync(d, x, b, cudaMemcpyHostToDevice, s0), "copy") ||
        !cuda_ok(cudaMemcpyAsync(d + n, y, b, cudaMemcpyHostToDevice, s0), "copy") ||
        !cuda_ok(cudaMemcpyAsync(d + 2 * n, z, b, cudaMemcpyHostToDevice, s0), "copy")) {
        return LFB_E_CUDA;
    }
    const int rc = jacobian_device(g, n, d, d + n, d + 2 * n, st.out.as<float>(), s0);
    if (rc) return rc;
    if (!cuda_ok(cudaMemcpyAsync(out, st.out.ptr, n * nv * sizeof(float),
                                 cudaMemcpyDeviceToHost, s0), "copy")) {
        return LFB_E_CUDA;
    }
    return cuda_ok(cudaStreamSynchronize(s0), "sync") ? 0 : LFB_E_CUDA;
}

bool grad_prepare(GpuTape& g)
{
    // the checkpointed kernels, which grad_device takes when they compile;
    // else the stored-partials kernels (m = 0: compile, no launch)
    if (jit_ckpt_prepare(g)) return true;
    if (!ensure_pslots(g)) return false;
    const uint32_t* hs = g.h_pslot.data();
    jit_partials(g, hs, 0, nullptr, nullptr, nullptr, nullptr, nullptr, 0);
    jit_backward(g, hs, 0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0);
    return true;
}

bool grad_prepared(GpuTape& g)
{
    std::lock_guard<std::mutex> lock(g.mu);
    if (g.jit[5].state == 1 && g.jit[6].state == 1) return true;
    return g.jit[5].state != 0 && g.jit[6].state != 0 && g.pslot_ready &&
           g.jit[2].state != 0 && g.jit[3].state != 0;
}

namespace {

/// sum of f^2 over the points, in FP64 (one atomic per block).
__global__ void __launch_bounds__(256) k_sum_squares(const float* __restrict__ f, uint64_t n,
                                                     double* out)
{
    __shared__ double part[8];
    double acc = 0.0;
    for (uint64_t i = blockIdx.x * 256ull + threadIdx.x; i < n; i += gridDim.x * 256ull) {
        const double v = f[i];
        acc += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < 8; ++w) b += part[w];
        atomicAdd(out, b);
    }
}

__global__ void k_mean_to_float(const double* sum, uint64_t n, float* out)
{
    *out = static_cast<float>(*sum / static_cast<double>(n));
}

__global__ void k_scale(const float* __restrict__ a, float s, uint64_t n, float* __restrict__ out)
{
    for (uint64_t i = blockIdx.x * 256ull + threadIdx.x; i < n; i += gridDim.x * 256ull) {
        out[i] = a[i] * s;
    }
}

}  // namespace

int eval_loss_grad(GpuTape& g, uint64_t n, const float* x, const float* y, const float* z,
                   float* f, float* gx, float* gy, float* gz, float* gvars, float* loss,
                   cudaStream_t s)
{
    if (!require_device()) return LFB_E_CUDA;
    if (!x || !y || !z || !f) return set_error(LFB_E_INVALID, "lfb_eval_loss_grad: null argument");
    if (n == 0) return set_error(LFB_E_INVALID, "lfb_eval_loss_grad: no points");
    std::lock_guard<std::mutex> lock(global_mutex());
    const float scale = static_cast<float>(2.0 / static_cast<double>(n));
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256,
                                                                     device_sm_count() * 8ull));
    auto& st = grad_staging();
    if (!st.out.reserve(sizeof(double))) return LFB_E_CUDA;
    double* sum = st.out.as<double>();
    if (const uint32_t ckf = jit_ckpt_prepare(g)) {
        // one forward pass gives f and the checkpoints; the backward pass
        // takes seed 2 f_i / n
        const uint64_t per_point = 4ull * ckf;
        const uint64_t cchunk = std::max<uint64_t>(kBlock, std::min<uint64_t>(
            (4ull << 30) / per_point / kBlock * kBlock, uint64_t(1) << 22));
        if (!st.partials.reserve(std::min(cchunk, n) * per_point)) return LFB_E_CUDA;
        float* C = st.partials.as<float>();
        const bool has_cv = tape_has_const_var(g);
        for (uint64_t off = 0; off < n; off += cchunk) {
            const uint32_t m = static_cast<uint32_t>(std::min(cchunk, n - off));
            if (!jit_ckpt_forward(g, m, x + off, y + off, z + off, C, f + off, s)) {
                return set_error(LFB_E_CUDA, "checkpointed gradient kernel launch failed");
            }
            float* ox = gx ? gx + off : nullptr;
            float* oy = gy ? gy + off : nullptr;
            float* oz = gz ? gz + off : nullptr;
            bool ok = true;
            if (!has_cv) {
                ok = jit_ckpt_backward(g, m, C, f + off, ox, oy, oz, gvars, 0, s, scale);
            } else {
                ok = jit_ckpt_backward(g, m, C, f + off, ox, oy, oz, nullptr, 0, s, scale) &&
                     (!gvars || jit_ckpt_backward(g, m, C, f + off, nullptr, nullptr, nullptr,
                                                  gvars, 1, s, scale));
            }
            if (!ok) return set_error(LFB_E_CUDA, "checkpointed gradient kernel launch failed");
        }
    } else {
        // without compiled kernels: values, then the gradient with seed 2 f / n
        const int rc = eval_values_device(g, n, x, y, z, f, s);
        if (rc) return rc;
        if (!st.in.reserve(n * sizeof(float))) return LFB_E_CUDA;
        float* seed = st.in.as<float>();
        k_scale<<<blocks, 256, 0, s>>>(f, scale, n, seed);
        note_launches(1);
        const int rc2 = grad_device(g, n, x, y, z, seed, nullptr, gx, gy, gz, gvars, s);
        if (rc2) return rc2;
    }
    if (loss) {
        cudaMemsetAsync(sum, 0, sizeof(double), s);
        k_sum_squares<<<blocks, 256, 0, s>>>(f, n, sum);
        k_mean_to_float<<<1, 1, 0, s>>>(sum, n, loss);
        note_launches(2);
    }
    return cuda_ok(cudaGetLastError(), "loss gradient") ? 0 : LFB_E_CUDA;
}

int eval_grad(GpuTape& g, uint64_t n, const float* x, const float* y, const float* z,
              const float* seed, float* f, float* gx, float* gy, float* gz, float* gvars,
              cudaStream_t s, bool device)
{
    if (!require_device()) return LFB_E_CUDA;
    if (!x || !y || !z) return set_error(LFB_E_INVALID, "lfb_eval_grad: null argument");
    std::lock_guard<std::mutex> lock(global_mutex());
    if (device) return grad_device(g, n, x, y, z, seed, f, gx, gy, gz, gvars, s);
    if (n == 0) return 0;
    // Host arrays: inputs x, y, z, seed; outputs f, gx, gy, gz; gvars.
    auto& st = grad_staging();
    const size_t nv = g.reg.n_vars;
    if (!st.in.reserve(n * 4 * sizeof(float)) ||
        !st.out.reserve((n * 4 + std::max<size_t>(nv, 1)) * sizeof(float))) {
        return LFB_E_CUDA;
    }
    float* d = st.in.as<float>();
    float* o = st.out.as<float>();
    const size_t b = n * sizeof(float);
    cudaStream_t s0 = 0;
    const float* ins[4] = {x, y, z, seed};
    for (int k = 0; k < 4; ++k) {
        if (ins[k] && !cuda_ok(cudaMemcpyAsync(d + k * n, ins[k], b, cudaMemcpyHostToDevice, s0),
                               "copy")) {
            return LFB_E_CUDA;
        }
    }
    float* gv = gvars ? o + 4 * n : nullptr;
    if (gv && !cuda_ok(cudaMemcpyAsync(gv, gvars, nv * sizeof(float), cudaMemcpyHostToDevice, s0),
                       "copy")) {
        return LFB_E_CUDA;
    }
    float* outs[4] = {f, gx, gy, gz};
    const int rc = grad_device(g, n, d, d + n, d + 2 * n, seed ? d + 3 * n : nullptr,
                               f ? o : nullptr, gx ? o + n : nullptr, gy ? o + 2 * n : nullptr,
                               gz ? o + 3 * n : nullptr, gv, s0);
    if (rc) return rc;
    for (int k = 0; k < 4; ++k) {
        if (outs[k] && !cuda_ok(cudaMemcpyAsync(outs[k], o + k * n, b, cudaMemcpyDeviceToHost, s0),
                                "copy")) {
            return LFB_E_CUDA;
        }
    }
    if (gv && !cuda_ok(cudaMemcpyAsync(gvars, gv, nv * sizeof(float), cudaMemcpyDeviceToHost, s0),
                       "copy")) {
        return LFB_E_CUDA;
    }
    return cuda_ok(cudaStreamSynchronize(s0), "sync") ? 0 : LFB_E_CUDA;
}

}  // namespace lfb
