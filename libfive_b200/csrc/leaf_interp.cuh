// Tape interpreters of the leaf stage (DCTree::evalLeaf, libfive/src/render/
// brep/dc/dc_tree.inl:131-552): the clauses of a leaf group's pruned tape
// evaluated by one warp at four points per lane (corners and edge search,
// ArrayEvaluator::values, eval_array.cpp:106-118) or at one point per lane
// with derivatives (DerivArrayEvaluator::derivs, eval_deriv_array.cpp:
// 101-117).
//
// Layout for throughput on an interpreter whose cost is per clause:
//  * the warp first decodes a chunk of kLeafOps register-tape clauses into
//    LeafOps in shared memory (one clause per lane): opcode and operand kinds
//    become one handler number, constant and free-variable operands become
//    an immediate value, so the evaluation loop reads one 16-byte broadcast
//    word per clause and branches once;
//  * the register file holds one float4 per (register, lane): the four
//    points of a lane (or value + gradient) move with one 128-bit shared
//    memory access per operand.
// Arithmetic is the per-opcode arithmetic of dev_point.cuh, operation for
// operation, so values are bit-identical to the other evaluators'.
#pragma once
#include "dc_features.cuh"
#include "dev_interval.cuh"
#include "dev_point.cuh"

namespace lfb {

/// One decoded clause.  a, b, o are register numbers; `imm` is the value
/// of the immediate operand (flags bit 0: a is immediate, bit 1: b is; an
/// operand kind of OPND_CONST or OPND_VAR).  A clause whose every operand is
/// immediate is folded into H_SET (imm = its result; flags bit 2: it is a
/// min / max whose arguments tie).
struct __align__(16) LeafOp {
    uint8_t h;
    uint8_t op;
    uint8_t flags;
    uint8_t pad0;
    uint16_t a, b, o;
    uint16_t pad1;
    float imm;
};
static_assert(sizeof(LeafOp) == 16, "LeafOp is one 16-byte word");

enum : uint8_t {
    H_ADD_RR, H_ADD_RI, H_MUL_RR, H_MUL_RI, H_SUB_RR, H_SUB_RI, H_SUB_IR,
    H_MIN_RR, H_MIN_RI, H_MIN_IR, H_MAX_RR, H_MAX_RI, H_MAX_IR,
    H_SQUARE, H_SQRT, H_NEG, H_ABS, H_COPY, H_SET, H_GENERIC,
};

constexpr uint32_t kLeafOps = 64;   // decoded clauses per warp and chunk

/// Decodes one register-tape clause.  ADD and MUL with an immediate first
/// operand are swapped (both are exactly commutative, values and
/// derivatives alike); MIN, MAX and SUB are not.  `prev_out` is the result
/// register of the clause before (or 0xffff): flags bit 3 / bit 4 say that
/// operand a / b is that result, which the interpreters then take from
/// their registers instead of the register file.
__device__ __forceinline__ LeafOp leaf_decode(const RegClause& c, const float* __restrict__ cpool,
                                              uint32_t prev_out)
{
    LeafOp L;
    L.op = c.op;
    L.pad0 = 0;
    L.pad1 = 0;
    L.a = c.a;
    L.b = c.b;
    L.o = c.out;
    const uint8_t ka = c.kinds & 3, kb = (c.kinds >> 2) & 3;
    const bool bin = dev_is_binary(c.op);
    const bool ai = ka != OPND_REG, bi = bin && kb != OPND_REG;
    const float va = ai ? __ldg(cpool + c.a) : 0.0f;
    const float vb = bi ? __ldg(cpool + c.b) : 0.0f;
    L.flags = (ai ? 1 : 0) | (bi ? 2 : 0);
    L.imm = ai ? va : vb;
    if (ai && (bi || !bin)) {
        L.h = H_SET;
        L.imm = dv_value(c.op, va, vb);
        if ((c.op == op::MIN || c.op == op::MAX) && va == vb) L.flags |= 4;
        return L;
    }
    uint8_t h = H_GENERIC;
    switch (c.op) {
        case op::ADD:
        case op::MUL: {
            const bool mul = c.op == op::MUL;
            if (!ai && !bi) {
                h = mul ? H_MUL_RR : H_ADD_RR;
            } else {
                h = mul ? H_MUL_RI : H_ADD_RI;
                if (ai) {   // swap: register first
                    L.a = c.b;
                    L.b = c.a;
                    L.flags = 2;
                }
            }
            break;
        }
        case op::SUB: h = ai ? H_SUB_IR : bi ? H_SUB_RI : H_SUB_RR; break;
        case op::MIN: h = ai ? H_MIN_IR : bi ? H_MIN_RI : H_MIN_RR; break;
        case op::MAX: h = ai ? H_MAX_IR : bi ? H_MAX_RI : H_MAX_RR; break;
        case op::SQUARE: h = H_SQUARE; break;
        case op::SQRT: h = H_SQRT; break;
        case op::NEG: h = H_NEG; break;
        case op::ABS: h = H_ABS; break;
        case op::CONST_VAR:
        case OP_COPY: h = H_COPY; break;
        default: h = H_GENERIC; break;
    }
    L.h = h;
    if (!(L.flags & 1) && L.a == prev_out) L.flags |= 8;
    if (!(L.flags & 2) && dev_is_binary(c.op) && L.b == prev_out) L.flags |= 16;
    return L;
}

__device__ __forceinline__ RegClause leaf_unpack(uint2 raw)
{
    RegClause c;
    c.op = raw.x & 0xff;
    c.kinds = (raw.x >> 8) & 0xff;
    c.out = raw.x >> 16;
    c.a = raw.y & 0xffff;
    c.b = raw.y >> 16;
    return c;
}

/// The raw words of clauses c0 + lane and c0 + 32 + lane (the lane's share
/// of one chunk), loaded ahead of leaf_decode_chunk.
struct LeafRaw {
    uint2 w[2];
};
__device__ __forceinline__ LeafRaw leaf_fetch(const RegClause* __restrict__ cl, uint32_t len,
                                              uint32_t c0, int lane)
{
    LeafRaw r;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const uint32_t i = c0 + lane + 32 * k;
        r.w[k] = i < len ? __ldg(reinterpret_cast<const uint2*>(cl + i)) : make_uint2(0, 0);
    }
    return r;
}

/// Decodes clauses [c0, c0 + kLeafOps) of a tape, whose raw words this lane
/// fetched into `raw`, into `ops` (the warp together); returns how many
/// there were.
__device__ __forceinline__ uint32_t leaf_decode_chunk(LeafOp* ops, const LeafRaw& raw,
                                                      uint32_t len, uint32_t c0,
                                                      const float* __restrict__ cpool, int lane)
{
    static_assert(kLeafOps == 64, "two clauses per lane");
    const uint32_t n = min(kLeafOps, len - c0);
    // result register of the clause before each of this lane's two
    const uint32_t out0 = raw.w[0].x >> 16, out1 = raw.w[1].x >> 16;
    const uint32_t up0 = __shfl_up_sync(0xffffffffu, out0, 1);
    const uint32_t last0 = __shfl_sync(0xffffffffu, out0, 31);
    const uint32_t up1 = __shfl_up_sync(0xffffffffu, out1, 1);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const uint32_t i = lane + 32 * k;
        if (i < n) {
            // the interpreters' forwarded result does not outlive a chunk:
            // nothing is forwarded into a chunk's first clause
            const uint32_t prev = lane > 0 ? (k ? up1 : up0) : (k ? last0 : 0xffffu);
            ops[i] = leaf_decode(leaf_unpack(raw.w[k]), cpool, prev);
        }
    }
    __syncwarp();
    return n;
}

__device__ __forceinline__ float4 splat4(float v) { return make_float4(v, v, v, v); }

#define LFB_MAP2(F, a, b) make_float4(F((a).x, (b).x), F((a).y, (b).y), F((a).z, (b).z), F((a).w, (b).w))
#define LFB_MAP1(F, a) make_float4(F((a).x), F((a).y), F((a).z), F((a).w))

__device__ __forceinline__ float f_square(float a) { return __fmul_rn(a, a); }
__device__ __forceinline__ float f_neg(float a) { return -a; }
__device__ __forceinline__ float f_sqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ float f_abs(float a) { return fabsf(a); }
__device__ __forceinline__ float f_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float f_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float f_mul(float a, float b) { return __fmul_rn(a, b); }

__device__ __forceinline__ uint32_t tie4(const float4& a, const float4& b)
{
    return (a.x == b.x ? 1u : 0u) | (a.y == b.y ? 2u : 0u) | (a.z == b.z ? 4u : 0u) |
           (a.w == b.w ? 8u : 0u);
}

/// Every other opcode on four points, out of line.
static __device__ __noinline__ float4 leaf_generic4(uint8_t o, float4 a, float4 b)
{
    return make_float4(dv_value(o, a.x, b.x), dv_value(o, a.y, b.y), dv_value(o, a.z, b.z),
                       dv_value(o, a.w, b.w));
}

#undef LFB_MAP1
#undef LFB_MAP2

__device__ __forceinline__ D4 d4_of(const float4& f) { return {f.x, f.y, f.z, f.w}; }

/// The derivative interpreter's clause loop (one point per lane, value and
/// d/dx, d/dy, d/dz per register as a float4) with the tie settling of the
/// feature rules: see leaf_deriv in dc_kernels.cu.  `taint` holds one bit per
/// register (registers above 63 share bits and are reported as lost).
__device__ __forceinline__ void leaf_run_deriv(const LeafOp* __restrict__ ops, uint32_t n,
                                               float4* R, uint64_t& taint, bool& amb,
                                               bool& lost, bool trackable)
{
    float4 last = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    LeafOp L = ops[0];
#pragma unroll 1
    for (uint32_t c = 0; c < n; ++c) {
        const LeafOp next = ops[c + 1 < n ? c + 1 : c];
        D4 r;
        bool t_out;
        if (L.h == H_SET) {
            if (L.flags & 4) {
                amb = true;
                lost |= !trackable;
            }
            r = D4{L.imm, 0.0f, 0.0f, 0.0f};
            t_out = false;
        } else {
            const uint8_t o = L.op;
            const bool ai = L.flags & 1, bi = L.flags & 2;
            const bool binary = dev_is_binary(o);
            const D4 a = ai ? D4{L.imm, 0.0f, 0.0f, 0.0f}
                            : d4_of(L.flags & 8 ? last : R[L.a * 32]);
            const D4 b = bi ? D4{L.imm, 0.0f, 0.0f, 0.0f}
                            : binary ? d4_of(L.flags & 16 ? last : R[L.b * 32])
                                     : D4{0.0f, 0.0f, 0.0f, 0.0f};
            const bool ta = !ai && ((taint >> (L.a & 63)) & 1);
            const bool tbb = binary && !bi && ((taint >> (L.b & 63)) & 1);
            if ((o == op::MIN || o == op::MAX) && a.v == b.v) {
                amb = true;
                lost |= !trackable;
                const bool is_min = o == op::MIN;
                const float e[3] = {is_min ? b.dx - a.dx : a.dx - b.dx,
                                    is_min ? b.dy - a.dy : a.dy - b.dy,
                                    is_min ? b.dz - a.dz : a.dz - b.dz};
                const float nrm = sqrtf(fdot(e, e));
                bool take_b = false;
                t_out = ta || tbb;
                if (!t_out && nrm != 0) {
                    const float dd[3] = {b.dx - a.dx, b.dy - a.dy, b.dz - a.dz};
                    if (!(static_cast<double>(fdot(dd, dd)) < 1e-10)) {
                        t_out = true;
                    } else {
                        const float en[3] = {e[0] / nrm, e[1] / nrm, e[2] / nrm};
                        const float ep[3] = {-en[0], -en[1], -en[2]};
                        const float ad[3] = {a.dx, a.dy, a.dz}, bd[3] = {b.dx, b.dy, b.dz};
                        // Candidate order: b's feature carries -e, a's carries e.
                        const int cmp = vcmp3(ep, en);
                        take_b = cmp != 0 ? cmp < 0 : vcmp3(bd, ad) < 0;
                    }
                }
                r = take_b ? D4{dv_value(o, a.v, b.v), b.dx, b.dy, b.dz}
                           : D4{dv_value(o, a.v, b.v), a.dx, a.dy, a.dz};
            } else {
                r = dv_deriv(o, a, b, false);
                if (o == op::MIN) t_out = (a.v < b.v) ? ta : tbb;
                else if (o == op::MAX) t_out = (a.v < b.v) ? tbb : ta;
                else t_out = ta || tbb;
            }
        }
        if (t_out) taint |= 1ull << (L.o & 63);
        else taint &= ~(1ull << (L.o & 63));
        last = make_float4(r.v, r.dx, r.dy, r.dz);
        R[L.o * 32] = last;
        L = next;
    }
}

}  // namespace lfb
