// Point-wise value and derivative rules of the tape evaluators
// (ArrayEvaluator::operator(), libfive/src/eval/eval_array.cpp:221-369, and
// DerivArrayEvaluator::operator(), libfive/src/eval/eval_deriv_array.cpp:
// 119-256).  Included by the CUDA sources and, as text, by kernels compiled
// at run time, so it depends only on the opcode numbers and the scalar ops.
#pragma once
#ifndef __CUDACC_RTC__
#include <cstdint>
#endif

#include "opcode_ids.h"
#include "scalar_ops.h"

namespace lfb {

////////////////////////////////////////////////////////////////////////////////
// Value mode

/// Opcodes that call a math-library function or have long bodies; kept out
/// of line so that the interpreters' hot switch stays small.
static __device__ __noinline__ float dv_value_rare(uint8_t o, float a, float b)
{
    switch (o) {
        case op::ATAN2: return atan2f(a, b);
        case op::POW: return powf(a, b);
        case op::NTH_ROOT: return sc_nth_root(a, b);
        case op::MOD: {
            float d = fabsf(__fdiv_rn(a, b));
            if ((a < 0) ^ (b < 0)) d = -ceilf(d); else d = floorf(d);
            float out = __fsub_rn(a, __fmul_rn(b, d));
            if ((b > 0 && out > b) || (b < 0 && out < b)) out = b;
            if ((b > 0.0f && out < 0.0f) || (b < 0.0f && out > 0.0f)) out = 0.0f;
            return out;
        }
        case op::NANFILL: return (a != a) ? b : a;
        case op::COMPARE: return sc_compare(a, b);
        case op::SIN: return sinf(a);
        case op::COS: return cosf(a);
        case op::TAN: return tanf(a);
        case op::ASIN: return asinf(a);
        case op::ACOS: return acosf(a);
        case op::ATAN: return atanf(a);
        default: return __int_as_float(0x7fc00000);
    }
}

__device__ __forceinline__ float dv_value(uint8_t o, float a, float b)
{
    switch (o) {
        case op::ADD: return __fadd_rn(a, b);
        case op::MUL: return __fmul_rn(a, b);
        case op::MIN: return sc_min(a, b);
        case op::MAX: return sc_max(a, b);
        case op::SUB: return __fsub_rn(a, b);
        case op::DIV: return __fdiv_rn(a, b);
        case op::SQUARE: return __fmul_rn(a, a);
        case op::SQRT: return __fsqrt_rn(a);
        case op::NEG: return -a;
        case op::LOG: return logf(a);
        case op::EXP: return expf(a);
        case op::ABS: return fabsf(a);
        case op::RECIP: return __fdiv_rn(1.0f, a);
        case op::CONST_VAR: return a;
        case OP_COPY: return a;
        default: return dv_value_rare(o, a, b);
    }
}

/// dv_value on four independent points (one clause, four lanes' worth of
/// work per thread): the clause is decoded once for all four.
__device__ __forceinline__ void dv_value4(uint8_t o, const float (&a)[4],
                                          const float (&b)[4], float (&r)[4])
{
#define LFB_EACH(expr) _Pragma("unroll") for (int k = 0; k < 4; ++k) r[k] = (expr); break
    switch (o) {
        case op::ADD: LFB_EACH(__fadd_rn(a[k], b[k]));
        case op::MUL: LFB_EACH(__fmul_rn(a[k], b[k]));
        case op::MIN: LFB_EACH(sc_min(a[k], b[k]));
        case op::MAX: LFB_EACH(sc_max(a[k], b[k]));
        case op::SUB: LFB_EACH(__fsub_rn(a[k], b[k]));
        case op::DIV: LFB_EACH(__fdiv_rn(a[k], b[k]));
        case op::SQUARE: LFB_EACH(__fmul_rn(a[k], a[k]));
        case op::SQRT: LFB_EACH(__fsqrt_rn(a[k]));
        case op::NEG: LFB_EACH(-a[k]);
        case op::LOG: LFB_EACH(logf(a[k]));
        case op::EXP: LFB_EACH(expf(a[k]));
        case op::ABS: LFB_EACH(fabsf(a[k]));
        case op::RECIP: LFB_EACH(__fdiv_rn(1.0f, a[k]));
        case op::CONST_VAR:
        case OP_COPY: LFB_EACH(a[k]);
        default: LFB_EACH(dv_value_rare(o, a[k], b[k]));
    }
#undef LFB_EACH
}

////////////////////////////////////////////////////////////////////////////////
// Derivative mode: value in .x, partials in .y/.z/.w (d/dx, d/dy, d/dz)

struct D4 {
    float v, dx, dy, dz;
};

// Applies a scalar factor to all three partials, in the same order as the
// reference's Eigen expressions (partial * factor).
__device__ __forceinline__ D4 d4_scale(float v, const D4& a, float f)
{
    return {v, __fmul_rn(a.dx, f), __fmul_rn(a.dy, f), __fmul_rn(a.dz, f)};
}

static __device__ __noinline__ D4 dv_deriv_all(uint8_t o, const D4& a, const D4& b,
                                               bool clear_vars)
{
    const float av = a.v, bv = b.v;
    const float ov = dv_value(o, av, bv);
    switch (o) {
        case op::ADD:
            return {ov, __fadd_rn(a.dx, b.dx), __fadd_rn(a.dy, b.dy),
                    __fadd_rn(a.dz, b.dz)};
        case op::SUB:
            return {ov, __fsub_rn(a.dx, b.dx), __fsub_rn(a.dy, b.dy),
                    __fsub_rn(a.dz, b.dz)};
        case op::MUL:
            // od = bd * av + ad * bv
            return {ov,
                    __fadd_rn(__fmul_rn(b.dx, av), __fmul_rn(a.dx, bv)),
                    __fadd_rn(__fmul_rn(b.dy, av), __fmul_rn(a.dy, bv)),
                    __fadd_rn(__fmul_rn(b.dz, av), __fmul_rn(a.dz, bv))};
        case op::MIN:
            return (av < bv) ? D4{ov, a.dx, a.dy, a.dz}
                             : D4{ov, b.dx, b.dy, b.dz};
        case op::MAX:
            return (av < bv) ? D4{ov, b.dx, b.dy, b.dz}
                             : D4{ov, a.dx, a.dy, a.dz};
        case op::DIV: {
            // od = (ad * bv - bd * av) / bv^2
            const float den = __fmul_rn(bv, bv);
            return {ov,
                    __fdiv_rn(__fsub_rn(__fmul_rn(a.dx, bv), __fmul_rn(b.dx, av)), den),
                    __fdiv_rn(__fsub_rn(__fmul_rn(a.dy, bv), __fmul_rn(b.dy, av)), den),
                    __fdiv_rn(__fsub_rn(__fmul_rn(a.dz, bv), __fmul_rn(b.dz, av)), den)};
        }
        case op::ATAN2: {
            const float den = __fadd_rn(__fmul_rn(av, av), __fmul_rn(bv, bv));
            return {ov,
                    __fdiv_rn(__fsub_rn(__fmul_rn(a.dx, bv), __fmul_rn(b.dx, av)), den),
                    __fdiv_rn(__fsub_rn(__fmul_rn(a.dy, bv), __fmul_rn(b.dy, av)), den),
                    __fdiv_rn(__fsub_rn(__fmul_rn(a.dz, bv), __fmul_rn(b.dz, av)), den)};
        }
        case op::POW: {
            // The exponent is a constant, so only the base contributes.
            const float f = __fmul_rn(bv, powf(av, __fsub_rn(bv, 1.0f)));
            return d4_scale(ov, a, f);
        }
        case op::NTH_ROOT: {
            const float f = __fdiv_rn(powf(av, __fsub_rn(__fdiv_rn(1.0f, bv), 1.0f)), bv);
            return {ov, a.dx == 0 ? 0.0f : __fmul_rn(a.dx, f),
                        a.dy == 0 ? 0.0f : __fmul_rn(a.dy, f),
                        a.dz == 0 ? 0.0f : __fmul_rn(a.dz, f)};
        }
        case op::MOD:
            return {ov, a.dx, a.dy, a.dz};
        case op::NANFILL:
            return (av != av) ? D4{ov, b.dx, b.dy, b.dz}
                              : D4{ov, a.dx, a.dy, a.dz};
        case op::COMPARE:
            return {ov, 0.0f, 0.0f, 0.0f};
        case op::SQUARE:
            // od = ad * av * 2
            return {ov, __fmul_rn(__fmul_rn(a.dx, av), 2.0f),
                        __fmul_rn(__fmul_rn(a.dy, av), 2.0f),
                        __fmul_rn(__fmul_rn(a.dz, av), 2.0f)};
        case op::SQRT: {
            const float den = __fmul_rn(2.0f, ov);
            const bool neg = av < 0;
            return {ov, (neg || a.dx == 0) ? 0.0f : __fdiv_rn(a.dx, den),
                        (neg || a.dy == 0) ? 0.0f : __fdiv_rn(a.dy, den),
                        (neg || a.dz == 0) ? 0.0f : __fdiv_rn(a.dz, den)};
        }
        case op::NEG:
            return {ov, -a.dx, -a.dy, -a.dz};
        case op::SIN:
            return d4_scale(ov, a, cosf(av));
        case op::COS:
            return d4_scale(ov, a, -sinf(av));
        case op::TAN: {
            const float s = __fdiv_rn(1.0f, cosf(av));
            return d4_scale(ov, a, __fmul_rn(s, s));
        }
        case op::ASIN: {
            const float den = __fsqrt_rn(__fsub_rn(1.0f, __fmul_rn(av, av)));
            return {ov, __fdiv_rn(a.dx, den), __fdiv_rn(a.dy, den),
                        __fdiv_rn(a.dz, den)};
        }
        case op::ACOS: {
            const float den = -__fsqrt_rn(__fsub_rn(1.0f, __fmul_rn(av, av)));
            return {ov, __fdiv_rn(a.dx, den), __fdiv_rn(a.dy, den),
                        __fdiv_rn(a.dz, den)};
        }
        case op::ATAN: {
            const float den = __fadd_rn(__fmul_rn(av, av), 1.0f);
            return {ov, __fdiv_rn(a.dx, den), __fdiv_rn(a.dy, den),
                        __fdiv_rn(a.dz, den)};
        }
        case op::LOG:
            return {ov, __fdiv_rn(a.dx, av), __fdiv_rn(a.dy, av),
                        __fdiv_rn(a.dz, av)};
        case op::EXP:
            return d4_scale(ov, a, expf(av));
        case op::ABS:
            return (av > 0) ? D4{ov, a.dx, a.dy, a.dz}
                            : D4{ov, -a.dx, -a.dy, -a.dz};
        case op::RECIP: {
            const float den = -__fmul_rn(av, av);
            return {ov, __fdiv_rn(a.dx, den), __fdiv_rn(a.dy, den),
                        __fdiv_rn(a.dz, den)};
        }
        case op::CONST_VAR:
            return clear_vars ? D4{ov, 0.0f, 0.0f, 0.0f}
                              : D4{ov, a.dx, a.dy, a.dz};
        case OP_COPY:
            return a;
        default:
            return {__int_as_float(0x7fc00000), 0.0f, 0.0f, 0.0f};
    }
}

/// Hot-path derivative rules inline; everything else out of line.
__device__ __forceinline__ D4 dv_deriv(uint8_t o, const D4& a, const D4& b,
                                       bool clear_vars)
{
    const float av = a.v, bv = b.v;
    switch (o) {
        case op::ADD:
            return {__fadd_rn(av, bv), __fadd_rn(a.dx, b.dx), __fadd_rn(a.dy, b.dy),
                    __fadd_rn(a.dz, b.dz)};
        case op::SUB:
            return {__fsub_rn(av, bv), __fsub_rn(a.dx, b.dx), __fsub_rn(a.dy, b.dy),
                    __fsub_rn(a.dz, b.dz)};
        case op::MUL:
            return {__fmul_rn(av, bv),
                    __fadd_rn(__fmul_rn(b.dx, av), __fmul_rn(a.dx, bv)),
                    __fadd_rn(__fmul_rn(b.dy, av), __fmul_rn(a.dy, bv)),
                    __fadd_rn(__fmul_rn(b.dz, av), __fmul_rn(a.dz, bv))};
        case op::MIN:
            return (av < bv) ? D4{sc_min(av, bv), a.dx, a.dy, a.dz}
                             : D4{sc_min(av, bv), b.dx, b.dy, b.dz};
        case op::MAX:
            return (av < bv) ? D4{sc_max(av, bv), b.dx, b.dy, b.dz}
                             : D4{sc_max(av, bv), a.dx, a.dy, a.dz};
        case op::SQUARE:
            return {__fmul_rn(av, av), __fmul_rn(__fmul_rn(a.dx, av), 2.0f),
                    __fmul_rn(__fmul_rn(a.dy, av), 2.0f),
                    __fmul_rn(__fmul_rn(a.dz, av), 2.0f)};
        case op::NEG:
            return {-av, -a.dx, -a.dy, -a.dz};
        case op::ABS:
            return (av > 0) ? D4{fabsf(av), a.dx, a.dy, a.dz}
                            : D4{fabsf(av), -a.dx, -a.dy, -a.dz};
        case OP_COPY:
            return a;
        default:
            return dv_deriv_all(o, a, b, clear_vars);
    }
}

}  // namespace lfb
