// Interval arithmetic of the tape evaluators (IntervalEvaluator,
// libfive/src/eval/eval_interval.cpp:189-294, and Boost.Interval's rounded
// operations used by libfive/include/libfive/eval/interval.hpp:31-442).
// Included by the CUDA sources and, as text, by kernels compiled at run
// time, so it depends only on the opcode numbers and min/max.
#pragma once
#ifndef __CUDACC_RTC__
#include <cstdint>
#endif

#include "opcode_ids.h"
#include "scalar_minmax.h"

namespace lfb {

////////////////////////////////////////////////////////////////////////////////
// Interval mode

struct Iv {
    float lo, hi;
    bool nan;   // "may be NaN" flag of the reference's Interval
};

#define LF_INF __int_as_float(0x7f800000)
#define LF_QNAN __int_as_float(0x7fc00000)

// Boost.Interval's "checking_base" emptiness test: any NaN bound or
// lower > upper marks the interval as empty, represented as [NaN, NaN].
__device__ __forceinline__ bool iv_bad(float lo, float hi) { return !(lo <= hi); }
__device__ __forceinline__ bool iv_bad(const Iv& a) { return !(a.lo <= a.hi); }

/// Interval(lower, upper): the flag is set for NaN bounds, and an invalid
/// pair becomes the empty interval (boost interval constructor).
__device__ __forceinline__ Iv iv_make(float lo, float hi)
{
    const bool n = (lo != lo) || (hi != hi);
    if (iv_bad(lo, hi)) return {LF_QNAN, LF_QNAN, n};
    return {lo, hi, n};
}

__device__ __forceinline__ float ulp_down(float v, int k)
{
    for (int i = 0; i < k; ++i) v = nextafterf(v, -LF_INF);
    return v;
}
__device__ __forceinline__ float ulp_up(float v, int k)
{
    for (int i = 0; i < k; ++i) v = nextafterf(v, LF_INF);
    return v;
}

// Outward-widened transcendental bounds.  The reference calls the C library
// function under FE_DOWNWARD / FE_UPWARD (Boost's rounded_transc_std), which
// is not a directed bound; here each CUDA function result is widened
// outward by more than its documented maximum ULP error so that the true
// value, and the C library's, is enclosed.
#define LF_TRANSC_ULPS 4
#define LF_TRANSC_ULPS_WIDE 6

__device__ __forceinline__ float pi_f_lo() { return 3.14159250259399414062f; }  // 13176794 / 2^22
__device__ __forceinline__ float pi_f_hi() { return 3.14159274101257324219f; }  // 13176795 / 2^22

// Scalar times interval (Boost operator*(T, interval)).
__device__ __forceinline__ Iv iv_smul(float x, float lo, float hi)
{
    if ((x != x) || iv_bad(lo, hi)) return {LF_QNAN, LF_QNAN, false};
    if (x < 0) return {__fmul_rd(x, hi), __fmul_ru(x, lo), false};
    if (x == 0) return {0.0f, 0.0f, false};
    return {__fmul_rd(x, lo), __fmul_ru(x, hi), false};
}

__device__ __forceinline__ Iv iv_isub(float alo, float ahi, float blo, float bhi)
{
    if (iv_bad(alo, ahi) || iv_bad(blo, bhi)) return {LF_QNAN, LF_QNAN, false};
    return {__fsub_rd(alo, bhi), __fsub_ru(ahi, blo), false};
}

// Boost fmod(interval, interval) used by the trigonometric functions.
__device__ __forceinline__ Iv iv_fmod(float xlo, float xhi, float ylo, float yhi)
{
    if (iv_bad(xlo, xhi) || iv_bad(ylo, yhi)) return {LF_QNAN, LF_QNAN, false};
    const float yb = (xlo < 0) ? ylo : yhi;
    const float n = floorf(__fdiv_rd(xlo, yb));
    const Iv ny = iv_smul(n, ylo, yhi);
    return iv_isub(xlo, xhi, ny.lo, ny.hi);
}

__device__ inline Iv iv_cos_bounds(float lo, float hi, int depth = 0)
{
    if (iv_bad(lo, hi)) return {LF_QNAN, LF_QNAN, false};
    const float pi2lo = __fmul_rd(pi_f_lo(), 2.0f);
    const float pi2hi = __fmul_ru(pi_f_hi(), 2.0f);
    Iv tmp = iv_fmod(lo, hi, pi2lo, pi2hi);
    if (iv_bad(tmp)) return {LF_QNAN, LF_QNAN, false};
    if (__fsub_ru(tmp.hi, tmp.lo) >= pi2lo) return {-1.0f, 1.0f, false};
    if (tmp.lo >= pi_f_hi()) {
        if (depth > 2) return {-1.0f, 1.0f, false};
        const Iv s = iv_isub(tmp.lo, tmp.hi, pi_f_lo(), pi_f_hi());
        const Iv c = iv_cos_bounds(s.lo, s.hi, depth + 1);
        if (iv_bad(c)) return c;
        return {-c.hi, -c.lo, false};
    }
    const float l = tmp.lo, u = tmp.hi;
    if (u <= pi_f_lo()) {
        return {fmaxf(-1.0f, ulp_down(cosf(u), LF_TRANSC_ULPS)),
                fminf(1.0f, ulp_up(cosf(l), LF_TRANSC_ULPS))};
    } else if (u <= pi2lo) {
        const float m = sc_min(__fsub_rd(pi2lo, u), l);
        return {-1.0f, fminf(1.0f, ulp_up(cosf(m), LF_TRANSC_ULPS))};
    }
    return {-1.0f, 1.0f, false};
}

__device__ __forceinline__ Iv iv_binary(uint8_t o, const Iv& a, const Iv& b)
{
    const bool bad = iv_bad(a) || iv_bad(b);
    switch (o) {
        case op::ADD: {
            const bool u = a.nan || b.nan || (a.lo == -LF_INF && b.hi == LF_INF) ||
                           (b.lo == -LF_INF && a.hi == LF_INF);
            if (bad) return {LF_QNAN, LF_QNAN, u};
            return {__fadd_rd(a.lo, b.lo), __fadd_ru(a.hi, b.hi), u};
        }
        case op::SUB: {
            const bool u = a.nan || b.nan ||
                           (a.lo == -LF_INF && b.lo == -LF_INF) ||
                           (a.hi == -LF_INF && b.hi == -LF_INF);
            if (bad) return {LF_QNAN, LF_QNAN, u};
            return {__fsub_rd(a.lo, b.hi), __fsub_ru(a.hi, b.lo), u};
        }
        case op::MUL: {
            const bool u = a.nan || b.nan ||
                ((a.lo == -LF_INF || a.hi == LF_INF) && b.lo <= 0.0f && b.hi >= 0.0f) ||
                ((b.lo == -LF_INF || b.hi == LF_INF) && a.lo <= 0.0f && a.hi >= 0.0f);
            if (bad) return {LF_QNAN, LF_QNAN, u};
            const float xl = a.lo, xu = a.hi, yl = b.lo, yu = b.hi;
            // Boost's nine-case sign analysis (P/M/N/Z for each argument).
            if (xl < 0) {
                if (xu > 0) {
                    if (yl < 0) {
                        if (yu > 0)
                            return {sc_min(__fmul_rd(xl, yu), __fmul_rd(xu, yl)),
                                    sc_max(__fmul_ru(xl, yl), __fmul_ru(xu, yu)), u};
                        return {__fmul_rd(xu, yl), __fmul_ru(xl, yl), u};
                    }
                    if (yu > 0) return {__fmul_rd(xl, yu), __fmul_ru(xu, yu), u};
                    return {0.0f, 0.0f, u};
                }
                if (yl < 0) {
                    if (yu > 0) return {__fmul_rd(xl, yu), __fmul_ru(xl, yl), u};
                    return {__fmul_rd(xu, yu), __fmul_ru(xl, yl), u};
                }
                if (yu > 0) return {__fmul_rd(xl, yu), __fmul_ru(xu, yl), u};
                return {0.0f, 0.0f, u};
            }
            if (xu > 0) {
                if (yl < 0) {
                    if (yu > 0) return {__fmul_rd(xu, yl), __fmul_ru(xu, yu), u};
                    return {__fmul_rd(xu, yl), __fmul_ru(xl, yu), u};
                }
                if (yu > 0) return {__fmul_rd(xl, yl), __fmul_ru(xu, yu), u};
                return {0.0f, 0.0f, u};
            }
            return {0.0f, 0.0f, u};
        }
        case op::DIV: {
            const bool u = a.nan || b.nan ||
                ((a.lo == -LF_INF || a.hi == LF_INF) &&
                 (b.lo == -LF_INF || b.hi == LF_INF)) ||
                (a.lo <= 0.0f && a.hi >= 0.0f && b.lo <= 0.0f && b.hi >= 0.0f);
            if (b.lo <= 0.0f && b.hi >= 0.0f) return {-LF_INF, LF_INF, u};
            if (bad) return {LF_QNAN, LF_QNAN, u};
            const float xl = a.lo, xu = a.hi, yl = b.lo, yu = b.hi;
            if (xu < 0) {
                if (yu < 0) return {__fdiv_rd(xu, yl), __fdiv_ru(xl, yu), u};
                return {__fdiv_rd(xl, yl), __fdiv_ru(xu, yu), u};
            } else if (xl < 0) {
                if (yu < 0) return {__fdiv_rd(xu, yu), __fdiv_ru(xl, yu), u};
                return {__fdiv_rd(xl, yl), __fdiv_ru(xu, yl), u};
            }
            if (yu < 0) return {__fdiv_rd(xu, yu), __fdiv_ru(xl, yl), u};
            return {__fdiv_rd(xl, yu), __fdiv_ru(xu, yl), u};
        }
        case op::MIN:
        case op::MAX: {
            Iv r;
            if (bad) {
                r = {LF_QNAN, LF_QNAN, false};
            } else if (o == op::MIN) {
                r = {sc_min(a.lo, b.lo), sc_min(a.hi, b.hi), false};
            } else {
                r = {sc_max(a.lo, b.lo), sc_max(a.hi, b.hi), false};
            }
            // std::min / std::max return NaN only through the first argument,
            // so a possibly-NaN second argument widens the result to include
            // the first (interval.hpp:93-137).
            if (b.nan) {
                const bool br = iv_bad(r), ba = iv_bad(a);
                if (br && ba) r = {LF_QNAN, LF_QNAN, false};
                else if (br) r = {a.lo, a.hi, false};
                else if (!ba) r = {sc_min(r.lo, a.lo), sc_max(r.hi, a.hi), false};
            }
            r.nan = a.nan;
            return r;
        }
        case op::ATAN2: {
            const Iv y = a, x = b;
            const bool u = y.nan || x.nan ||
                (x.lo <= 0.0f && x.hi >= 0.0f && y.lo <= 0.0f && y.hi >= 0.0f);
            const int k = LF_TRANSC_ULPS_WIDE;
            auto dn = [&](float p, float q) { return ulp_down(atan2f(p, q), k); };
            auto up = [&](float p, float q) { return ulp_up(atan2f(p, q), k); };
            const float PI = 3.14159274101257324219f;
            Iv r;
            if (x.lo > 0) {
                if (y.lo > 0) r = iv_make(dn(y.lo, x.hi), up(y.hi, x.lo));
                else if (y.hi < 0) r = iv_make(dn(y.lo, x.lo), up(y.hi, x.hi));
                else r = iv_make(dn(y.lo, x.lo), up(y.hi, x.lo));
            } else if (x.hi < 0) {
                if (y.lo > 0) r = iv_make(dn(y.hi, x.hi), up(y.lo, x.lo));
                else if (y.hi < 0) r = iv_make(dn(y.hi, x.lo), up(y.lo, x.hi));
                else r = iv_make(-PI, PI);
            } else {
                if (y.lo > 0) r = iv_make(dn(y.lo, x.hi), up(y.lo, x.lo));
                else if (y.hi < 0) r = iv_make(dn(y.hi, x.lo), up(y.hi, x.hi));
                else r = iv_make(-PI, PI);
            }
            r.nan = u;
            return r;
        }
        case op::POW: {
            // Integer power by repeated squaring with directed rounding
            // (Boost pow(interval, int)).
            // The flag follows interval.hpp:181-205 on a C library where
            // pow(0, -1) is +inf (a pole, not NaN) and pow(-1, n) is never
            // NaN for an integer n: only 0^0 and NaN inputs set it.
            const int p0 = static_cast<int>(b.lo);
            const bool a_zero = a.lo <= 0.0f && a.hi >= 0.0f;
            const bool u = a.nan || b.nan || (a_zero && p0 == 0);
            if (iv_bad(a)) return {LF_QNAN, LF_QNAN, u};
            auto pw = [](float x, int n, bool up_) {
                float y = (n & 1) ? x : 1.0f;
                n >>= 1;
                while (n > 0) {
                    x = up_ ? __fmul_ru(x, x) : __fmul_rd(x, x);
                    if (n & 1) y = up_ ? __fmul_ru(x, y) : __fmul_rd(x, y);
                    n >>= 1;
                }
                return y;
            };
            int p = p0 < 0 ? -p0 : p0;
            Iv r;
            if (p == 0) {
                if (a.lo == 0 && a.hi == 0) r = {LF_QNAN, LF_QNAN, u};
                else r = {1.0f, 1.0f, u};
                return r;
            }
            if (a.hi < 0) {
                const float yl = pw(-a.hi, p, false), yu = pw(-a.lo, p, true);
                r = (p & 1) ? Iv{-yu, -yl, u} : Iv{yl, yu, u};
            } else if (a.lo < 0) {
                if (p & 1) r = {-pw(-a.lo, p, true), pw(a.hi, p, true), u};
                else r = {0.0f, pw(sc_max(-a.lo, a.hi), p, true), u};
            } else {
                r = {pw(a.lo, p, false), pw(a.hi, p, true), u};
            }
            if (p0 < 0) {
                // 1 / r with Boost's division-by-interval rules.
                if (iv_bad(r)) return {LF_QNAN, LF_QNAN, u};
                if (r.lo <= 0 && r.hi >= 0) {
                    if (r.lo != 0 && r.hi != 0) return {-LF_INF, LF_INF, u};
                    if (r.lo != 0) return {-LF_INF, __fdiv_ru(1.0f, r.lo), u};
                    if (r.hi != 0) return {__fdiv_rd(1.0f, r.hi), LF_INF, u};
                    return {LF_QNAN, LF_QNAN, u};
                }
                return {__fdiv_rd(1.0f, r.hi), __fdiv_ru(1.0f, r.lo), u};
            }
            return r;
        }
        case op::NTH_ROOT: {
            const int k = static_cast<int>(b.lo);
            const bool u = a.nan || b.nan || (a.lo <= 0.0f && !(k & 2));
            if (iv_bad(a) || k <= 0) return {LF_QNAN, LF_QNAN, u};
            if (k == 1) return {a.lo, a.hi, u};
            const float inv = __fdiv_rn(1.0f, static_cast<float>(k));
            auto root_up = [&](float x) { return ulp_up(powf(x, inv), LF_TRANSC_ULPS_WIDE); };
            auto root_dn = [&](float x) { return ulp_down(powf(x, inv), LF_TRANSC_ULPS_WIDE); };
            if (!(a.hi > 0)) {
                if (a.hi == 0) {
                    if (!(k & 1) || a.lo == 0) return {0.0f, 0.0f, u};
                    return {-root_up(-a.lo), 0.0f, u};
                }
                if (!(k & 1)) return {LF_QNAN, LF_QNAN, u};
                return {-root_up(-a.lo), -root_dn(-a.hi), u};
            }
            const float hi = root_up(a.hi);
            if (!(a.lo > 0)) {
                if (!(k & 1) || a.lo == 0) return {0.0f, hi, u};
                return {-root_up(-a.lo), hi, u};
            }
            return {fmaxf(0.0f, root_dn(a.lo)), hi, u};
        }
        case op::MOD: {
            // Default: the whole range of possible remainders.
            Iv out = iv_make(fminf(b.lo, 0.0f), fmaxf(0.0f, b.hi));
            out.nan = false;
            if (isfinite(a.hi) && isfinite(a.lo)) {
                const int position = (b.hi >= 0.0f) + 2 * (b.lo <= 0.0f);
                float ulo = a.lo, uhi = a.hi;
                if (position == 2) { ulo = -a.hi; uhi = -a.lo; }
                if (position == 1 || position == 2) {
                    // |b| as an interval (b does not contain zero here)
                    float blo = b.lo, bhi = b.hi;
                    if (!(blo >= 0)) {
                        const float t = -bhi; bhi = -blo; blo = t;
                    }
                    const Iv q = iv_binary(op::DIV, Iv{ulo, uhi, false}, Iv{blo, bhi, false});
                    const int qi = static_cast<int>(floorf(q.lo));
                    if (qi == static_cast<int>(floorf(q.hi))) {
                        const Iv bq = iv_smul(static_cast<float>(qi), b.lo, b.hi);
                        out = iv_isub(a.lo, a.hi, bq.lo, bq.hi);
                    }
                } else if (position == 0) {
                    out = {LF_QNAN, LF_QNAN, false};
                }
            }
            out.nan = b.hi >= 0.0f && b.lo <= 0.0f;
            return out;
        }
        case op::NANFILL: {
            if (a.nan) {
                const bool ba = iv_bad(a), bb = iv_bad(b);
                Iv r;
                if (ba && bb) r = {LF_QNAN, LF_QNAN, false};
                else if (ba) r = {b.lo, b.hi, false};
                else if (bb) r = {a.lo, a.hi, false};
                else r = {sc_min(a.lo, b.lo), sc_max(a.hi, b.hi), false};
                r.nan = b.nan;
                return r;
            }
            return {a.lo, a.hi, false};
        }
        case op::COMPARE:
            if (a.hi < b.lo) return {-1.0f, -1.0f, false};
            if (a.lo > b.hi) return {1.0f, 1.0f, false};
            return {-1.0f, 1.0f, false};
        default:
            return {LF_QNAN, LF_QNAN, true};
    }
}

__device__ __forceinline__ Iv iv_unary(uint8_t o, const Iv& a)
{
    const bool bad = iv_bad(a);
    const float lo = a.lo, hi = a.hi;
    switch (o) {
        case op::SQUARE: {
            if (bad) return {LF_QNAN, LF_QNAN, a.nan};
            if (hi < 0) return {__fmul_rd(hi, hi), __fmul_ru(lo, lo), a.nan};
            if (lo > 0) return {__fmul_rd(lo, lo), __fmul_ru(hi, hi), a.nan};
            return {0.0f, (-lo > hi) ? __fmul_ru(lo, lo) : __fmul_ru(hi, hi), a.nan};
        }
        case op::SQRT: {
            const bool u = a.nan || lo < 0.0f;
            if (bad || hi < 0) return {LF_QNAN, LF_QNAN, u};
            return {(lo > 0) ? __fsqrt_rd(lo) : 0.0f, __fsqrt_ru(hi), u};
        }
        case op::NEG:
            if (bad) return {LF_QNAN, LF_QNAN, a.nan};
            return {-hi, -lo, a.nan};
        case op::ABS:
            if (bad) return {LF_QNAN, LF_QNAN, a.nan};
            if (!(lo < 0)) return {lo, hi, a.nan};
            if (!(hi > 0)) return {-hi, -lo, a.nan};
            return {0.0f, sc_max(-lo, hi), a.nan};
        case op::RECIP: {
            // 1 / interval (Boost operator/(T, interval)); a zero-crossing
            // denominator maps to the half lines or the whole line.
            if (bad) return {LF_QNAN, LF_QNAN, a.nan};
            if (lo <= 0 && hi >= 0) {
                if (lo != 0) {
                    if (hi != 0) return {-LF_INF, LF_INF, a.nan};
                    return {-LF_INF, __fdiv_ru(1.0f, lo), a.nan};
                }
                if (hi != 0) return {__fdiv_rd(1.0f, hi), LF_INF, a.nan};
                return {LF_QNAN, LF_QNAN, a.nan};
            }
            return {__fdiv_rd(1.0f, hi), __fdiv_ru(1.0f, lo), a.nan};
        }
        case op::EXP:
            if (bad) return {LF_QNAN, LF_QNAN, a.nan};
            return {fmaxf(0.0f, ulp_down(expf(lo), LF_TRANSC_ULPS)),
                    ulp_up(expf(hi), LF_TRANSC_ULPS), a.nan};
        case op::LOG: {
            const bool u = a.nan || lo < 0.0f;
            if (bad || !(hi > 0)) return {LF_QNAN, LF_QNAN, u};
            const float l = !(lo > 0) ? -LF_INF : ulp_down(logf(lo), LF_TRANSC_ULPS);
            return {l, ulp_up(logf(hi), LF_TRANSC_ULPS), u};
        }
        case op::COS: {
            Iv r = iv_cos_bounds(lo, hi);
            r.nan = a.nan;
            return r;
        }
        case op::SIN: {
            // sin(x) = cos(x - pi/2) with pi/2 as an interval.
            if (bad) return {LF_QNAN, LF_QNAN, a.nan};
            const Iv s = iv_isub(lo, hi, pi_f_lo() * 0.5f, pi_f_hi() * 0.5f);
            Iv r = iv_cos_bounds(s.lo, s.hi);
            r.nan = a.nan;
            return r;
        }
        case op::TAN: {
            if (bad) return {LF_QNAN, LF_QNAN, a.nan};
            Iv t = iv_fmod(lo, hi, pi_f_lo(), pi_f_hi());
            const float half = pi_f_lo() * 0.5f;
            if (t.lo >= half) t = iv_isub(t.lo, t.hi, pi_f_lo(), pi_f_hi());
            if (t.lo <= -half || t.hi >= half) return {-LF_INF, LF_INF, a.nan};
            return {ulp_down(tanf(t.lo), LF_TRANSC_ULPS_WIDE),
                    ulp_up(tanf(t.hi), LF_TRANSC_ULPS_WIDE), a.nan};
        }
        case op::ASIN: {
            const bool u = a.nan || lo < -1.0f || hi > 1.0f;
            if (bad || hi < -1.0f || lo > 1.0f) return {LF_QNAN, LF_QNAN, u};
            const float half_hi = pi_f_hi() * 0.5f;
            const float l = (lo <= -1.0f) ? -half_hi : ulp_down(asinf(lo), LF_TRANSC_ULPS);
            const float h = (hi >= 1.0f) ? half_hi : ulp_up(asinf(hi), LF_TRANSC_ULPS);
            return {l, h, u};
        }
        case op::ACOS: {
            const bool u = a.nan || lo < -1.0f || hi > 1.0f;
            if (bad || hi < -1.0f || lo > 1.0f) return {LF_QNAN, LF_QNAN, u};
            const float l = (hi >= 1.0f) ? 0.0f : fmaxf(0.0f, ulp_down(acosf(hi), LF_TRANSC_ULPS));
            const float h = (lo <= -1.0f) ? pi_f_hi() : ulp_up(acosf(lo), LF_TRANSC_ULPS);
            return {l, h, u};
        }
        case op::ATAN: {
            if (isinf(lo) || isinf(hi)) {
                return {-1.57079637050628662109f, 1.57079637050628662109f, a.nan};
            }
            if (bad) return {LF_QNAN, LF_QNAN, a.nan};
            return {ulp_down(atanf(lo), LF_TRANSC_ULPS),
                    ulp_up(atanf(hi), LF_TRANSC_ULPS), a.nan};
        }
        case op::CONST_VAR:
        case OP_COPY:
            return a;
        default:
            return {LF_QNAN, LF_QNAN, true};
    }
}

__device__ __forceinline__ bool dev_is_binary(uint8_t o)
{
    return (o >= op::ADD && o <= op::NANFILL) || o == op::COMPARE;
}

__device__ __forceinline__ Iv iv_apply(uint8_t o, const Iv& a, const Iv& b)
{
    return dev_is_binary(o) ? iv_binary(o, a, b) : iv_unary(o, a);
}

/// Interval::state(): AMBIGUOUS when the value may be NaN.
enum : uint8_t { ST_EMPTY = 0, ST_FILLED = 1, ST_AMBIGUOUS = 2, ST_UNKNOWN = 3 };
__device__ __forceinline__ uint8_t iv_state(const Iv& a)
{
    if (a.nan) return ST_AMBIGUOUS;
    if (a.lo > 0) return ST_EMPTY;
    if (a.hi < 0) return ST_FILLED;
    return ST_AMBIGUOUS;
}

}  // namespace lfb
