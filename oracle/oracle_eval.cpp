// CPU oracle evaluators (TEST INFRASTRUCTURE ONLY; see oracle.hpp).
#include <algorithm>
#include <atomic>
#include <cfenv>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <unordered_set>

#include "oracle_eval.hpp"

#pragma STDC FENV_ACCESS ON

namespace ora {

////////////////////////////////////////////////////////////////////////////////
// Point semantics (eval_array.cpp:221-369)

static inline float fmin_std(float a, float b) { return (b < a) ? b : a; }   // std::min
static inline float fmax_std(float a, float b) { return (a < b) ? b : a; }   // std::max

////////////////////////////////////////////////////////////////////////////////
// Library calls of the point evaluators (sin, cos, tan, asin, acos, atan, exp,
// log).  By default they call the host C library.  For parity checks of whole
// tapes the caller can instead supply the results of another implementation
// (the GPU's) for given inputs: in record mode every (opcode, input) pair is
// collected; in replay mode results come from the supplied table, and inputs
// missing from it fall back to the C library, are counted and recorded, so a
// caller can iterate until nothing is missing.  Every other operation is
// exactly rounded, so with the same library results the oracle and the GPU
// must agree bit for bit.

static float host_libm(int op, float a)
{
    switch (op) {
        case OP_SIN: return sinf(a);
        case OP_COS: return cosf(a);
        case OP_TAN: return tanf(a);
        case OP_ASIN: return asinf(a);
        case OP_ACOS: return acosf(a);
        case OP_ATAN: return atanf(a);
        case OP_LOG: return logf(a);
        case OP_EXP: return expf(a);
    }
    return NAN;
}

namespace {
struct LibmHook {
    std::atomic<int> mode{0};   // 0 host, 1 record, 2 replay
    std::mutex mu;
    std::vector<std::unordered_set<uint64_t>*> sets;   // one per recording thread
    std::vector<uint64_t> keys;                        // replay table, sorted
    std::vector<uint32_t> vals;
    std::atomic<uint64_t> misses{0};
    std::atomic<uint64_t> generation{1};
};
LibmHook g_hook;

std::unordered_set<uint64_t>& record_set()
{
    thread_local std::unordered_set<uint64_t>* set = nullptr;
    thread_local uint64_t gen = 0;
    const uint64_t now = g_hook.generation.load();
    if (!set || gen != now) {
        std::lock_guard<std::mutex> lk(g_hook.mu);
        set = new std::unordered_set<uint64_t>();
        g_hook.sets.push_back(set);
        gen = now;
    }
    return *set;
}
}  // namespace

static float libm(int op, float a)
{
    const int mode = g_hook.mode.load(std::memory_order_relaxed);
    if (mode == 0) return host_libm(op, a);
    uint32_t bits;
    std::memcpy(&bits, &a, 4);
    const uint64_t key = (static_cast<uint64_t>(op) << 32) | bits;
    if (mode == 2) {
        auto it = std::lower_bound(g_hook.keys.begin(), g_hook.keys.end(), key);
        if (it != g_hook.keys.end() && *it == key) {
            float r;
            std::memcpy(&r, &g_hook.vals[it - g_hook.keys.begin()], 4);
            return r;
        }
        g_hook.misses.fetch_add(1, std::memory_order_relaxed);
    }
    record_set().insert(key);
    return host_libm(op, a);
}

// Mode changes and table updates must not overlap evaluations.
void libm_set_mode(int mode)
{
    std::lock_guard<std::mutex> lk(g_hook.mu);
    for (auto* s : g_hook.sets) delete s;
    g_hook.sets.clear();
    g_hook.generation.fetch_add(1);
    g_hook.misses = 0;
    g_hook.mode = mode;
}

void libm_set_table(const uint64_t* keys, const uint32_t* vals, uint64_t n)
{
    std::vector<std::pair<uint64_t, uint32_t>> kv(n);
    for (uint64_t i = 0; i < n; ++i) kv[i] = {keys[i], vals[i]};
    std::sort(kv.begin(), kv.end());
    g_hook.keys.resize(n);
    g_hook.vals.resize(n);
    for (uint64_t i = 0; i < n; ++i) {
        g_hook.keys[i] = kv[i].first;
        g_hook.vals[i] = kv[i].second;
    }
}

uint64_t libm_take(uint64_t* out, uint64_t max)
{
    std::lock_guard<std::mutex> lk(g_hook.mu);
    std::unordered_set<uint64_t> all;
    for (auto* s : g_hook.sets) all.insert(s->begin(), s->end());
    std::vector<uint64_t> v(all.begin(), all.end());
    std::sort(v.begin(), v.end());
    if (out) std::copy(v.begin(), v.begin() + std::min<uint64_t>(max, v.size()), out);
    return v.size();
}

uint64_t libm_misses() { return g_hook.misses.load(); }

float value_op(int op, float a, float b)
{
    switch (op) {
        case OP_ADD: return a + b;
        case OP_MUL: return a * b;
        case OP_MIN: return fmin_std(a, b);
        case OP_MAX: return fmax_std(a, b);
        case OP_SUB: return a - b;
        case OP_DIV: return a / b;
        case OP_ATAN2: return atan2f(a, b);
        case OP_POW: return powf(a, b);
        case OP_NTH_ROOT:
            if (a < 0) {
                // Boost nth_root of the point interval [a, a]: odd roots of a
                // negative number are negative, even roots are NaN.
                const int k = static_cast<int>(b);
                return (k & 1) ? -powf(-a, 1.0f / b) : NAN;
            }
            return powf(a, 1.0f / b);
        case OP_MOD: {
            float d = std::fabs(a / b);
            if ((a < 0) ^ (b < 0)) d = -std::ceil(d);
            else d = std::floor(d);
            const float bd = b * d;
            float out = a - bd;
            if ((b > 0 && out > b) || (b < 0 && out < b)) out = b;
            if ((b > 0.0f && out < 0.0f) || (b < 0.0f && out > 0.0f)) out = 0.0f;
            return out;
        }
        case OP_NANFILL: return std::isnan(a) ? b : a;
        case OP_COMPARE: return (a < b) ? -1.0f : (a > b) ? 1.0f : 0.0f;
        case OP_SQUARE: return a * a;
        case OP_SQRT: return std::sqrt(a);
        case OP_NEG: return -a;
        case OP_SIN: return libm(OP_SIN, a);
        case OP_COS: return libm(OP_COS, a);
        case OP_TAN: return libm(OP_TAN, a);
        case OP_ASIN: return libm(OP_ASIN, a);
        case OP_ACOS: return libm(OP_ACOS, a);
        case OP_ATAN: return libm(OP_ATAN, a);
        case OP_LOG: return libm(OP_LOG, a);
        case OP_EXP: return libm(OP_EXP, a);
        case OP_ABS: return std::fabs(a);
        case OP_RECIP: return 1.0f / a;
        case OP_CONST_VAR: return a;
    }
    return NAN;
}

// eval_deriv_array.cpp:119-256; `ov` is this clause's value.
void deriv_op(int op, float av, float bv, float ov, const float* ad,
              const float* bd, float* od, bool clear_vars)
{
    for (int k = 0; k < 3; ++k) {
        const float a = ad[k], b = bd ? bd[k] : 0.0f;
        float r = 0.0f;
        switch (op) {
            case OP_ADD: r = a + b; break;
            case OP_MUL: { const float p = b * av; const float q = a * bv; r = p + q; break; }
            case OP_MIN: r = (av < bv) ? a : b; break;
            case OP_MAX: r = (av < bv) ? b : a; break;
            case OP_SUB: r = a - b; break;
            case OP_DIV: {
                const float p = a * bv, q = b * av, den = bv * bv;
                r = (p - q) / den;
                break;
            }
            case OP_ATAN2: {
                const float p = a * bv, q = b * av;
                const float s1 = av * av, s2 = bv * bv;
                const float den = s1 + s2;
                r = (p - q) / den;
                break;
            }
            case OP_POW: {
                const float f = bv * powf(av, bv - 1);
                r = a * f;
                break;
            }
            case OP_NTH_ROOT: {
                const float f = powf(av, 1.0f / bv - 1) / bv;
                r = (a == 0) ? 0.0f : a * f;
                break;
            }
            case OP_MOD: r = a; break;
            case OP_NANFILL: r = std::isnan(av) ? b : a; break;
            case OP_COMPARE: r = 0.0f; break;
            case OP_SQUARE: { const float p = a * av; r = p * 2; break; }
            case OP_SQRT: {
                const float den = 2 * ov;
                r = (av < 0 || a == 0) ? 0.0f : a / den;
                break;
            }
            case OP_NEG: r = -a; break;
            case OP_SIN: r = a * libm(OP_COS, av); break;
            case OP_COS: r = a * -libm(OP_SIN, av); break;
            case OP_TAN: { const float s = 1 / libm(OP_COS, av); const float s2 = s * s; r = a * s2; break; }
            case OP_ASIN: { const float q = av * av; r = a / std::sqrt(1 - q); break; }
            case OP_ACOS: { const float q = av * av; r = a / -std::sqrt(1 - q); break; }
            case OP_ATAN: { const float q = av * av; r = a / (q + 1); break; }
            case OP_LOG: r = a / av; break;
            case OP_EXP: r = a * libm(OP_EXP, av); break;
            case OP_ABS: r = (av > 0) ? a : -a; break;
            case OP_RECIP: { const float q = av * av; r = a / -q; break; }
            case OP_CONST_VAR: r = clear_vars ? 0.0f : a; break;
            default: r = NAN;
        }
        od[k] = r;
    }
}

////////////////////////////////////////////////////////////////////////////////
// Directed rounding (Boost rounded_arith_std / rounded_transc_std restated
// with fesetround).

namespace rnd {
template <class F>
static inline float dn(F f)
{
    std::fesetround(FE_DOWNWARD);
    volatile float r = f();
    std::fesetround(FE_TONEAREST);
    return r;
}
template <class F>
static inline float up(F f)
{
    std::fesetround(FE_UPWARD);
    volatile float r = f();
    std::fesetround(FE_TONEAREST);
    return r;
}
static float add_dn(float a, float b) { return dn([&] { volatile float x = a, y = b; return x + y; }); }
static float add_up(float a, float b) { return up([&] { volatile float x = a, y = b; return x + y; }); }
static float sub_dn(float a, float b) { return dn([&] { volatile float x = a, y = b; return x - y; }); }
static float sub_up(float a, float b) { return up([&] { volatile float x = a, y = b; return x - y; }); }
static float mul_dn(float a, float b) { return dn([&] { volatile float x = a, y = b; return x * y; }); }
static float mul_up(float a, float b) { return up([&] { volatile float x = a, y = b; return x * y; }); }
static float div_dn(float a, float b) { return dn([&] { volatile float x = a, y = b; return x / y; }); }
static float div_up(float a, float b) { return up([&] { volatile float x = a, y = b; return x / y; }); }
static float sqrt_dn(float a) { return dn([&] { volatile float x = a; return std::sqrt(x); }); }
static float sqrt_up(float a) { return up([&] { volatile float x = a; return std::sqrt(x); }); }
static float int_dn(float a) { return dn([&] { volatile float x = a; return std::nearbyint(x); }); }
#define ORA_TRANSC(name, fn)                                                     \
    static float name##_dn(float a) { return dn([&] { volatile float x = a; return fn(x); }); } \
    static float name##_up(float a) { return up([&] { volatile float x = a; return fn(x); }); }
ORA_TRANSC(exp, expf)
ORA_TRANSC(log, logf)
ORA_TRANSC(cos, cosf)
ORA_TRANSC(tan, tanf)
ORA_TRANSC(asin, asinf)
ORA_TRANSC(acos, acosf)
ORA_TRANSC(atan, atanf)
#undef ORA_TRANSC
}  // namespace rnd

// Boost interval<float> with checking_base: invalid bounds mean empty,
// stored as [NaN, NaN].
BI BI::empty() { return {NAN, NAN}; }
BI BI::make(float l, float u)
{
    if (std::isnan(l) || std::isnan(u) || !(l <= u)) return empty();
    return {l, u};
}

static BI bi_add(BI x, BI y)
{
    if (x.bad() || y.bad()) return BI::empty();
    return {rnd::add_dn(x.lo, y.lo), rnd::add_up(x.hi, y.hi)};
}
static BI bi_sub(BI x, BI y)
{
    if (x.bad() || y.bad()) return BI::empty();
    return {rnd::sub_dn(x.lo, y.hi), rnd::sub_up(x.hi, y.lo)};
}
static BI bi_neg(BI x)
{
    if (x.bad()) return BI::empty();
    return {-x.hi, -x.lo};
}
static BI bi_mul(BI x, BI y)
{
    if (x.bad() || y.bad()) return BI::empty();
    const float xl = x.lo, xu = x.hi, yl = y.lo, yu = y.hi;
    using namespace rnd;
    if (xl < 0) {
        if (xu > 0) {
            if (yl < 0) {
                if (yu > 0) return {std::min(mul_dn(xl, yu), mul_dn(xu, yl)),
                                    std::max(mul_up(xl, yl), mul_up(xu, yu))};
                return {mul_dn(xu, yl), mul_up(xl, yl)};
            }
            if (yu > 0) return {mul_dn(xl, yu), mul_up(xu, yu)};
            return {0, 0};
        }
        if (yl < 0) {
            if (yu > 0) return {mul_dn(xl, yu), mul_up(xl, yl)};
            return {mul_dn(xu, yu), mul_up(xl, yl)};
        }
        if (yu > 0) return {mul_dn(xl, yu), mul_up(xu, yl)};
        return {0, 0};
    }
    if (xu > 0) {
        if (yl < 0) {
            if (yu > 0) return {mul_dn(xu, yl), mul_up(xu, yu)};
            return {mul_dn(xu, yl), mul_up(xl, yu)};
        }
        if (yu > 0) return {mul_dn(xl, yl), mul_up(xu, yu)};
        return {0, 0};
    }
    return {0, 0};
}
static BI bi_smul(float x, BI y)   // scalar * interval
{
    if (std::isnan(x) || y.bad()) return BI::empty();
    if (x < 0) return {rnd::mul_dn(x, y.hi), rnd::mul_up(x, y.lo)};
    if (x == 0) return {0, 0};
    return {rnd::mul_dn(x, y.lo), rnd::mul_up(x, y.hi)};
}
static BI bi_div_nonzero(BI x, BI y)
{
    const float xl = x.lo, xu = x.hi, yl = y.lo, yu = y.hi;
    using namespace rnd;
    if (xu < 0) {
        if (yu < 0) return {div_dn(xu, yl), div_up(xl, yu)};
        return {div_dn(xl, yl), div_up(xu, yu)};
    } else if (xl < 0) {
        if (yu < 0) return {div_dn(xu, yu), div_up(xl, yu)};
        return {div_dn(xl, yl), div_up(xu, yl)};
    }
    if (yu < 0) return {div_dn(xu, yu), div_up(xl, yl)};
    return {div_dn(xl, yu), div_up(xu, yl)};
}
static BI bi_div(BI x, BI y)   // interval / interval
{
    if (x.bad() || y.bad()) return BI::empty();
    const bool zero_in = !(y.lo > 0) && !(y.hi < 0);
    if (zero_in) {
        if (y.lo != 0) {
            if (y.hi != 0) return {-INFINITY, INFINITY};
            // div_negative
            if (x.lo == 0 && x.hi == 0) return x;
            if (x.hi < 0) return {rnd::div_dn(x.hi, y.lo), INFINITY};
            if (x.lo < 0) return {-INFINITY, INFINITY};
            return {-INFINITY, rnd::div_up(x.lo, y.lo)};
        }
        if (y.hi != 0) {
            // div_positive
            if (x.lo == 0 && x.hi == 0) return x;
            if (x.hi < 0) return {-INFINITY, rnd::div_up(x.hi, y.hi)};
            if (x.lo < 0) return {-INFINITY, INFINITY};
            return {rnd::div_dn(x.lo, y.hi), INFINITY};
        }
        return BI::empty();
    }
    return bi_div_nonzero(x, y);
}
static BI bi_recip(BI y)   // 1 / interval
{
    if (y.bad()) return BI::empty();
    const bool zero_in = !(y.lo > 0) && !(y.hi < 0);
    if (zero_in) {
        if (y.lo != 0) {
            if (y.hi != 0) return {-INFINITY, INFINITY};
            return {-INFINITY, rnd::div_up(1.0f, y.lo)};
        }
        if (y.hi != 0) return {rnd::div_dn(1.0f, y.hi), INFINITY};
        return BI::empty();
    }
    return {rnd::div_dn(1.0f, y.hi), rnd::div_up(1.0f, y.lo)};
}
static BI bi_min(BI x, BI y)
{
    if (x.bad() || y.bad()) return BI::empty();
    return {std::min(x.lo, y.lo), std::min(x.hi, y.hi)};
}
static BI bi_max(BI x, BI y)
{
    if (x.bad() || y.bad()) return BI::empty();
    return {std::max(x.lo, y.lo), std::max(x.hi, y.hi)};
}
static BI bi_hull(BI x, BI y)
{
    const bool bx = x.bad(), by = y.bad();
    if (bx) return by ? BI::empty() : y;
    if (by) return x;
    return {std::min(x.lo, y.lo), std::max(x.hi, y.hi)};
}
static BI bi_square(BI x)
{
    if (x.bad()) return BI::empty();
    if (x.hi < 0) return {rnd::mul_dn(x.hi, x.hi), rnd::mul_up(x.lo, x.lo)};
    if (x.lo > 0) return {rnd::mul_dn(x.lo, x.lo), rnd::mul_up(x.hi, x.hi)};
    return {0, (-x.lo > x.hi) ? rnd::mul_up(x.lo, x.lo) : rnd::mul_up(x.hi, x.hi)};
}
static BI bi_sqrt(BI x)
{
    if (x.bad() || x.hi < 0) return BI::empty();
    return {(x.lo > 0) ? rnd::sqrt_dn(x.lo) : 0.0f, rnd::sqrt_up(x.hi)};
}
static BI bi_abs(BI x)
{
    if (x.bad()) return BI::empty();
    if (!(x.lo < 0)) return x;
    if (!(x.hi > 0)) return {-x.hi, -x.lo};
    return {0, std::max(-x.lo, x.hi)};
}
static const float PI_L = 13176794.0f / (1 << 22);
static const float PI_U = 13176795.0f / (1 << 22);
static BI bi_fmod(BI x, BI y)
{
    if (x.bad() || y.bad()) return BI::empty();
    const float yb = (x.lo < 0) ? y.lo : y.hi;
    const float n = rnd::int_dn(rnd::div_dn(x.lo, yb));
    return bi_sub(x, bi_smul(n, y));
}
static BI bi_cos(BI x)
{
    if (x.bad()) return BI::empty();
    const BI pi2 = {PI_L * 2, PI_U * 2};
    BI tmp = bi_fmod(x, pi2);
    if (rnd::sub_up(tmp.hi, tmp.lo) >= pi2.lo) return {-1, 1};
    if (tmp.lo >= PI_U) return bi_neg(bi_cos(bi_sub(tmp, BI{PI_L, PI_U})));
    const float l = tmp.lo, u = tmp.hi;
    if (u <= PI_L) return {rnd::cos_dn(u), rnd::cos_up(l)};
    if (u <= pi2.lo) return {-1, rnd::cos_up(std::min(rnd::sub_dn(pi2.lo, u), l))};
    return {-1, 1};
}
static BI bi_sin(BI x)
{
    if (x.bad()) return BI::empty();
    return bi_cos(bi_sub(x, BI{PI_L / 2, PI_U / 2}));
}
static BI bi_tan(BI x)
{
    if (x.bad()) return BI::empty();
    BI tmp = bi_fmod(x, BI{PI_L, PI_U});
    const float half = PI_L / 2;
    if (tmp.lo >= half) tmp = bi_sub(tmp, BI{PI_L, PI_U});
    if (tmp.lo <= -half || tmp.hi >= half) return {-INFINITY, INFINITY};
    return {rnd::tan_dn(tmp.lo), rnd::tan_up(tmp.hi)};
}
static int ipow_bits(int p) { return p; }
static float pow_dn(float x, int p)
{
    float y = (p & 1) ? x : 1.0f;
    p >>= 1;
    while (p > 0) {
        x = rnd::mul_dn(x, x);
        if (p & 1) y = rnd::mul_dn(x, y);
        p >>= 1;
    }
    return y;
}
static float pow_up(float x, int p)
{
    float y = (p & 1) ? x : 1.0f;
    p >>= 1;
    while (p > 0) {
        x = rnd::mul_up(x, x);
        if (p & 1) y = rnd::mul_up(x, y);
        p >>= 1;
    }
    return y;
}
static BI bi_ipow(BI x, int pwr)
{
    if (x.bad()) return BI::empty();
    if (pwr == 0) {
        if (x.lo == 0 && x.hi == 0) return BI::empty();
        return {1, 1};
    }
    if (pwr < 0) return bi_recip(bi_ipow(x, -pwr));
    const int p = ipow_bits(pwr);
    if (x.hi < 0) {
        const float yl = pow_dn(-x.hi, p), yu = pow_up(-x.lo, p);
        return (p & 1) ? BI{-yu, -yl} : BI{yl, yu};
    }
    if (x.lo < 0) {
        if (p & 1) return {-pow_up(-x.lo, p), pow_up(x.hi, p)};
        return {0, pow_up(std::max(-x.lo, x.hi), p)};
    }
    return {pow_dn(x.lo, p), pow_up(x.hi, p)};
}

// Interval (interval.hpp:31-442)
static Iv iv_point(float f)
{
    return {BI::make(f, f), std::isnan(f)};
}

Iv iv_make(float lo, float hi)
{
    return {BI::make(lo, hi), std::isnan(lo) || std::isnan(hi)};
}

static Iv iv_op(int op, const Iv& a, const Iv& b)
{
    const float al = a.i.lo, au = a.i.hi, bl = b.i.lo, bu = b.i.hi;
    switch (op) {
        case OP_ADD:
            return {bi_add(a.i, b.i), a.nan || b.nan ||
                    (al == -INFINITY && bu == INFINITY) ||
                    (bl == -INFINITY && au == INFINITY)};
        case OP_MUL:
            return {bi_mul(a.i, b.i), a.nan || b.nan ||
                    ((al == -INFINITY || au == INFINITY) && bl <= 0.0f && bu >= 0.0f) ||
                    ((bl == -INFINITY || bu == INFINITY) && al <= 0.0f && au >= 0.0f)};
        case OP_MIN: {
            BI r = bi_min(a.i, b.i);
            if (b.nan) r = bi_hull(r, a.i);
            return {r, a.nan};
        }
        case OP_MAX: {
            BI r = bi_max(a.i, b.i);
            if (b.nan) r = bi_hull(r, a.i);
            return {r, a.nan};
        }
        case OP_SUB:
            return {bi_sub(a.i, b.i), a.nan || b.nan ||
                    (al == -INFINITY && bl == -INFINITY) ||
                    (au == -INFINITY && bu == -INFINITY)};
        case OP_DIV: {
            const BI r = (bl <= 0.0f && bu >= 0.0f) ? BI{-INFINITY, INFINITY}
                                                   : bi_div(a.i, b.i);
            return {r, a.nan || b.nan ||
                    ((al == -INFINITY || au == INFINITY) &&
                     (bl == -INFINITY || bu == INFINITY)) ||
                    (al <= 0.0f && au >= 0.0f && bl <= 0.0f && bu >= 0.0f)};
        }
        case OP_ATAN2: {
            const BI& y = a.i;
            const BI& x = b.i;
            const bool u = a.nan || b.nan ||
                (x.lo <= 0.0f && x.hi >= 0.0f && y.lo <= 0.0f && y.hi >= 0.0f);
            auto at = [](float p, float q) { return atan2f(p, q); };
            const float PI = static_cast<float>(M_PI);
            if (x.lo > 0) {
                if (y.lo > 0) return {BI::make(at(y.lo, x.hi), at(y.hi, x.lo)), u};
                if (y.hi < 0) return {BI::make(at(y.lo, x.lo), at(y.hi, x.hi)), u};
                return {BI::make(at(y.lo, x.lo), at(y.hi, x.lo)), u};
            } else if (x.hi < 0) {
                if (y.lo > 0) return {BI::make(at(y.hi, x.hi), at(y.lo, x.lo)), u};
                if (y.hi < 0) return {BI::make(at(y.hi, x.lo), at(y.lo, x.hi)), u};
                return {BI::make(-PI, PI), u};
            }
            if (y.lo > 0) return {BI::make(at(y.lo, x.hi), at(y.lo, x.lo)), u};
            if (y.hi < 0) return {BI::make(at(y.hi, x.lo), at(y.hi, x.hi)), u};
            return {BI::make(-PI, PI), u};
        }
        case OP_POW: {
            const int p = static_cast<int>(bl);
            const bool a_zero = al <= 0.0f && au >= 0.0f;
            return {bi_ipow(a.i, p), a.nan || b.nan || (a_zero && p == 0)};
        }
        case OP_NTH_ROOT: {
            const int k = static_cast<int>(bl);
            const bool u = a.nan || b.nan || (al <= 0.0f && !(k & 2));
            if (a.i.bad() || k <= 0) return {BI::empty(), u};
            if (k == 1) return {a.i, u};
            const float inv = 1.0f / k;
            auto up = [&](float x) { return nextafterf(powf(x, inv), INFINITY); };
            auto dn = [&](float x) { return nextafterf(powf(x, inv), -INFINITY); };
            if (!(au > 0)) {
                if (au == 0) {
                    if (!(k & 1) || al == 0) return {BI{0, 0}, u};
                    return {BI{-up(-al), 0}, u};
                }
                if (!(k & 1)) return {BI::empty(), u};
                return {BI{-up(-al), -dn(-au)}, u};
            }
            const float hi = up(au);
            if (!(al > 0)) {
                if (!(k & 1) || al == 0) return {BI{0, hi}, u};
                return {BI{-up(-al), hi}, u};
            }
            return {BI{std::max(0.0f, dn(al)), hi}, u};
        }
        case OP_MOD: {
            BI out = BI::make(std::fmin(bl, 0.0f), std::fmax(0.0f, bu));
            if (std::isfinite(au) && std::isfinite(al)) {
                const int position = (bu >= 0.0f) + 2 * (bl <= 0.0f);
                BI usedA = a.i;
                if (position == 2) usedA = bi_smul(-1.0f, usedA);
                if (position == 1 || position == 2) {
                    const BI absB = bi_abs(b.i);
                    const BI q = bi_div(usedA, absB);
                    const int qi = static_cast<int>(std::floor(q.lo));
                    if (qi == static_cast<int>(std::floor(q.hi))) {
                        out = bi_sub(a.i, bi_smul(static_cast<float>(qi), b.i));
                    }
                } else if (position == 0) {
                    out = BI::empty();
                }
            }
            return {out, bu >= 0.0f && bl <= 0.0f};
        }
        case OP_NANFILL:
            if (a.nan) return {bi_hull(a.i, b.i), b.nan};
            return {a.i, false};
        case OP_COMPARE:
            if (au < bl) return {BI{-1, -1}, false};
            if (al > bu) return {BI{1, 1}, false};
            return {BI{-1, 1}, false};
        case OP_SQUARE: return {bi_square(a.i), a.nan};
        case OP_SQRT: return {bi_sqrt(a.i), a.nan || al < 0.0f};
        case OP_NEG: return {bi_neg(a.i), a.nan};
        case OP_SIN: return {bi_sin(a.i), a.nan};
        case OP_COS: return {bi_cos(a.i), a.nan};
        case OP_TAN: return {bi_tan(a.i), a.nan};
        case OP_ASIN: {
            const bool u = a.nan || al < -1.0f || au > 1.0f;
            if (a.i.bad() || au < -1.0f || al > 1.0f) return {BI::empty(), u};
            const float hu = PI_U / 2;
            return {BI{(al <= -1.0f) ? -hu : rnd::asin_dn(al),
                       (au >= 1.0f) ? hu : rnd::asin_up(au)}, u};
        }
        case OP_ACOS: {
            const bool u = a.nan || al < -1.0f || au > 1.0f;
            if (a.i.bad() || au < -1.0f || al > 1.0f) return {BI::empty(), u};
            return {BI{(au >= 1.0f) ? 0.0f : rnd::acos_dn(au),
                       (al <= -1.0f) ? PI_U : rnd::acos_up(al)}, u};
        }
        case OP_ATAN: {
            if (std::isinf(al) || std::isinf(au)) {
                return {BI{static_cast<float>(-M_PI / 2), static_cast<float>(M_PI / 2)}, a.nan};
            }
            if (a.i.bad()) return {BI::empty(), a.nan};
            return {BI{rnd::atan_dn(al), rnd::atan_up(au)}, a.nan};
        }
        case OP_EXP:
            if (a.i.bad()) return {BI::empty(), a.nan};
            return {BI{rnd::exp_dn(al), rnd::exp_up(au)}, a.nan};
        case OP_LOG: {
            const bool u = a.nan || al < 0.0f;
            if (a.i.bad() || !(au > 0)) return {BI::empty(), u};
            return {BI{!(al > 0) ? -INFINITY : rnd::log_dn(al), rnd::log_up(au)}, u};
        }
        case OP_ABS: return {bi_abs(a.i), a.nan};
        case OP_RECIP: return {bi_recip(a.i), a.nan};
        case OP_CONST_VAR: return a;
    }
    return {BI::empty(), true};
}

////////////////////////////////////////////////////////////////////////////////
// Evaluator

Evaluator::Evaluator(const Tape& base_)
    : base(std::make_shared<Tape>(base_))
{
    const size_t n = base->num_clauses + 1;
    v.assign(n * NB, 0.0f);
    d.assign(n * 3 * NB, 0.0f);
    iv.assign(n, Iv{BI{0, 0}, false});
    disabled.assign(n, 0);
    remap.assign(n, 0);
    for (auto& c : base->constants) {
        std::fill(v.begin() + c.first * NB, v.begin() + (c.first + 1) * NB, c.second);
        iv[c.first] = iv_point(c.second);
    }
    for (auto& var : base->vars) {
        std::fill(v.begin() + var.first * NB, v.begin() + (var.first + 1) * NB, var.second);
        iv[var.first] = iv_point(var.second);
    }
    float* dxp = &d[(base->X * 3 + 0) * NB];
    float* dyp = &d[(base->Y * 3 + 1) * NB];
    float* dzp = &d[(base->Z * 3 + 2) * NB];
    std::fill(dxp, dxp + NB, 1.0f);
    std::fill(dyp, dyp + NB, 1.0f);
    std::fill(dzp, dzp + NB, 1.0f);
    base->terminal = true;
    for (auto& c : base->t) {
        if (c.op == OP_MIN || c.op == OP_MAX) base->terminal = false;
    }
}

void Evaluator::set(float x, float y, float z, int i)
{
    v[base->X * NB + i] = x;
    v[base->Y * NB + i] = y;
    v[base->Z * NB + i] = z;
}

const float* Evaluator::values(int count, const Tape& tape)
{
    for (auto it = tape.t.rbegin(); it != tape.t.rend(); ++it) {
        float* out = &v[it->id * NB];
        const float* a = &v[it->a * NB];
        const float* b = &v[it->b * NB];
        const int op = it->op;
        for (int i = 0; i < count; ++i) {
            out[i] = value_op(op, a[i], b[i]);
        }
    }
    return &v[tape.root * NB];
}

void Evaluator::derivs(int count, const Tape& tape, float* out4)
{
    const float* vals = values(count, tape);
    for (int i = 0; i < count; ++i) out4[4 * i + 3] = vals[i];
    for (auto it = tape.t.rbegin(); it != tape.t.rend(); ++it) {
        const int op = it->op;
        const bool unary = op_arity(op) == 1;
        for (int i = 0; i < count; ++i) {
            float ad[3], bd[3], od[3];
            for (int k = 0; k < 3; ++k) {
                ad[k] = d[(it->a * 3 + k) * NB + i];
                bd[k] = unary ? 0.0f : d[(it->b * 3 + k) * NB + i];
            }
            deriv_op(op, v[it->a * NB + i], unary ? 0.0f : v[it->b * NB + i],
                     v[it->id * NB + i], ad, bd, od, clear_vars);
            for (int k = 0; k < 3; ++k) d[(it->id * 3 + k) * NB + i] = od[k];
        }
    }
    for (int i = 0; i < count; ++i) {
        for (int k = 0; k < 3; ++k) out4[4 * i + k] = d[(tape.root * 3 + k) * NB + i];
    }
}

void Evaluator::ambiguous(int count, const Tape& tape, bool* out)
{
    for (int i = 0; i < count; ++i) out[i] = false;
    for (auto it = tape.t.rbegin(); it != tape.t.rend(); ++it) {
        if (it->op == OP_MIN || it->op == OP_MAX) {
            for (int i = 0; i < count; ++i) {
                out[i] = out[i] || (v[it->a * NB + i] == v[it->b * NB + i]);
            }
        }
    }
}

Iv Evaluator::interval(float xl, float yl, float zl, float xu, float yu,
                       float zu, const Tape& tape)
{
    iv[base->X] = iv_make(xl, xu);
    iv[base->Y] = iv_make(yl, yu);
    iv[base->Z] = iv_make(zl, zu);
    for (auto it = tape.t.rbegin(); it != tape.t.rend(); ++it) {
        iv[it->id] = iv_op(it->op, iv[it->a], iv[it->b]);
    }
    return iv[tape.root];
}

// Tape::push (tape.cpp:23-160).
std::shared_ptr<Tape> Evaluator::push(const std::shared_ptr<Tape>& tape,
                                      const KeepFn& fn, int type)
{
    if (tape->terminal) return tape;
    std::fill(disabled.begin(), disabled.end(), 1);
    std::fill(remap.begin(), remap.end(), 0);
    disabled[tape->root] = 0;
    bool terminal = true;
    bool changed = false;
    for (const auto& c : tape->t) {
        if (!disabled[c.id]) {
            switch (fn(c.op, c.id, c.a, c.b)) {
                case KEEP_A: disabled[c.a] = 0; remap[c.id] = c.a; changed = true; break;
                case KEEP_B: disabled[c.b] = 0; remap[c.id] = c.b; changed = true; break;
                case KEEP_BOTH: terminal = false; break;
                case KEEP_ALWAYS: break;
            }
            if (remap[c.id]) {
                disabled[c.id] = 1;
            } else {
                disabled[c.a] = 0;
                disabled[c.b] = 0;
            }
        }
    }
    if (!changed) return tape;
    auto out = std::make_shared<Tape>();
    out->type = type;
    out->parent = tape.get();
    out->parent_keep = tape;
    out->terminal = terminal;
    out->X = tape->X; out->Y = tape->Y; out->Z = tape->Z;
    out->num_clauses = tape->num_clauses;
    for (const auto& c : tape->t) {
        if (!disabled[c.id]) {
            uint32_t ra = c.a, rb = c.b;
            while (remap[ra]) ra = remap[ra];
            while (remap[rb]) rb = remap[rb];
            out->t.push_back({c.op, c.id, ra, rb});
        }
    }
    out->root = tape->root;
    while (remap[out->root]) out->root = remap[out->root];
    return out;
}

// IntervalEvaluator::push (eval_interval.cpp:116-167): uses the results of
// the most recent interval() call.
std::shared_ptr<Tape> Evaluator::push_interval(const std::shared_ptr<Tape>& tape)
{
    auto out = push(tape, [&](int op, uint32_t, uint32_t a, uint32_t b) {
        if (op == OP_MAX) {
            if (a == b) return KEEP_A;
            if (iv[a].i.lo > iv[b].i.hi) return KEEP_A;
            if (iv[b].i.lo > iv[a].i.hi) return KEEP_B;
            return KEEP_BOTH;
        } else if (op == OP_MIN) {
            if (a == b) return KEEP_A;
            if (iv[a].i.lo > iv[b].i.hi) return KEEP_B;
            if (iv[b].i.lo > iv[a].i.hi) return KEEP_A;
            return KEEP_BOTH;
        }
        return KEEP_ALWAYS;
    }, 1);
    if (out != tape) {
        out->bx[0] = iv[base->X].i.lo; out->bx[1] = iv[base->X].i.hi;
        out->by[0] = iv[base->Y].i.lo; out->by[1] = iv[base->Y].i.hi;
        out->bz[0] = iv[base->Z].i.lo; out->bz[1] = iv[base->Z].i.hi;
    }
    return out;
}

// ArrayEvaluator::valueAndPush (eval_array.cpp:127-170), slot 0.
std::shared_ptr<Tape> Evaluator::value_and_push(float x, float y, float z,
                                                const std::shared_ptr<Tape>& tape,
                                                float* value)
{
    set(x, y, z, 0);
    *value = values(1, *tape)[0];
    return push(tape, [&](int op, uint32_t, uint32_t a, uint32_t b) {
        const float va = v[a * NB], vb = v[b * NB];
        if (op == OP_MAX) {
            if (va > vb) return KEEP_A;
            if (vb > va) return KEEP_B;
            return KEEP_BOTH;
        } else if (op == OP_MIN) {
            if (va > vb) return KEEP_B;
            if (vb > va) return KEEP_A;
            return KEEP_BOTH;
        }
        return KEEP_ALWAYS;
    }, 2);
}

// Tape::getBase(point) (tape.cpp:188-209).
const Tape* get_base(const Tape* tape, float x, float y, float z)
{
    while (tape->parent) {
        if (tape->type == 1 && x >= tape->bx[0] && x <= tape->bx[1] &&
            y >= tape->by[0] && y <= tape->by[1] && z >= tape->bz[0] &&
            z <= tape->bz[1]) {
            break;
        }
        tape = tape->parent;
    }
    return tape;
}

////////////////////////////////////////////////////////////////////////////////
// Features (feature.cpp:14-284, eval_feature.cpp:56-372)

static float dot3(const Vec3& a, const Vec3& b)
{
    const float p0 = a.x[0] * b.x[0], p1 = a.x[1] * b.x[1], p2 = a.x[2] * b.x[2];
    return (p0 + p1) + p2;
}
static float norm3(const Vec3& a) { return std::sqrt(dot3(a, a)); }

bool Feature::check(const Vec3& e, bool* dup) const
{
    for (const auto& i : eps) {
        if (static_cast<double>(dot3(e, i)) > 1 - 1e-8) {
            if (dup) *dup = true;
            return true;
        }
    }
    if (eps.empty()) return true;
    if (eps.size() == 1) return dot3(e, eps.front()) != -1;

    std::vector<Vec3> es = eps;
    es.push_back(e);
    std::vector<std::pair<Vec3, float>> planes;
    for (const auto& q : es) planes.push_back({q, 0.0f});
    const float axes[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0},
                              {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (auto& a : axes) planes.push_back({Vec3{{a[0], a[1], a[2]}}, 1.0f});

    std::vector<Vec3> corners;
    for (size_t i = 0; i < planes.size(); ++i) {
        for (size_t j = i; j < planes.size(); ++j) {
            for (size_t k = j; k < planes.size(); ++k) {
                const auto& A = planes[i];
                const auto& B = planes[j];
                const auto& C = planes[k];
                if (A.second == 0.0 && B.second == 0.0 && C.second == 0.0) continue;
                // M = [A B C] as columns (Eigen comma initializer of vectors)
                float m[3][3];
                for (int r = 0; r < 3; ++r) {
                    m[r][0] = A.first.x[r];
                    m[r][1] = B.first.x[r];
                    m[r][2] = C.first.x[r];
                }
                // Eigen's 3x3 determinant: cofactor expansion along row 0
                auto det3h = [&](int a, int b, int c) {
                    const float p = m[1][b] * m[2][c];
                    const float q = m[1][c] * m[2][b];
                    return m[0][a] * (p - q);
                };
                const float det = (det3h(0, 1, 2) - det3h(1, 0, 2)) + det3h(2, 0, 1);
                if (std::fabs(det) < 1e-6) continue;
                // Eigen's 3x3 inverse via cofactors
                auto cof = [&](int i_, int j_) {
                    const int i1 = (i_ + 1) % 3, i2 = (i_ + 2) % 3;
                    const int j1 = (j_ + 1) % 3, j2 = (j_ + 2) % 3;
                    const float p = m[i1][j1] * m[i2][j2];
                    const float q = m[i1][j2] * m[i2][j1];
                    return p - q;
                };
                const float c00 = cof(0, 0), c10 = cof(1, 0), c20 = cof(2, 0);
                const float dd = (c00 * m[0][0] + c10 * m[1][0]) + c20 * m[2][0];
                const float inv = 1.0f / dd;
                float mi[3][3];
                for (int jj = 0; jj < 3; ++jj) {
                    for (int ii = 0; ii < 3; ++ii) {
                        mi[ii][jj] = cof(jj, ii) * inv;
                    }
                }
                const float dv[3] = {A.second, B.second, C.second};
                Vec3 vert;
                for (int r = 0; r < 3; ++r) {
                    const float p0 = mi[r][0] * dv[0], p1 = mi[r][1] * dv[1],
                                p2 = mi[r][2] * dv[2];
                    vert.x[r] = (p0 + p1) + p2;
                }
                bool duplicate = false;
                for (const auto& c : corners) {
                    if (c.x[0] == vert.x[0] && c.x[1] == vert.x[1] && c.x[2] == vert.x[2]) {
                        duplicate = true;
                        break;
                    }
                }
                if (!duplicate) corners.push_back(vert);
            }
        }
    }
    for (const auto& c : corners) {
        bool okay = true;
        for (const auto& q : es) {
            if (dot3(c, q) <= 0) { okay = false; break; }
        }
        if (okay) return true;
    }
    for (const auto& c : corners) {
        for (const auto& dd : corners) {
            Vec3 p;
            for (int r = 0; r < 3; ++r) p.x[r] = (c.x[r] + dd.x[r]) / 2.0f;
            bool okay = true;
            for (const auto& q : es) {
                if (dot3(p, q) <= 0) { okay = false; break; }
            }
            if (okay) return true;
        }
    }
    return false;
}

bool Feature::push(const Vec3& e_)
{
    const float n = norm3(e_);
    if (n == 0) return false;
    Vec3 e;
    for (int r = 0; r < 3; ++r) e.x[r] = e_.x[r] / n;
    bool dup = false;
    if (check(e, &dup)) {
        if (!dup) eps.push_back(e);
        return true;
    }
    return false;
}

bool Feature::push_all(const Feature& other)
{
    for (const auto& e : other.eps) {
        if (!push(e)) return false;
    }
    return true;
}

static int vcmp(const Vec3& a, const Vec3& b)
{
    for (int i = 0; i < 3; ++i) {
        if (a.x[i] < b.x[i]) return -1;
        if (a.x[i] > b.x[i]) return 1;
    }
    return 0;
}

bool feature_less(const Feature& a, const Feature& b)
{
    size_t i = 0;
    for (; i < a.eps.size() && i < b.eps.size(); ++i) {
        const int c = vcmp(a.eps[i], b.eps[i]);
        if (c != 0) return c < 0;
    }
    if (i < a.eps.size()) return false;
    if (i < b.eps.size()) return true;
    return vcmp(a.deriv, b.deriv) < 0;
}

static bool same_eps(const Feature& a, const Feature& b)
{
    if (a.eps.size() != b.eps.size()) return false;
    for (size_t i = 0; i < a.eps.size(); ++i) {
        if (vcmp(a.eps[i], b.eps[i]) != 0) return false;
    }
    return true;
}

std::vector<Feature> Evaluator::feature_lists(const Tape& tape, uint32_t* root)
{
    // f[slot] for every slot used by the tape
    std::vector<std::vector<Feature>> f(base->num_clauses + 1);
    auto single = [](float x, float y, float z) {
        Feature ft;
        ft.deriv = Vec3{{x, y, z}};
        return std::vector<Feature>{ft};
    };
    f[base->X] = single(1, 0, 0);
    f[base->Y] = single(0, 1, 0);
    f[base->Z] = single(0, 0, 1);
    for (auto& var : base->vars) f[var.first] = single(0, 0, 0);
    for (auto& c : base->constants) f[c.first] = single(0, 0, 0);

    for (auto it = tape.t.rbegin(); it != tape.t.rend(); ++it) {
        const int op = it->op;
        const uint32_t a = it->a, b = it->b;
        std::vector<Feature> of;
        const float av = v[a * NB], bv = v[b * NB], ov = v[it->id * NB];
        if (op == OP_MIN || op == OP_MAX) {
            const bool is_min = op == OP_MIN;
            if (av < bv || a == b) {
                of = is_min ? f[a] : f[b];
            } else if (av > bv) {
                of = is_min ? f[b] : f[a];
            } else {
                for (const auto& fa : f[a]) {
                    for (const auto& fb : f[b]) {
                        Vec3 eps;
                        for (int k = 0; k < 3; ++k) {
                            eps.x[k] = is_min ? fb.deriv.x[k] - fa.deriv.x[k]
                                              : fa.deriv.x[k] - fb.deriv.x[k];
                        }
                        if (norm3(eps) == 0) {
                            if (!fa.eps.empty()) of.push_back(fa);
                            if (!fb.eps.empty()) of.push_back(fb);
                            if (fa.eps.empty() && fb.eps.empty()) of.push_back(fa);
                        } else {
                            Feature combined = fa;
                            if (combined.push_all(fb)) {
                                Feature ffa = combined;
                                ffa.deriv = fa.deriv;
                                if (ffa.push(eps)) of.push_back(ffa);
                                Feature ffb = combined;
                                ffb.deriv = fb.deriv;
                                Vec3 neg;
                                for (int k = 0; k < 3; ++k) neg.x[k] = -eps.x[k];
                                if (ffb.push(neg)) of.push_back(ffb);
                            }
                        }
                    }
                }
            }
        } else if (op_arity(op) == 1) {
            for (const auto& fa : f[a]) {
                Feature nf;
                deriv_op(op, av, 0.0f, ov, fa.deriv.x, nullptr, nf.deriv.x, false);
                nf.eps = fa.eps;
                of.push_back(nf);
            }
        } else {
            for (const auto& fa : f[a]) {
                for (const auto& fb : f[b]) {
                    Feature nf;
                    deriv_op(op, av, bv, ov, fa.deriv.x, fb.deriv.x, nf.deriv.x, false);
                    nf.eps = fa.eps;
                    for (const auto& e : fb.eps) {
                        bool found = false;
                        for (const auto& e2 : nf.eps) {
                            if (vcmp(e, e2) == 0) { found = true; break; }
                        }
                        if (!found) nf.eps.push_back(e);
                    }
                    of.push_back(nf);
                }
            }
        }
        if (of.size() > 1) {
            std::sort(of.begin(), of.end(), feature_less);
            std::vector<Feature> uniq;
            for (const auto& ft : of) {
                if (!uniq.empty()) {
                    const Feature& last = uniq.back();
                    Vec3 dd;
                    for (int k = 0; k < 3; ++k) dd.x[k] = ft.deriv.x[k] - last.deriv.x[k];
                    if (dot3(dd, dd) <= 1e-10 && same_eps(ft, last)) continue;
                }
                uniq.push_back(ft);
            }
            of.swap(uniq);
            const Vec3 first = of.front().deriv;
            bool all_same = true;
            for (const auto& ft : of) {
                Vec3 dd;
                for (int k = 0; k < 3; ++k) dd.x[k] = ft.deriv.x[k] - first.x[k];
                if (!(dot3(dd, dd) < 1e-10)) { all_same = false; break; }
            }
            if (all_same) {
                Feature one;
                one.deriv = first;
                of = {one};
            }
        }
        f[it->id] = std::move(of);
    }
    *root = tape.root;
    return f[tape.root];
}

bool Evaluator::is_inside(float x, float y, float z, const std::shared_ptr<Tape>& tape)
{
    float value;
    auto t = value_and_push(x, y, z, tape, &value);
    if (value < 0) return true;
    if (value > 0) return false;
    uint32_t root;
    const auto fs = feature_lists(*t, &root);
    if (fs.size() == 1) return norm3(fs.front().deriv) > 0;
    bool pos = false, neg = false;
    for (const auto& ft : fs) {
        Vec3 n;
        for (int k = 0; k < 3; ++k) n.x[k] = -ft.deriv.x[k];
        pos |= ft.check(ft.deriv);
        neg |= ft.check(n);
    }
    return !(pos && !neg);
}

std::vector<Vec3> Evaluator::features(float x, float y, float z,
                                      const std::shared_ptr<Tape>& tape)
{
    float value;
    auto t = value_and_push(x, y, z, tape, &value);
    uint32_t root;
    const auto fs = feature_lists(*t, &root);
    std::vector<Vec3> out;
    for (const auto& ft : fs) {
        bool found = false;
        for (const auto& o : out) {
            if (vcmp(o, ft.deriv) == 0) { found = true; break; }
        }
        if (!found) out.push_back(ft.deriv);
    }
    return out;
}

// JacobianEvaluator::gradient (eval_jacobian.cpp:49-115) at one point.
void Evaluator::jacobian(float x, float y, float z, float* out)
{
    const size_t nv = base->vars.size();
    const size_t n = base->num_clauses + 1;
    std::vector<float> saved(d);
    clear_vars = true;
    set(x, y, z, 0);
    values(1, *base);
    // Column i of the tangent block carries one variable; the reference
    // packs 3 per point-column, which yields the same per-variable sums.
    for (size_t k = 0; k < nv; ++k) {
        for (size_t s = 0; s < n; ++s) {
            d[(s * 3 + 0) * NB] = 0;
            d[(s * 3 + 1) * NB] = 0;
            d[(s * 3 + 2) * NB] = 0;
        }
        d[(base->vars[k].first * 3 + 0) * NB] = 1.0f;
        for (auto it = base->t.rbegin(); it != base->t.rend(); ++it) {
            const bool unary = op_arity(it->op) == 1;
            float ad[3], bd[3], od[3];
            for (int q = 0; q < 3; ++q) {
                ad[q] = d[(it->a * 3 + q) * NB];
                bd[q] = unary ? 0.0f : d[(it->b * 3 + q) * NB];
            }
            deriv_op(it->op, v[it->a * NB], unary ? 0.0f : v[it->b * NB],
                     v[it->id * NB], ad, bd, od, true);
            for (int q = 0; q < 3; ++q) d[(it->id * 3 + q) * NB] = od[q];
        }
        out[k] = d[(base->root * 3 + 0) * NB];
    }
    d.swap(saved);
    clear_vars = false;
}

int op_arity(int op)
{
    switch (op) {
        case OP_ADD: case OP_MUL: case OP_MIN: case OP_MAX: case OP_SUB:
        case OP_DIV: case OP_ATAN2: case OP_POW: case OP_NTH_ROOT:
        case OP_MOD: case OP_NANFILL: case OP_COMPARE:
            return 2;
        default:
            return 1;
    }
}

}  // namespace ora
