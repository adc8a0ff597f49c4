// Point-wise float32 semantics of every opcode, shared by host constant
// folding and the device evaluators so that both produce identical bits.
//
// Each function restates one case of ArrayEvaluator::operator()
// (libfive/src/eval/eval_array.cpp:221-369).  min/max follow std::min /
// std::max exactly (NaN propagates only from the first argument, and
// min(-0, +0) returns the first argument), which is what Eigen's cwiseMin /
// cwiseMax compute in the reference.  Every arithmetic step is written as
// an explicit, separately rounded IEEE operation; the translation units that
// include this header are compiled without FMA contraction.
#pragma once
#ifdef __CUDACC_RTC__
// kernels compiled at run time: math functions are built in
#ifndef NAN
#define NAN __int_as_float(0x7fc00000)
#endif
#else
#include <cmath>
#include <cstdint>
#endif

#include "scalar_minmax.h"

namespace lfb {

LF_HD bool sc_isnan(float a) { return a != a; }

/// Python-style modulo with the reference's clamping rules
/// (eval_array.cpp:262-286).
LF_HD float sc_mod(float a, float b)
{
    float d = fabsf(a / b);
    if ((a < 0) ^ (b < 0)) {
        d = -ceilf(d);
    } else {
        d = floorf(d);
    }
    const float bd = b * d;
    float out = a - bd;
    if ((b > 0 && out > b) || (b < 0 && out < b)) {
        out = b;
    }
    if ((b > 0.0f && out < 0.0f) || (b < 0.0f && out > 0.0f)) {
        out = 0.0f;
    }
    return out;
}

LF_HD float sc_compare(float a, float b)
{
    if (a < b) return -1.0f;
    if (a > b) return 1.0f;
    return 0.0f;
}

/// nth root of a point.  For a >= 0 this is powf(a, 1/b) as in
/// eval_array.cpp:248-260.  For a < 0 the reference evaluates Boost's
/// interval nth_root on [a, a]; that is -(|a|^(1/b)) for odd b and NaN for
/// even b, which is restated here with powf.
LF_HD float sc_nth_root(float a, float b)
{
    if (a < 0) {
        const int k = static_cast<int>(b);
        if ((k & 1) == 0) {
            return NAN;
        }
        return -powf(-a, 1.0f / b);
    }
    return powf(a, 1.0f / b);
}

}  // namespace lfb
