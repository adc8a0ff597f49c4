// std::min / std::max semantics of the reference's min and max (NaN only
// propagates from the first argument; min(-0, +0) is the first argument).
// No dependencies, so that run-time compiled kernels can include it too.
#pragma once

#ifdef __CUDACC__
#define LF_HD __host__ __device__ __forceinline__
#else
#define LF_HD inline
#endif

namespace lfb {

LF_HD float sc_min(float a, float b) { return (b < a) ? b : a; }
LF_HD float sc_max(float a, float b) { return (a < b) ? b : a; }

}  // namespace lfb
