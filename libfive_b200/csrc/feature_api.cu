// Batched FeatureEvaluator calls (lfb_eval_features): the device feature
// evaluator of the mesher (dc_features.cuh) at caller-given points.
//
// FeatureEvaluator::isInside (libfive/src/eval/eval_feature.cpp:56-116) and
// FeatureEvaluator::features (eval_feature.cpp:125-169): one warp per point,
// lane 0 running the feature evaluator while the warp serves its
// Feature::check requests, exactly as the leaf kernel does at exact zeros.
#include <algorithm>

#include "dc_features.cuh"
#include "eval_api.hpp"
#include "libfive_b200.h"

namespace lfb {

namespace {

/// FeatureEvaluator::features: the distinct feature gradients at a point
/// (warp-collective, every lane passes the same point).  Writes at most
/// `max` of them to out (3 floats each); returns how many there are.
__device__ __noinline__ uint32_t dev_feature_list(const FeatCtx& C, const DevTape& bt,
                                                  float x, float y, float z, float* out,
                                                  uint32_t max, int lane)
{
    uint32_t count = 0;
    __syncwarp();
    if (lane == 0) {
        float v;
        const float* fs;
        int n;
        feat_eval(C, bt, bt.clauses, bt.n, x, y, z, &v, &fs, &n);
        for (int i = 0; i < n; ++i) {
            const float* f = fs + i * kFeatFloats;
            bool seen = false;
            for (int j = 0; j < i && !seen; ++j) seen = vcmp3(f, fs + j * kFeatFloats) == 0;
            if (seen) continue;
            if (out && count < max) {
                out[3 * count + 0] = f[0];
                out[3 * count + 1] = f[1];
                out[3 * count + 2] = f[2];
            }
            ++count;
        }
        feat_done(C);
    } else {
        feat_serve(C, lane);
    }
    __syncwarp();
    return __shfl_sync(0xffffffffu, count, 0);
}

/// Value of the tape at one point, evaluated by one thread with the
/// register file in `R` (n_regs floats).
__device__ float serial_value(const DevTape& t, float* R, float x, float y, float z)
{
    R[0] = x;
    R[1] = y;
    R[2] = z;
    for (uint32_t c = 0; c < t.n; ++c) {
        const RegClause k = t.clauses[c];
        const uint8_t ka = k.kinds & 3, kb = (k.kinds >> 2) & 3;
        const float a = ka == OPND_REG ? R[k.a] : __ldg(t.cpool + k.a);
        const float b = kb == OPND_REG ? R[k.b] : __ldg(t.cpool + k.b);
        R[k.out] = dv_value(k.op, a, b);
    }
    return t.root_kind == OPND_REG ? R[t.root] : __ldg(t.cpool + t.root);
}

constexpr int kWarpsPerBlock = 4;

__global__ void __launch_bounds__(32 * kWarpsPerBlock)
k_features(DevTape t, uint32_t n, const float* __restrict__ P, uint8_t* inside, float* feats,
           uint32_t max_feats, uint32_t* n_feats, float* featws, FeatureScratch* scratch,
           uint32_t* status)
{
    const int lane = threadIdx.x & 31;
    const uint32_t warp = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const uint32_t n_warps = gridDim.x * kWarpsPerBlock;
    const FeatCtx fc{featws + static_cast<size_t>(warp) * t.n_regs * kRegBlock,
                     scratch + warp, status};
    for (uint32_t i = warp; i < n; i += n_warps) {
        const float x = P[i], y = P[n + i], z = P[2 * static_cast<size_t>(n) + i];
        // isInside decides by the value alone unless it is zero (or NaN)
        // (eval_feature.cpp:56-72); only then are features built.
        float v = 0.0f;
        if (lane == 0) v = serial_value(t, fc.regs, x, y, z);
        v = __shfl_sync(0xffffffffu, v, 0);
        __syncwarp();
        const bool in = v < 0 ? true : v > 0 ? false
                                             : dev_is_inside(fc, t, t.clauses, t.n, x, y, z, lane);
        if (lane == 0) inside[i] = in ? 1 : 0;
        if (n_feats) {
            const uint32_t c = dev_feature_list(
                fc, t, x, y, z, feats ? feats + static_cast<size_t>(i) * max_feats * 3 : nullptr,
                max_feats, lane);
            if (lane == 0) n_feats[i] = c;
        }
    }
}

}  // namespace

int eval_features_host(GpuTape& g, uint64_t n, const float* x, const float* y, const float* z,
                       uint8_t* inside, float* feats, uint32_t max_feats, uint32_t* n_feats)
{
    if (!require_device()) return LFB_E_CUDA;
    if (n == 0) return 0;
    if (n > (1u << 24)) return set_error(LFB_E_INVALID, "at most 2^24 points per call");
    if (feats && !n_feats) return set_error(LFB_E_INVALID, "feats needs n_feats");
    std::lock_guard<std::mutex> lock(global_mutex());
    const DevTape t = g.dev();
    const uint32_t m = static_cast<uint32_t>(n);
    const unsigned blocks = static_cast<unsigned>(
        std::min<uint64_t>((n + kWarpsPerBlock - 1) / kWarpsPerBlock, 148 * 4));
    const uint32_t warps = blocks * kWarpsPerBlock;
    static DevBuf pts, outs, ws, scr;
    const size_t fbytes = feats ? static_cast<size_t>(n) * max_feats * 3 * sizeof(float) : 0;
    if (!pts.reserve(3 * n * sizeof(float)) ||
        !outs.reserve(n + 16 + n * sizeof(uint32_t) + fbytes + 16) ||
        !ws.reserve(static_cast<size_t>(warps) * t.n_regs * kRegBlock * sizeof(float)) ||
        !scr.reserve(warps * sizeof(FeatureScratch) + sizeof(uint32_t))) {
        return LFB_E_CUDA;
    }
    cudaStream_t s = 0;
    float* dp = pts.as<float>();
    const size_t b = n * sizeof(float);
    if (!cuda_ok(cudaMemcpyAsync(dp, x, b, cudaMemcpyHostToDevice, s), "copy") ||
        !cuda_ok(cudaMemcpyAsync(dp + n, y, b, cudaMemcpyHostToDevice, s), "copy") ||
        !cuda_ok(cudaMemcpyAsync(dp + 2 * n, z, b, cudaMemcpyHostToDevice, s), "copy")) {
        return LFB_E_CUDA;
    }
    uint8_t* d_in = outs.as<uint8_t>();
    uint32_t* d_nf = reinterpret_cast<uint32_t*>(d_in + (n + 15) / 16 * 16);
    float* d_f = reinterpret_cast<float*>(d_nf + n);
    FeatureScratch* d_scr = scr.as<FeatureScratch>();
    uint32_t* d_status = reinterpret_cast<uint32_t*>(d_scr + warps);
    if (!cuda_ok(cudaMemsetAsync(d_status, 0, sizeof(uint32_t), s), "memset")) return LFB_E_CUDA;
    k_features<<<blocks, 32 * kWarpsPerBlock, 0, s>>>(t, m, dp, d_in, feats ? d_f : nullptr,
                                                      max_feats, n_feats ? d_nf : nullptr,
                                                      ws.as<float>(), d_scr, d_status);
    note_launches(1);
    if (!cuda_ok(cudaGetLastError(), "feature kernel")) return LFB_E_CUDA;
    uint32_t status = 0;
    if (!cuda_ok(cudaMemcpyAsync(&status, d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
                 "copy") ||
        (inside && !cuda_ok(cudaMemcpyAsync(inside, d_in, n, cudaMemcpyDeviceToHost, s), "copy")) ||
        (n_feats && !cuda_ok(cudaMemcpyAsync(n_feats, d_nf, n * sizeof(uint32_t),
                                             cudaMemcpyDeviceToHost, s), "copy")) ||
        (feats && !cuda_ok(cudaMemcpyAsync(feats, d_f, fbytes, cudaMemcpyDeviceToHost, s),
                           "copy")) ||
        !cuda_ok(cudaStreamSynchronize(s), "sync")) {
        return LFB_E_CUDA;
    }
    if (status & ST_FEATURE_OVERFLOW) {
        return set_error(LFB_E_CAPACITY, "feature list capacity exceeded");
    }
    return 0;
}

}  // namespace lfb
