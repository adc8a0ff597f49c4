#include "eval_api.hpp"

#include <vector>

#include "eval_kernels.cuh"
#include "jit.hpp"
#include "libfive_b200.h"

namespace lfb {

static constexpr uint64_t kChunk = 1ull << 30;

int eval_values_device(GpuTape& g, uint64_t n, const float* x, const float* y,
                       const float* z, float* out, cudaStream_t s)
{
    if (!require_device()) return LFB_E_CUDA;
    if (jit_values(g, n, x, y, z, out, s)) return 0;
    const DevTape t = g.dev();
    for (uint64_t off = 0; off < n; off += kChunk) {
        const uint32_t m = static_cast<uint32_t>(std::min(kChunk, n - off));
        if (!cuda_ok(launch_values(t, m, x + off, y + off, z + off, out + off, s),
                     "value kernel")) {
            return LFB_E_CUDA;
        }
        note_launches(1);
    }
    return 0;
}

namespace {
// LFB_E_CUDA when an interpreter block gave up waiting for its clause copy
// (its results were not written), else 0.
int stage_status()
{
    if (!stage_fault_take()) return 0;
    return set_error(LFB_E_CUDA, "interpreter: clause stream copy timed out");
}

struct Staging {
    DevBuf buf;
};
Staging& staging()
{
    static Staging s;
    return s;
}
}  // namespace

int eval_values_host(GpuTape& g, uint64_t n, const float* x, const float* y,
                     const float* z, float* out)
{
    if (!require_device()) return LFB_E_CUDA;
    if (n == 0) return 0;
    std::lock_guard<std::mutex> lock(global_mutex());
    auto& st = staging();
    if (!st.buf.reserve(n * 4 * sizeof(float))) return LFB_E_CUDA;
    float* d = st.buf.as<float>();
    const size_t b = n * sizeof(float);
    cudaStream_t s = 0;
    if (!cuda_ok(cudaMemcpyAsync(d, x, b, cudaMemcpyHostToDevice, s), "copy") ||
        !cuda_ok(cudaMemcpyAsync(d + n, y, b, cudaMemcpyHostToDevice, s), "copy") ||
        !cuda_ok(cudaMemcpyAsync(d + 2 * n, z, b, cudaMemcpyHostToDevice, s), "copy")) {
        return LFB_E_CUDA;
    }
    int rc = eval_values_device(g, n, d, d + n, d + 2 * n, d + 3 * n, s);
    if (rc) return rc;
    if (!cuda_ok(cudaMemcpyAsync(out, d + 3 * n, b, cudaMemcpyDeviceToHost, s), "copy") ||
        !cuda_ok(stage_fault_fetch(s), "copy") ||
        !cuda_ok(cudaStreamSynchronize(s), "sync")) {
        return LFB_E_CUDA;
    }
    return stage_status();
}

int eval_derivs_device(GpuTape& g, uint64_t n, const float* x, const float* y,
                       const float* z, float* v, float* dx, float* dy,
                       float* dz, cudaStream_t s)
{
    if (!require_device()) return LFB_E_CUDA;
    if (jit_derivs(g, n, x, y, z, v, dx, dy, dz, s)) return 0;
    const DevTape t = g.dev();
    for (uint64_t off = 0; off < n; off += kChunk) {
        const uint32_t m = static_cast<uint32_t>(std::min(kChunk, n - off));
        if (!cuda_ok(launch_derivs(t, m, x + off, y + off, z + off, v + off,
                                   dx ? dx + off : nullptr,
                                   dy ? dy + off : nullptr,
                                   dz ? dz + off : nullptr, s),
                     "derivative kernel")) {
            return LFB_E_CUDA;
        }
        note_launches(1);
    }
    return 0;
}

int eval_derivs_host(GpuTape& g, uint64_t n, const float* x, const float* y,
                     const float* z, float* v, float* dx, float* dy, float* dz)
{
    if (!require_device()) return LFB_E_CUDA;
    if (n == 0) return 0;
    std::lock_guard<std::mutex> lock(global_mutex());
    auto& st = staging();
    if (!st.buf.reserve(n * 7 * sizeof(float))) return LFB_E_CUDA;
    float* d = st.buf.as<float>();
    const size_t b = n * sizeof(float);
    cudaStream_t s = 0;
    if (!cuda_ok(cudaMemcpyAsync(d, x, b, cudaMemcpyHostToDevice, s), "copy") ||
        !cuda_ok(cudaMemcpyAsync(d + n, y, b, cudaMemcpyHostToDevice, s), "copy") ||
        !cuda_ok(cudaMemcpyAsync(d + 2 * n, z, b, cudaMemcpyHostToDevice, s), "copy")) {
        return LFB_E_CUDA;
    }
    int rc = eval_derivs_device(g, n, d, d + n, d + 2 * n, d + 3 * n,
                                d + 4 * n, d + 5 * n, d + 6 * n, s);
    if (rc) return rc;
    float* outs[4] = {v, dx, dy, dz};
    for (int k = 0; k < 4; ++k) {
        if (outs[k] &&
            !cuda_ok(cudaMemcpyAsync(outs[k], d + (3 + k) * n, b,
                                     cudaMemcpyDeviceToHost, s), "copy")) {
            return LFB_E_CUDA;
        }
    }
    if (!cuda_ok(stage_fault_fetch(s), "copy") ||
        !cuda_ok(cudaStreamSynchronize(s), "sync")) {
        return LFB_E_CUDA;
    }
    return stage_status();
}

int eval_intervals_device(GpuTape& g, uint64_t n, const float* xlo,
                          const float* xhi, const float* ylo,
                          const float* yhi, const float* zlo,
                          const float* zhi, float* olo, float* ohi,
                          uint8_t* onan, cudaStream_t s)
{
    if (!require_device()) return LFB_E_CUDA;
    if (jit_intervals(g, n, xlo, xhi, ylo, yhi, zlo, zhi, olo, ohi, onan, s)) return 0;
    const DevTape t = g.dev();
    for (uint64_t off = 0; off < n; off += kChunk) {
        const uint32_t m = static_cast<uint32_t>(std::min(kChunk, n - off));
        if (!cuda_ok(launch_intervals(t, m, xlo + off, xhi + off, ylo + off,
                                      yhi + off, zlo + off, zhi + off,
                                      olo + off, ohi + off, onan + off, s),
                     "interval kernel")) {
            return LFB_E_CUDA;
        }
        note_launches(1);
    }
    return 0;
}

int eval_intervals_host(GpuTape& g, uint64_t n, const float* xlo,
                        const float* xhi, const float* ylo, const float* yhi,
                        const float* zlo, const float* zhi, float* olo,
                        float* ohi, uint8_t* onan)
{
    if (!require_device()) return LFB_E_CUDA;
    if (n == 0) return 0;
    std::lock_guard<std::mutex> lock(global_mutex());
    auto& st = staging();
    if (!st.buf.reserve(n * 9 * sizeof(float))) return LFB_E_CUDA;
    float* d = st.buf.as<float>();
    const size_t b = n * sizeof(float);
    cudaStream_t s = 0;
    const float* ins[6] = {xlo, xhi, ylo, yhi, zlo, zhi};
    for (int k = 0; k < 6; ++k) {
        if (!cuda_ok(cudaMemcpyAsync(d + k * n, ins[k], b,
                                     cudaMemcpyHostToDevice, s), "copy")) {
            return LFB_E_CUDA;
        }
    }
    uint8_t* dn = reinterpret_cast<uint8_t*>(d + 8 * n);
    int rc = eval_intervals_device(g, n, d, d + n, d + 2 * n, d + 3 * n,
                                   d + 4 * n, d + 5 * n, d + 6 * n, d + 7 * n,
                                   dn, s);
    if (rc) return rc;
    if (!cuda_ok(cudaMemcpyAsync(olo, d + 6 * n, b, cudaMemcpyDeviceToHost, s), "copy") ||
        !cuda_ok(cudaMemcpyAsync(ohi, d + 7 * n, b, cudaMemcpyDeviceToHost, s), "copy") ||
        !cuda_ok(cudaMemcpyAsync(onan, dn, n, cudaMemcpyDeviceToHost, s), "copy")) {
        return LFB_E_CUDA;
    }
    if (!cuda_ok(stage_fault_fetch(s), "copy") ||
        !cuda_ok(cudaStreamSynchronize(s), "sync")) {
        return LFB_E_CUDA;
    }
    return stage_status();
}

}  // namespace lfb
