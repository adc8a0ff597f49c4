// Value-and-gradient evaluation of host points without any device allocation.
//
// Some callers cannot allocate device memory while they run: a renderer
// whose frame loop must never hit cudaMalloc / cudaFree (both synchronise
// the whole device and can stall other streams), or a host application
// that has handed its entire device memory budget to its own allocator.
// lfb_eval_derivs_static serves them: it stages the points and results
// through one fixed array that is part of the library image, so the call
// itself allocates nothing.
//
// The array is a file-scope __device__ variable of kStaticPoints * 7 floats
// (7 MiB).  Every process that loads the library holds it on every GPU it
// uses, until exit.  Host code cannot use the variable's name as a device
// address: the address is looked up with cudaGetSymbolAddress once per
// device, with that device current, on the first call made on that device.
// CUDA loads a library's device code lazily, so that first lookup is also
// when the array's 7 MiB are reserved on the device: the first call on each
// device does take device memory, once, and should be made during set-up,
// before any stream capture begins (a call with n == 0 returns before the
// lookup and does not do it).
//
// The kernel is the tape's compiled value + derivative kernel when that
// kernel is already loaded (a previous lfb_eval_derivs compiled it; the
// static path never compiles or loads anything itself), otherwise the
// interpreter, which needs the tape's register file in shared memory: tapes
// of more than about 100 registers are rejected with LFB_E_CUDA.  Both give
// the same bits as lfb_eval_derivs.
//
// All calls share the array and it keeps the last call's contents.  Each
// call overwrites every element it reads before reading it, so nothing needs
// clearing, and each call waits for its own copies before returning.  Calls
// made through this function are serialised by a host mutex; any other work
// that touches the array while a call is in flight on the same device (for
// example a second copy of the library's code in the same process) races
// with it, so such calls must not overlap on the GPU.
#include <mutex>

#include "eval_kernels.cuh"
#include "jit.hpp"
#include "libfive_b200.h"
#include "runtime.hpp"

namespace lfb {

GpuTape* tape_of(lfb_tape t);

namespace {

constexpr uint64_t kStaticPoints = 262144;   // points per call, at most
constexpr int kMaxDevices = 64;

// x, y, z, value, d/dx, d/dy, d/dz planes of kStaticPoints floats each.
static __device__ __align__(256) float g_static_scratch[7 * kStaticPoints];

std::mutex g_static_mu;
float* g_static_ptr[kMaxDevices] = {};

/// Device address of g_static_scratch on the current device (looked up on
/// the first call per device).
float* static_scratch(int dev)
{
    if (dev < 0 || dev >= kMaxDevices) {
        set_error(LFB_E_CUDA, "lfb_eval_derivs_static: device ordinal out of range");
        return nullptr;
    }
    if (!g_static_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p) {
            set_error(LFB_E_CUDA, std::string("lfb_eval_derivs_static: "
                                              "cudaGetSymbolAddress failed: ") +
                                      cudaGetErrorString(e));
            return nullptr;
        }
        g_static_ptr[dev] = static_cast<float*>(p);
    }
    return g_static_ptr[dev];
}

}  // namespace

}  // namespace lfb

using namespace lfb;

extern "C" int lfb_eval_derivs_static(lfb_tape t, uint64_t n, const float* x,
                                      const float* y, const float* z,
                                      float* v, float* dx, float* dy,
                                      float* dz)
{
    clear_error();
    GpuTape* g = tape_of(t);
    if (!g || !x || !y || !z || !v) {
        return set_error(LFB_E_INVALID, "lfb_eval_derivs_static: null argument");
    }
    if (n > kStaticPoints) {
        return set_error(LFB_E_INVALID,
                         "lfb_eval_derivs_static: at most 262144 points per call "
                         "(the fixed device buffer holds no more)");
    }
    if (!require_device()) return LFB_E_CUDA;
    if (n == 0) return 0;
    if (!g->on_current_device()) return LFB_E_INVALID;

    std::lock_guard<std::mutex> lock(g_static_mu);
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "lfb_eval_derivs_static")) return LFB_E_CUDA;
    float* base = static_scratch(dev);
    if (!base) return LFB_E_CUDA;

    cudaStream_t s = 0;
    const size_t b = n * sizeof(float);
    float* planes[7];
    for (int k = 0; k < 7; ++k) planes[k] = base + k * kStaticPoints;
    const float* ins[3] = {x, y, z};
    for (int k = 0; k < 3; ++k) {
        if (!cuda_ok(cudaMemcpyAsync(planes[k], ins[k], b, cudaMemcpyHostToDevice, s),
                     "lfb_eval_derivs_static: copy in")) {
            return LFB_E_CUDA;
        }
    }
    if (!jit_derivs_if_loaded(*g, n, planes[0], planes[1], planes[2], planes[3], planes[4],
                              planes[5], planes[6], s)) {
        if (!cuda_ok(launch_derivs(g->dev(), static_cast<uint32_t>(n), planes[0],
                                   planes[1], planes[2], planes[3], planes[4],
                                   planes[5], planes[6], s),
                     "lfb_eval_derivs_static: kernel")) {
            return LFB_E_CUDA;
        }
        note_launches(1);
    }
    float* outs[4] = {v, dx, dy, dz};
    for (int k = 0; k < 4; ++k) {
        if (outs[k] && !cuda_ok(cudaMemcpyAsync(outs[k], planes[3 + k], b,
                                                cudaMemcpyDeviceToHost, s),
                                "lfb_eval_derivs_static: copy out")) {
            return LFB_E_CUDA;
        }
    }
    return cuda_ok(cudaStreamSynchronize(s), "lfb_eval_derivs_static: sync")
        ? 0 : LFB_E_CUDA;
}
