// Batched least-squares fitting of free variables (lfb_fit_adam_step).
//
// The reference has no optimiser: its JacobianEvaluator (eval_jacobian.cpp
// :49-115) gives df/dvar at one point, and fitting is left to the caller.
// Here one call takes one Adam step (Kingma & Ba, 2015) on many tapes at
// once, on loss_j = mean_i f_j(p_i)^2 over each shape's own points:
//
//  1. per shape, the reverse mode of grad_kernels.cu with seed f (the
//     forward pass writes f before the backward pass reads it as the seed),
//     which sums f_i df_i/dvar into a per-shape gradient;
//  2. one kernel, one block per shape: the loss (squares of f summed in
//     double, in a fixed order, so it does not depend on scheduling) and
//     the Adam update of the shape's variables, written into the tape's
//     variable slots in its device constant pool, where every evaluator and
//     the mesher read them.
//
// The arithmetic of the update is that of torch.optim.Adam's single-tensor
// step (no weight decay, no amsgrad): m lerped towards g by 1 - beta1,
// v = beta2 v + (1 - beta2) g g, var -= step_size * m / (sqrt(v) /
// sqrt(1 - beta2^t) + eps) with step_size = lr / (1 - beta1^t).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <exception>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "eval_api.hpp"
#include "libfive_b200.h"

namespace lfb {

namespace {

constexpr int kFitBlock = 512;
// Shapes per launch: the descriptors travel in the kernel's parameter
// block, which stays under 4 KB.
constexpr int kFitShapesPerLaunch = 48;

struct FitShape {
    const float* f;      // f at the shape's points (reverse-mode forward pass)
    const float* grad;   // sum_i f_i df_i/dvar_k
    float* vars;         // the tape's variable slots (device constant pool)
    float* m;            // Adam moments of the shape's variables
    float* v;
    float* loss;         // mean f^2 out
    uint64_t n;          // points
    uint32_t n_vars;
    float scale;         // 2 / n: d(mean f^2)/df_i = (2 / n) f_i
};

struct FitBatch {
    FitShape s[kFitShapesPerLaunch];
    float one_minus_beta1;
    float beta2;
    float one_minus_beta2;
    float step_size;     // lr / (1 - beta1^t)
    float bc2_sqrt;      // sqrt(1 - beta2^t)
    float eps;
};
static_assert(sizeof(FitBatch) <= 4000, "fit descriptors exceed the parameter block");

__global__ void __launch_bounds__(kFitBlock) k_fit_loss_adam(const FitBatch B)
{
    const FitShape& sh = B.s[blockIdx.x];
    const unsigned tid = threadIdx.x;

    // loss: per-thread sums over a fixed stride, then a fixed tree
    double acc = 0.0;
    for (uint64_t i = tid; i < sh.n; i += kFitBlock) {
        const double fi = static_cast<double>(sh.f[i]);
        acc += fi * fi;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    __shared__ double part[kFitBlock / 32];
    if ((tid & 31) == 0) part[tid >> 5] = acc;
    __syncthreads();
    if (tid < 32) {
        double a = tid < kFitBlock / 32 ? part[tid] : 0.0;
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (tid == 0) *sh.loss = static_cast<float>(a / static_cast<double>(sh.n));
    }

    // Adam, one variable per thread (built with -fmad=false: every product
    // and sum below is rounded on its own)
    for (uint32_t k = tid; k < sh.n_vars; k += kFitBlock) {
        const float g = sh.grad[k] * sh.scale;
        float m = sh.m[k];
        float v = sh.v[k];
        m = m + B.one_minus_beta1 * (g - m);
        v = v * B.beta2 + (B.one_minus_beta2 * g) * g;
        const float denom = sqrtf(v) / B.bc2_sqrt + B.eps;
        sh.vars[k] = sh.vars[k] + (-B.step_size) * (m / denom);
        sh.m[k] = m;
        sh.v[k] = v;
    }
}

/// Scratch of the fit step: f at every point and the per-shape gradients.
struct FitScratch {
    std::mutex mu;
    DevBuf f, grad;
};

FitScratch& fit_scratch()
{
    static FitScratch s;
    return s;
}

/// Prepares the reverse mode of every tape that has not been prepared, on
/// up to 16 host threads (the compiled kernels of a tape are built with
/// NVRTC, which takes most of a first call).
int prepare_all(GpuTape* const* tapes, uint32_t n)
{
    std::vector<GpuTape*> todo;
    for (uint32_t j = 0; j < n; ++j) {
        if (!grad_prepared(*tapes[j]) &&
            std::find(todo.begin(), todo.end(), tapes[j]) == todo.end()) {
            todo.push_back(tapes[j]);
        }
    }
    if (todo.empty()) return 0;
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "fit set-up")) return LFB_E_CUDA;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t n_threads = std::min<size_t>({todo.size(), hw, 16});
    std::atomic<size_t> next{0};
    std::mutex err_mu;
    int err_code = 0;
    std::string err_msg;
    auto work = [&] {
        // cudaFree(0) makes the device's context current on this thread, for
        // the module loads of the compiled kernels
        if (cudaSetDevice(dev) != cudaSuccess || cudaFree(nullptr) != cudaSuccess) {
            std::lock_guard<std::mutex> lock(err_mu);
            if (!err_code) { err_code = LFB_E_CUDA; err_msg = "fit set-up: cudaSetDevice failed"; }
            return;
        }
        for (size_t i; (i = next.fetch_add(1)) < todo.size();) {
            if (!grad_prepare(*todo[i])) {
                std::string msg;
                const int code = last_error(&msg);
                std::lock_guard<std::mutex> lock(err_mu);
                if (!err_code) { err_code = code ? code : LFB_E_CUDA; err_msg = msg; }
            }
        }
    };
    if (n_threads <= 1) {
        work();
    } else {
        std::vector<std::thread> pool;
        try {
            for (size_t t = 0; t < n_threads; ++t) pool.emplace_back(work);
        } catch (const std::exception&) {
            // fewer threads than asked for: this thread helps below
        }
        if (pool.size() < n_threads) work();
        for (auto& t : pool) t.join();
    }
    return err_code ? set_error(err_code, err_msg) : 0;
}

}  // namespace

int fit_adam_step(GpuTape* const* tapes, uint32_t n_shapes, const uint64_t* poff,
                  const float* x, const float* y, const float* z, const uint64_t* voff,
                  float* m, float* v, const lfb_adam_settings& a, uint32_t step,
                  float* losses, cudaStream_t s)
{
    if (!require_device()) return LFB_E_CUDA;
    if (n_shapes == 0) return 0;
    if (!poff || !voff || !x || !y || !z || !losses) {
        return set_error(LFB_E_INVALID, "lfb_fit_adam_step: null argument");
    }
    if (step == 0) return set_error(LFB_E_INVALID, "lfb_fit_adam_step: step counts from 1");
    if (!(a.lr >= 0.0f) || !(a.beta1 >= 0.0f && a.beta1 < 1.0f) ||
        !(a.beta2 >= 0.0f && a.beta2 < 1.0f) || !(a.eps > 0.0f)) {
        return set_error(LFB_E_INVALID, "lfb_fit_adam_step: Adam settings out of range "
                                        "(lr >= 0, 0 <= beta < 1, eps > 0)");
    }
    for (uint32_t j = 0; j < n_shapes; ++j) {
        if (poff[j + 1] <= poff[j]) {
            return set_error(LFB_E_INVALID, "lfb_fit_adam_step: shape " + std::to_string(j) +
                                                " has no points (point_offsets must increase)");
        }
        if (voff[j + 1] < voff[j] || voff[j + 1] - voff[j] != tapes[j]->reg.n_vars) {
            return set_error(LFB_E_INVALID,
                             "lfb_fit_adam_step: var_offsets of shape " + std::to_string(j) +
                                 " span " + std::to_string(voff[j + 1] - voff[j]) +
                                 " variables, its tape has " +
                                 std::to_string(tapes[j]->reg.n_vars));
        }
    }
    {
        // one block updates each shape's variables: a tape listed twice
        // would be updated by two blocks at once
        std::vector<GpuTape*> sorted(tapes, tapes + n_shapes);
        std::sort(sorted.begin(), sorted.end());
        if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end()) {
            return set_error(LFB_E_INVALID, "lfb_fit_adam_step: a tape is listed twice");
        }
    }
    if (voff[n_shapes] > voff[0] && (!m || !v)) {
        return set_error(LFB_E_INVALID, "lfb_fit_adam_step: null Adam moments");
    }
    const uint64_t p0 = poff[0], n_points = poff[n_shapes] - p0;
    const uint64_t v0 = voff[0], n_vars = voff[n_shapes] - v0;

    FitScratch& sc = fit_scratch();
    std::lock_guard<std::mutex> lock(sc.mu);
    if (int rc = prepare_all(tapes, n_shapes)) return rc;
    if (!sc.f.reserve(n_points * sizeof(float)) ||
        !sc.grad.reserve(std::max<uint64_t>(n_vars, 1) * sizeof(float))) {
        return LFB_E_CUDA;
    }
    float* f = sc.f.as<float>();
    float* grad = sc.grad.as<float>();
    if (n_vars && !cuda_ok(cudaMemsetAsync(grad, 0, n_vars * sizeof(float), s), "fit")) {
        return LFB_E_CUDA;
    }
    for (uint32_t j = 0; j < n_shapes; ++j) {
        const uint64_t o = poff[j] - p0, n = poff[j + 1] - poff[j];
        float* gv = voff[j + 1] > voff[j] ? grad + (voff[j] - v0) : nullptr;
        if (int rc = eval_grad(*tapes[j], n, x + poff[j], y + poff[j], z + poff[j], f + o, f + o,
                               nullptr, nullptr, nullptr, gv, s, true)) {
            return rc;
        }
    }

    FitBatch B{};
    B.one_minus_beta1 = 1.0f - a.beta1;
    B.beta2 = a.beta2;
    B.one_minus_beta2 = 1.0f - a.beta2;
    const double t = static_cast<double>(step);
    B.step_size = static_cast<float>(a.lr / (1.0 - std::pow(static_cast<double>(a.beta1), t)));
    B.bc2_sqrt = static_cast<float>(std::sqrt(1.0 - std::pow(static_cast<double>(a.beta2), t)));
    B.eps = a.eps;
    for (uint32_t j0 = 0; j0 < n_shapes; j0 += kFitShapesPerLaunch) {
        const uint32_t cnt = std::min<uint32_t>(kFitShapesPerLaunch, n_shapes - j0);
        for (uint32_t c = 0; c < cnt; ++c) {
            const uint32_t j = j0 + c;
            GpuTape& g = *tapes[j];
            FitShape& d = B.s[c];
            d.f = f + (poff[j] - p0);
            d.n = poff[j + 1] - poff[j];
            d.grad = grad + (voff[j] - v0);
            d.vars = g.d_cpool + g.reg.n_const;
            d.m = m ? m + voff[j] : nullptr;
            d.v = v ? v + voff[j] : nullptr;
            d.n_vars = g.reg.n_vars;
            d.loss = losses + j;
            d.scale = static_cast<float>(2.0 / static_cast<double>(d.n));
        }
        k_fit_loss_adam<<<cnt, kFitBlock, 0, s>>>(B);
        if (!cuda_ok(cudaGetLastError(), "fit kernel")) return LFB_E_CUDA;
        note_launches(1);
    }
    for (uint32_t j = 0; j < n_shapes; ++j) {
        std::lock_guard<std::mutex> tl(tapes[j]->mu);
        if (tapes[j]->reg.n_vars) tapes[j]->vars_on_device = true;
    }
    return 0;
}

}  // namespace lfb
