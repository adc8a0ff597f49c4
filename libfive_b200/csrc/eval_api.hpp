// Host-side drivers for the batched evaluation kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "libfive_b200.h"
#include "runtime.hpp"

namespace lfb {

int eval_values_device(GpuTape& g, uint64_t n, const float* x, const float* y,
                       const float* z, float* out, cudaStream_t s);
int eval_values_host(GpuTape& g, uint64_t n, const float* x, const float* y,
                     const float* z, float* out);

int eval_derivs_device(GpuTape& g, uint64_t n, const float* x, const float* y,
                       const float* z, float* v, float* dx, float* dy,
                       float* dz, cudaStream_t s);
int eval_derivs_host(GpuTape& g, uint64_t n, const float* x, const float* y,
                     const float* z, float* v, float* dx, float* dy,
                     float* dz);

int eval_intervals_device(GpuTape& g, uint64_t n, const float* xlo,
                          const float* xhi, const float* ylo,
                          const float* yhi, const float* zlo,
                          const float* zhi, float* olo, float* ohi,
                          uint8_t* onan, cudaStream_t s);
int eval_intervals_host(GpuTape& g, uint64_t n, const float* xlo,
                        const float* xhi, const float* ylo, const float* yhi,
                        const float* zlo, const float* zhi, float* olo,
                        float* ohi, uint8_t* onan);

/// lfb_eval_features (feature_api.cu); host arrays.
int eval_features_host(GpuTape& g, uint64_t n, const float* x, const float* y, const float* z,
                       uint8_t* inside, float* feats, uint32_t max_feats, uint32_t* n_feats);

int eval_jacobian(GpuTape& g, uint64_t n, const float* x, const float* y,
                  const float* z, float* out, cudaStream_t s, bool device);

/// lfb_eval_loss_grad (device arrays).
int eval_loss_grad(GpuTape& g, uint64_t n, const float* x, const float* y, const float* z,
                   float* f, float* gx, float* gy, float* gz, float* gvars, float* loss,
                   cudaStream_t s);

int eval_grad(GpuTape& g, uint64_t n, const float* x, const float* y,
              const float* z, const float* seed, float* f, float* gx,
              float* gy, float* gz, float* gvars, cudaStream_t s,
              bool device);

/// Builds what the reverse mode needs for this tape (partial-slot table,
/// compiled partials and backward kernels) without launching anything, so
/// that many tapes can be prepared on several host threads at once.
bool grad_prepare(GpuTape& g);
/// True once grad_prepare (or a gradient call) has run for the tape.
bool grad_prepared(GpuTape& g);

/// lfb_fit_adam_step (fit.cu); every pointer as documented there.
int fit_adam_step(GpuTape* const* tapes, uint32_t n_shapes, const uint64_t* point_offsets,
                  const float* x, const float* y, const float* z, const uint64_t* var_offsets,
                  float* m, float* v, const lfb_adam_settings& adam, uint32_t step,
                  float* losses, cudaStream_t s);

}  // namespace lfb
