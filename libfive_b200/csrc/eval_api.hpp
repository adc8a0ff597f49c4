// Host-side drivers for the batched evaluation kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

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

int eval_jacobian(GpuTape& g, uint64_t n, const float* x, const float* y,
                  const float* z, float* out, cudaStream_t s, bool device);

int eval_grad(GpuTape& g, uint64_t n, const float* x, const float* y,
              const float* z, const float* seed, float* f, float* gx,
              float* gy, float* gz, float* gvars, cudaStream_t s,
              bool device);

}  // namespace lfb
