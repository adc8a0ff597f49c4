#pragma once
#include <cuda_runtime.h>

#include "dev_ops.cuh"

namespace lfb {

int device_sm_count();

cudaError_t launch_values(const DevTape& t, uint32_t n, const float* x,
                          const float* y, const float* z, float* out,
                          cudaStream_t s);

cudaError_t launch_derivs(const DevTape& t, uint32_t n, const float* x,
                          const float* y, const float* z, float* v,
                          float* dx, float* dy, float* dz, cudaStream_t s);

cudaError_t launch_intervals(const DevTape& t, uint32_t n, const float* xlo,
                             const float* xhi, const float* ylo,
                             const float* yhi, const float* zlo,
                             const float* zhi, float* olo, float* ohi,
                             uint8_t* onan, cudaStream_t s);

// The interpreters' clause-copy timeout flag (clause_stage.cuh): fetch
// enqueues a copy of the device flag to page-locked host memory on `s`;
// after the stream has been synchronised, take() says whether it was set
// and clears it.
cudaError_t stage_fault_fetch(cudaStream_t s);
bool stage_fault_take();

}  // namespace lfb
