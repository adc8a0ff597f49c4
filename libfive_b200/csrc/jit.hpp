// Tapes compiled to straight-line CUDA kernels at run time (NVRTC).
//
// The value interpreter spends most of its instructions decoding clauses and
// moving operands through a shared-memory register file.  For a tape that
// is evaluated over many points, compiling it once into a kernel whose body
// is the clause list itself (each clause one or two instructions, operands
// in hardware registers) removes that overhead.  The generated code uses
// the same separately rounded operations as the interpreters (written out
// for the common opcodes, the interpreters' own functions from
// dev_point.cuh / dev_interval.cuh for the rest), so both give identical
// bits; tapes longer than kJitMaxClauses stay on the interpreters.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "runtime.hpp"

namespace lfb {

constexpr uint32_t kJitMaxClauses = 4096;
/// The interval kernel's limit is lower: its compile time grows much faster
/// than the tape (NVRTC for sm_100a on a development host: 5 s for 703
/// clauses, 69 s for 1924), while the interval interpreter gives the same
/// bounds and takes milliseconds for a height map's boxes.
constexpr uint32_t kJitMaxIntervalClauses = 1024;
/// Longer tapes are compiled in segments of a few hundred clauses (one
/// function each, registers passed through local memory), whose compile time
/// grows with the length: the value kernel and the checkpointed reverse mode
/// take tapes up to this length.
constexpr uint32_t kJitMaxSegmentedClauses = 65536;

/// Values of the tape at n points through its compiled kernel (compiled on
/// first use).  Returns false, with no error set, when the tape has no
/// compiled kernel (too long, NVRTC or the driver unavailable, or LFB_JIT=0
/// in the environment); the caller then uses the interpreter.
bool jit_values(GpuTape& g, uint64_t n, const float* x, const float* y, const float* z,
                float* out, cudaStream_t s);

/// Values and d/dx, d/dy, d/dz (dx / dy / dz may be null) through the
/// tape's compiled derivative kernel; the same conditions as jit_values, and
/// the same bits as DerivArrayEvaluator's rules in dv_deriv.
bool jit_derivs(GpuTape& g, uint64_t n, const float* x, const float* y, const float* z,
                float* v, float* dx, float* dy, float* dz, cudaStream_t s);
/// jit_derivs only when the tape's compiled kernel is already loaded (never
/// compiles or loads a module); false otherwise.
bool jit_derivs_if_loaded(GpuTape& g, uint64_t n, const float* x, const float* y,
                          const float* z, float* v, float* dx, float* dy, float* dz,
                          cudaStream_t s);

/// Reverse mode through compiled kernels: the forward pass storing the
/// local partials at P[slot * m + i] (slot table of partial_slots), and the
/// backward pass (block_cv: CONST_VAR blocks the adjoint).  Same
/// arithmetic, clause by clause, as the interpreted reverse mode; false when
/// the tape has no compiled form (then nothing was launched).
bool jit_partials(GpuTape& g, const uint32_t* slots, uint32_t m, const float* x,
                  const float* y, const float* z, float* P, float* f, cudaStream_t s);
bool jit_backward(GpuTape& g, const uint32_t* slots, uint32_t m, const float* P,
                  const float* seed, float* gx, float* gy, float* gz, float* gvars,
                  int block_cv, cudaStream_t s);

/// Intervals of the tape over n boxes through its compiled interval kernel
/// (the interval operations of dev_interval.cuh, written out per clause):
/// the same bounds and NaN flags as the interval interpreter.
bool jit_intervals(GpuTape& g, uint64_t n, const float* xlo, const float* xhi,
                   const float* ylo, const float* yhi, const float* zlo, const float* zhi,
                   float* olo, float* ohi, uint8_t* onan, cudaStream_t s);

/// Source of the interval kernel (empty when the tape has no compiled form)
/// and its compilation to a cubin, for checks that need no GPU.
std::string jit_interval_source(const RegTape& t);
bool jit_compile(const std::string& src, std::vector<char>* cubin, std::string* log);

/// Checkpointed reverse mode (compiled in segments): the forward kernel
/// writes f and, per point, the registers each segment reads from earlier
/// segments (C[slot * m + i], jit_ckpt_prepare's count of slots); the
/// backward kernel recomputes each segment from them and sweeps its
/// adjoints back, with the products and sums of the partials / backward
/// kernels.  jit_ckpt_prepare compiles both and returns the slot count, or 0
/// when the tape has no compiled form.
uint32_t jit_ckpt_prepare(GpuTape& g);
bool jit_ckpt_forward(GpuTape& g, uint32_t m, const float* x, const float* y, const float* z,
                      float* C, float* f, cudaStream_t s);
/// The seed of point i is seed[i] (1 when seed is null) times seed_scale.
bool jit_ckpt_backward(GpuTape& g, uint32_t m, const float* C, const float* seed, float* gx,
                       float* gy, float* gz, float* gvars, int block_cv, cudaStream_t s,
                       float seed_scale = 1.0f);

/// Releases a tape's compiled kernels (called when the tape is destroyed).
void jit_release(GpuTape& g);

}  // namespace lfb
