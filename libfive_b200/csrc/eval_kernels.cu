// Batched point / box evaluation kernels.
//
// One thread evaluates one point (or box) through the whole register tape.
// Every thread of a block walks the same clause stream, so the clause fetch
// is a uniform (broadcast) load and the opcode switch never diverges; the
// register file lives in shared memory as [n_regs][blockDim] planes so that
// consecutive threads touch consecutive banks.
//
// These kernels replace the per-clause loops of
//   ArrayEvaluator::values       (libfive/src/eval/eval_array.cpp:106-118)
//   DerivArrayEvaluator::derivs  (libfive/src/eval/eval_deriv_array.cpp:101-117)
//   IntervalEvaluator::eval      (libfive/src/eval/eval_interval.cpp:68-93)
// which process at most 256 points per pass on one CPU thread.  The clause
// stream reaches shared memory by bulk asynchronous copies (clause_stage.cuh);
// the register planes follow the staging ring.
#include "clause_stage.cuh"
#include "eval_kernels.cuh"
#include "runtime.hpp"

namespace lfb {

__device__ __forceinline__ float fetch_v(uint8_t kind, uint16_t idx,
                                         const float* R, int tid, int B,
                                         const float* __restrict__ cp)
{
    return kind == OPND_REG ? R[idx * B + tid] : __ldg(cp + idx);
}

template <int PTS>
__global__ void __launch_bounds__(128)
k_values(DevTape t, uint32_t n, const float* __restrict__ X,
         const float* __restrict__ Y, const float* __restrict__ Z,
         float* __restrict__ out)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int B = blockDim.x * PTS;
    const int tid0 = threadIdx.x;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * B;
    ClauseStage stage(t, smem_raw, block_passes(n, B));
    float* R = reinterpret_cast<float*>(smem_raw + stage_bytes(t.n));
    const float* __restrict__ cp = t.cpool;
    for (uint64_t base = static_cast<uint64_t>(blockIdx.x) * B; base < n;
         base += stride) {
#pragma unroll
        for (int p = 0; p < PTS; ++p) {
            const int tid = tid0 + p * blockDim.x;
            const uint64_t i = base + tid;
            const bool ok = i < n;
            R[0 * B + tid] = ok ? X[i] : 0.0f;
            R[1 * B + tid] = ok ? Y[i] : 0.0f;
            R[2 * B + tid] = ok ? Z[i] : 0.0f;
        }
        const bool ok = stage.walk([&](uint8_t o, uint8_t kinds, uint16_t ro,
                                       uint16_t ra, uint16_t rb) {
#pragma unroll
            for (int p = 0; p < PTS; ++p) {
                const int tid = tid0 + p * blockDim.x;
                const float a = fetch_v(kinds & 3, ra, R, tid, B, cp);
                const float b = fetch_v((kinds >> 2) & 3, rb, R, tid, B, cp);
                R[ro * B + tid] = dv_value(o, a, b);
            }
        });
        if (!ok) return;
#pragma unroll
        for (int p = 0; p < PTS; ++p) {
            const int tid = tid0 + p * blockDim.x;
            const uint64_t i = base + tid;
            if (i < n) {
                out[i] = fetch_v(t.root_kind, t.root, R, tid, B, cp);
            }
        }
    }
    stage.finish();
}

__device__ __forceinline__ D4 fetch_d(uint8_t kind, uint16_t idx,
                                      const float* R, int tid, int B,
                                      const float* __restrict__ cp)
{
    if (kind == OPND_REG) {
        const float* r = R + idx * 4 * B + tid;
        return {r[0], r[B], r[2 * B], r[3 * B]};
    }
    return {__ldg(cp + idx), 0.0f, 0.0f, 0.0f};
}

__global__ void __launch_bounds__(128)
k_derivs(DevTape t, uint32_t n, const float* __restrict__ X,
         const float* __restrict__ Y, const float* __restrict__ Z,
         float* __restrict__ ov, float* __restrict__ odx,
         float* __restrict__ ody, float* __restrict__ odz)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int B = blockDim.x;
    const int tid = threadIdx.x;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * B;
    ClauseStage stage(t, smem_raw, block_passes(n, B));
    float* R = reinterpret_cast<float*>(smem_raw + stage_bytes(t.n));
    const float* __restrict__ cp = t.cpool;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * B + tid;
         i - tid < n; i += stride) {
        const bool ok = i < n;
        const float px = ok ? X[i] : 0.0f;
        const float py = ok ? Y[i] : 0.0f;
        const float pz = ok ? Z[i] : 0.0f;
        float* r0 = R + 0 * 4 * B + tid;
        r0[0] = px; r0[B] = 1.0f; r0[2 * B] = 0.0f; r0[3 * B] = 0.0f;
        float* r1 = R + 1 * 4 * B + tid;
        r1[0] = py; r1[B] = 0.0f; r1[2 * B] = 1.0f; r1[3 * B] = 0.0f;
        float* r2 = R + 2 * 4 * B + tid;
        r2[0] = pz; r2[B] = 0.0f; r2[2 * B] = 0.0f; r2[3 * B] = 1.0f;
        const bool live = stage.walk([&](uint8_t o, uint8_t kinds, uint16_t ro,
                                         uint16_t ra, uint16_t rb) {
            const D4 a = fetch_d(kinds & 3, ra, R, tid, B, cp);
            const D4 b = fetch_d((kinds >> 2) & 3, rb, R, tid, B, cp);
            const D4 d = dv_deriv(o, a, b, false);
            float* r = R + ro * 4 * B + tid;
            r[0] = d.v; r[B] = d.dx; r[2 * B] = d.dy; r[3 * B] = d.dz;
        });
        if (!live) return;
        if (ok) {
            const D4 d = fetch_d(t.root_kind, t.root, R, tid, B, cp);
            ov[i] = d.v;
            if (odx) odx[i] = d.dx;
            if (ody) ody[i] = d.dy;
            if (odz) odz[i] = d.dz;
        }
    }
    stage.finish();
}

__device__ __forceinline__ Iv fetch_i(uint8_t kind, uint16_t idx,
                                      const float* R, const uint8_t* N,
                                      int tid, int B,
                                      const float* __restrict__ cp)
{
    if (kind == OPND_REG) {
        return {R[idx * 2 * B + tid], R[idx * 2 * B + B + tid],
                N[idx * B + tid] != 0};
    }
    const float v = __ldg(cp + idx);
    return iv_make(v, v);
}

__global__ void __launch_bounds__(128)
k_intervals(DevTape t, uint32_t n,
            const float* __restrict__ xlo, const float* __restrict__ xhi,
            const float* __restrict__ ylo, const float* __restrict__ yhi,
            const float* __restrict__ zlo, const float* __restrict__ zhi,
            float* __restrict__ olo, float* __restrict__ ohi,
            uint8_t* __restrict__ onan)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int B = blockDim.x;
    const int tid = threadIdx.x;
    ClauseStage stage(t, smem_raw, block_passes(n, B));
    float* R = reinterpret_cast<float*>(smem_raw + stage_bytes(t.n));
    uint8_t* N = reinterpret_cast<uint8_t*>(R + t.n_regs * 2 * B);
    const float* __restrict__ cp = t.cpool;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * B;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * B + tid;
         i - tid < n; i += stride) {
        const bool ok = i < n;
        const float b[6] = {ok ? xlo[i] : 0.0f, ok ? xhi[i] : 0.0f,
                            ok ? ylo[i] : 0.0f, ok ? yhi[i] : 0.0f,
                            ok ? zlo[i] : 0.0f, ok ? zhi[i] : 0.0f};
        for (int a = 0; a < 3; ++a) {
            const Iv v = iv_make(b[2 * a], b[2 * a + 1]);
            R[a * 2 * B + tid] = v.lo;
            R[a * 2 * B + B + tid] = v.hi;
            N[a * B + tid] = v.nan;
        }
        const bool live = stage.walk([&](uint8_t o, uint8_t kinds, uint16_t ro,
                                         uint16_t ra, uint16_t rb) {
            const Iv a = fetch_i(kinds & 3, ra, R, N, tid, B, cp);
            const Iv bb = fetch_i((kinds >> 2) & 3, rb, R, N, tid, B, cp);
            const Iv r = iv_apply(o, a, bb);
            R[ro * 2 * B + tid] = r.lo;
            R[ro * 2 * B + B + tid] = r.hi;
            N[ro * B + tid] = r.nan;
        });
        if (!live) return;
        if (ok) {
            const Iv r = fetch_i(t.root_kind, t.root, R, N, tid, B, cp);
            olo[i] = r.lo;
            ohi[i] = r.hi;
            onan[i] = r.nan;
        }
    }
    stage.finish();
}

////////////////////////////////////////////////////////////////////////////////
// Launchers

static unsigned int* fault_pinned()
{
    static unsigned int* p = [] {
        void* q = nullptr;
        if (cudaHostAlloc(&q, sizeof(unsigned int), cudaHostAllocDefault) != cudaSuccess) {
            return static_cast<unsigned int*>(nullptr);
        }
        *static_cast<unsigned int*>(q) = 0;
        return static_cast<unsigned int*>(q);
    }();
    return p;
}

cudaError_t stage_fault_fetch(cudaStream_t s)
{
    unsigned int* p = fault_pinned();
    if (!p) return cudaErrorMemoryAllocation;
    return cudaMemcpyFromSymbolAsync(p, lfb_stage_fault, sizeof(unsigned int), 0,
                                     cudaMemcpyDeviceToHost, s);
}

bool stage_fault_take()
{
    unsigned int* p = fault_pinned();
    if (!p || *p == 0) return false;
    *p = 0;
    const unsigned int zero = 0;
    cudaMemcpyToSymbol(lfb_stage_fault, &zero, sizeof(zero));
    return true;
}

static int grid_for(uint64_t n, int block, int sm_count, int per_sm)
{
    const uint64_t blocks = (n + block - 1) / block;
    const uint64_t cap = static_cast<uint64_t>(sm_count) * per_sm;
    return static_cast<int>(blocks < cap ? (blocks ? blocks : 1) : cap);
}

int device_sm_count()
{
    static const int sms = [] {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n > 0 ? n : 1;
    }();
    return sms;
}

cudaError_t launch_values(const DevTape& t, uint32_t n, const float* x,
                          const float* y, const float* z, float* out,
                          cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    constexpr int PTS = 2;
    const int block = 128;
    const size_t planes = static_cast<size_t>(t.n_regs) * block * PTS * sizeof(float);
    if (planes > 200 * 1024) return cudaErrorInvalidConfiguration;
    const size_t smem = stage_bytes(t.n) + planes;
    if (!raise_smem_limit(reinterpret_cast<const void*>(k_values<PTS>), smem)) {
        return cudaErrorInvalidValue;
    }
    const int grid = grid_for((n + PTS - 1) / PTS, block, device_sm_count(), 16);
    k_values<PTS><<<grid, block, smem, s>>>(t, n, x, y, z, out);
    return cudaGetLastError();
}

cudaError_t launch_derivs(const DevTape& t, uint32_t n, const float* x,
                          const float* y, const float* z, float* v,
                          float* dx, float* dy, float* dz, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    const int block = 128;
    const size_t planes = static_cast<size_t>(t.n_regs) * block * 4 * sizeof(float);
    if (planes > 200 * 1024) return cudaErrorInvalidConfiguration;
    const size_t smem = stage_bytes(t.n) + planes;
    if (!raise_smem_limit(reinterpret_cast<const void*>(k_derivs), smem)) {
        return cudaErrorInvalidValue;
    }
    const int grid = grid_for(n, block, device_sm_count(), 16);
    k_derivs<<<grid, block, smem, s>>>(t, n, x, y, z, v, dx, dy, dz);
    return cudaGetLastError();
}

cudaError_t launch_intervals(const DevTape& t, uint32_t n, const float* xlo,
                             const float* xhi, const float* ylo,
                             const float* yhi, const float* zlo,
                             const float* zhi, float* olo, float* ohi,
                             uint8_t* onan, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    const int block = 128;
    const size_t planes = static_cast<size_t>(t.n_regs) * block * (2 * sizeof(float) + 1);
    if (planes > 200 * 1024) return cudaErrorInvalidConfiguration;
    const size_t smem = stage_bytes(t.n) + planes;
    if (!raise_smem_limit(reinterpret_cast<const void*>(k_intervals), smem)) {
        return cudaErrorInvalidValue;
    }
    const int grid = grid_for(n, block, device_sm_count(), 16);
    k_intervals<<<grid, block, smem, s>>>(t, n, xlo, xhi, ylo, yhi, zlo, zhi,
                                          olo, ohi, onan);
    return cudaGetLastError();
}

}  // namespace lfb
