// Clause stream staged in shared memory by bulk asynchronous copies (TMA).
//
// The batched interpreters (k_values / k_derivs / k_intervals) walk one tape
// with every thread of a block.  Instead of each warp fetching every clause
// through the read-only cache, one thread per block copies the tape into
// shared memory with cp.async.bulk (completion counted on an mbarrier), and
// every thread reads its clauses from there.  Replaces the clause fetch of
// the per-clause loops in ArrayEvaluator::values (libfive/src/eval/
// eval_array.cpp:112-114), DerivArrayEvaluator::derivs (eval_deriv_array.cpp:
// 101-117) and IntervalEvaluator::eval (eval_interval.cpp:68-93).
//
// Two forms, by tape length:
//  * resident (at most kResidentClauses clauses): the whole tape is copied
//    once when the block starts and stays for all of the block's
//    grid-stride passes; after the first wait no walk synchronises.
//  * streamed (longer tapes): chunks of kStageClauses clauses go through a
//    two-slot ring, one chunk ahead of the threads that read it.  Chunk j
//    of a block's walk (counted over all of its passes) sits in slot j & 1
//    and completes phase j >> 1 of that slot's mbarrier.  The copy of chunk
//    j + 1 is issued when chunk j is about to be read; its slot last held
//    chunk j - 1, which every thread finished before the block barrier that
//    ends chunk j - 1.
//
// Layout in dynamic shared memory: the clause buffer (stage_bytes(n) -
// 16 bytes), then 2 mbarriers, then the kernel's register planes.  Copies
// are tape-aligned: the tape's device allocation is padded to an even clause
// count, so every copy is a multiple of 16 bytes from a 16-byte aligned
// address.  Waits are bounded: a copy that does not land within the limit
// sets lfb_stage_fault and the block returns after waiting (again bounded)
// for its other copy in flight.
#pragma once
#include <cstdint>

#include "dev_tape.h"

namespace lfb {

constexpr uint32_t kStageClauses = 512;
constexpr uint32_t kResidentClauses = 2048;

// Set (to 1) by a block whose clause copy did not complete in time (one
// per translation unit that includes this header; the file that launches
// the kernels reads and clears it).
static __device__ unsigned int lfb_stage_fault = 0;

/// Shared memory of the clause buffer and its mbarriers for a tape of n
/// clauses (a multiple of 16 bytes).
__host__ __device__ constexpr size_t stage_bytes(uint32_t n)
{
    return (n <= kResidentClauses ? ((n + 1) & ~1u) : 2 * kStageClauses) * sizeof(RegClause) +
           2 * sizeof(uint64_t);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    for (uint32_t k = 0; k < (1u << 20); ++k) {
        if (mbar_try_wait(bar, parity)) return true;
    }
    return false;
}

class ClauseStage {
public:
    // Called by every thread of the block before the first walk.  `passes`
    // = how many times this block walks the whole tape.
    __device__ ClauseStage(const DevTape& t, void* smem, uint32_t passes)
        : src_(t.clauses), n_(t.n),
          ring_(static_cast<RegClause*>(smem)),
          bar_(reinterpret_cast<uint64_t*>(static_cast<unsigned char*>(smem) +
                                            stage_bytes(t.n) - 2 * sizeof(uint64_t))),
          resident_(t.n <= kResidentClauses),
          chunks_(t.n <= kResidentClauses ? (t.n ? 1 : 0)
                                          : (t.n + kStageClauses - 1) / kStageClauses),
          total_(resident_ ? chunks_ * (passes ? 1 : 0) : chunks_ * passes), j_(0)
    {
        if (threadIdx.x == 0) {
            for (int s = 0; s < 2; ++s) {
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;"
                             :: "r"(smem_addr(bar_ + s)) : "memory");
            }
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        if (threadIdx.x == 0 && total_ > 0) issue(0);
    }

    // Walks the whole tape once, calling f(op, kinds, out, a, b) per clause
    // in order.  Returns false (every thread of the block alike) when a copy
    // timed out; the caller then returns without writing results.
    template <class F>
    __device__ __forceinline__ bool walk(F&& f)
    {
        if (resident_) {
            if (j_ < total_) {   // the first walk waits for the copy
                const bool ok = mbar_wait_bounded(bar_, 0);
                if (__syncthreads_or(!ok)) {
                    give_up();
                    return false;
                }
                j_ = total_;
            }
            const uint2* c = reinterpret_cast<const uint2*>(ring_);
            for (uint32_t k = 0; k < n_; ++k) run(f, c[k]);
            return true;
        }
        for (uint32_t ck = 0; ck < chunks_; ++ck, ++j_) {
            if (threadIdx.x == 0 && j_ + 1 < total_) issue(j_ + 1);
            const bool ok = mbar_wait_bounded(bar_ + (j_ & 1), (j_ >> 1) & 1);
            if (__syncthreads_or(!ok)) {
                give_up();
                return false;
            }
            const uint2* c = reinterpret_cast<const uint2*>(ring_ + (j_ & 1) * kStageClauses);
            const uint32_t m = min(kStageClauses, n_ - ck * kStageClauses);
            for (uint32_t k = 0; k < m; ++k) run(f, c[k]);
            __syncthreads();
        }
        return true;
    }

    // At the end of the kernel: a chunk issued but never walked (only when
    // the caller walked fewer times than it announced) is waited for, so no
    // copy is in flight when the block exits.
    __device__ __forceinline__ void finish()
    {
        if (threadIdx.x == 0 && j_ < total_) {
            mbar_wait_bounded(bar_ + (j_ & 1), (j_ >> 1) & 1);
        }
    }

private:
    template <class F>
    __device__ __forceinline__ static void run(F& f, const uint2 raw)
    {
        f(static_cast<uint8_t>(raw.x & 0xff),
          static_cast<uint8_t>((raw.x >> 8) & 0xff),
          static_cast<uint16_t>(raw.x >> 16),
          static_cast<uint16_t>(raw.y & 0xffff),
          static_cast<uint16_t>(raw.y >> 16));
    }

    __device__ __forceinline__ void issue(uint32_t j)
    {
        const uint32_t ck = j % chunks_;
        const uint32_t first = ck * kStageClauses;
        const uint32_t m = resident_ ? n_ : min(kStageClauses, n_ - first);
        const uint32_t bytes = ((m + 1) & ~1u) * static_cast<uint32_t>(sizeof(RegClause));
        uint64_t* bar = bar_ + (j & 1);
        RegClause* dst = resident_ ? ring_ : ring_ + (j & 1) * kStageClauses;
        // the slot's previous contents were read through the generic proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                     :: "r"(smem_addr(bar)), "r"(bytes) : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
            " [%0], [%1], %2, [%3];"
            :: "r"(smem_addr(dst)), "l"(src_ + first), "r"(bytes), "r"(smem_addr(bar))
            : "memory");
    }

    // After a timed-out wait on chunk j_: the copy of chunk j_ + 1 may be in
    // flight too; wait for it (bounded) before the block leaves.
    __device__ void give_up()
    {
        if (threadIdx.x == 0) {
            atomicExch(&lfb_stage_fault, 1u);
            const uint32_t nx = j_ + 1;
            if (!resident_ && nx < total_) mbar_wait_bounded(bar_ + (nx & 1), (nx >> 1) & 1);
            mbar_wait_bounded(bar_ + (j_ & 1), (j_ >> 1) & 1);
        }
        __syncthreads();
    }

    const RegClause* src_;
    uint32_t n_;
    RegClause* ring_;
    uint64_t* bar_;
    bool resident_;
    uint32_t chunks_;
    uint32_t total_;
    uint32_t j_;
};

// How many grid-stride passes a block makes over `n` items, `per_pass`
// items per block pass.
__device__ __forceinline__ uint32_t block_passes(uint64_t n, uint64_t per_pass)
{
    const uint64_t first = static_cast<uint64_t>(blockIdx.x) * per_pass;
    if (first >= n) return 0;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * per_pass;
    return static_cast<uint32_t>((n - 1 - first) / stride + 1);
}

}  // namespace lfb
