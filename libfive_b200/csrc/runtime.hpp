// Host runtime: device tapes, error state, scratch buffers.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "dev_tape.h"
#include "tape.hpp"
#include "tree.hpp"

namespace lfb {

/// Records the failure for lfb_last_error and returns `code`.
int set_error(int code, const std::string& msg);
void clear_error();
int last_error(std::string* msg);

/// Fails with LFB_E_CUDA unless a CUDA device is usable.  There is no CPU
/// path: every evaluation in this library runs on the GPU.
bool require_device();

/// Converts a CUDA status into an error record; returns true on success.
bool cuda_ok(cudaError_t e, const char* what);

/// A tree flattened into both tape layouts, resident on the device.
struct GpuTape {
    Tree tree;
    SlotTape slot;
    RegTape reg;
    RegClause* d_clauses = nullptr;
    float* d_cpool = nullptr;
    std::mutex mu;   // guards cpool updates and the level-ordered copy

    // Level-ordered copy of the tape for the mesher's interval stage, built
    // on first use (build_wide_list).
    WideEntry* d_wide = nullptr;
    uint32_t wide_root = 0;
    bool wide_ready = false;
    bool ensure_wide();

    // Reverse mode: where each clause's local partials are stored per point
    // (slot | kind << 28, see grad_kernels.cu), built on first use.
    uint32_t* d_pslot = nullptr;
    std::vector<uint32_t> h_pslot;
    uint32_t n_pslot = 0;
    bool pslot_ready = false;

    // Compiled kernels (jit.cpp), [0] values, [1] values + derivatives,
    // [2] reverse-mode partials, [3] reverse-mode backward pass,
    // [4] intervals:
    // state 0 not tried, 1 ready, -1 none.
    struct JitKernel {
        int state = 0;
        void* module = nullptr;
        void* function = nullptr;
    };
    // [5] / [6] checkpointed reverse mode, forward / backward
    JitKernel jit[7];
    uint32_t ckpt_floats = 0;   // checkpoint slots per point (0: not prepared)

    // The CUDA device that was current when the tape was made: its arrays
    // live there, so every call must run with that device current.
    int device = -1;
    /// False (with an LFB_E_INVALID error recorded) unless the current
    /// device is the tape's.
    bool on_current_device() const;

    // Set when a kernel (the fit step, fit.cu) has written the variable
    // slots of d_cpool, so that the host copy in reg.cpool is out of date.
    bool vars_on_device = false;

    ~GpuTape();
    DevTape dev() const;
    /// Sets variable values by tree id; returns true if any value changed.
    bool set_vars(const void* const* ids, const float* values, uint32_t n);
    bool upload_cpool();
    /// Copies the device's variable values into reg.cpool when a kernel has
    /// changed them (waits for the device).  Call with `mu` held.
    bool pull_vars();
};

std::shared_ptr<GpuTape> make_tape(const Tree& t);

/// Cached device tape for a C API tree handle (free variables at zero).
std::shared_ptr<GpuTape> cached_tape(const Node* root);
void invalidate_cached(const Node* root);

/// Test hooks (lfb_debug_set): the number of device allocations left before
/// one is made to fail (0: none is), and whether meshes start from minimal
/// capacities.
struct DebugHooks {
    std::atomic<int64_t> fail_alloc_after{0};
    std::atomic<int> small_capacity{0};
};
DebugHooks& debug_hooks();
/// False when the allocation-failure hook says this allocation must fail.
bool debug_alloc_allowed();
/// Whether a scratch allocation of this thread ran the device out of memory
/// since the last call (injected failures do not count); clears the flag.
bool take_device_oom();
/// Records that an allocation outside DevBuf found the device out of memory.
void note_device_oom();

/// Growable device buffer.  With `ordered` set, it is allocated and freed
/// in stream order on `stream` (cudaMallocAsync / cudaFreeAsync from the
/// device's memory pool): no device-wide synchronisation, and memory a
/// buffer gives back is reused by the other streams' buffers.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    bool ordered = false;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf();
    bool reserve(size_t n);
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};

/// Keeps up to `bytes` of freed memory cached in the current device's
/// default memory pool across synchronisations (once per device).
void keep_pool_memory(uint64_t bytes);

/// Lets `fn` (a __global__ function) be launched with `bytes` of dynamic
/// shared memory on the current device.  The limit only ever rises, under a
/// lock, so that a thread that has raised it for its launch cannot have it
/// lowered by another thread between the raise and the launch.
bool raise_smem_limit(const void* fn, size_t bytes);

/// Counts kernel launches of this library (reported by lfb_kernel_launches).
void note_launches(uint64_t n);
uint64_t launches();

/// Serialises use of the library's default stream and scratch buffers.
std::mutex& global_mutex();

}  // namespace lfb
