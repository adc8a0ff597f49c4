#include "runtime.hpp"

#include "jit.hpp"

#include <map>

#include <atomic>
#include <cstdio>

#include "libfive_b200.h"

namespace lfb {

// Set when a scratch allocation found the device out of memory (not an
// injected failure); read and cleared by take_device_oom.
thread_local bool t_device_oom = false;


static thread_local int t_code = 0;
static thread_local std::string t_msg;

int set_error(int code, const std::string& msg)
{
    t_code = code;
    t_msg = msg;
    return code;
}

void clear_error()
{
    t_code = 0;
    t_msg.clear();
}

int last_error(std::string* msg)
{
    if (msg) *msg = t_msg;
    return t_code;
}

bool cuda_ok(cudaError_t e, const char* what)
{
    if (e == cudaSuccess) {
        return true;
    }
    set_error(LFB_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

bool require_device()
{
    static const int state = [] {   // 0 none, 1 ok
        int n = 0;
        const cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess || n <= 0) {
            cudaGetLastError();
            return 0;
        }
        return 1;
    }();
    if (!state) {
        set_error(LFB_E_CUDA,
                  "no CUDA device: libfive_b200 evaluates on the GPU only");
        return false;
    }
    return true;
}

bool raise_smem_limit(const void* fn, size_t bytes)
{
    if (bytes <= 48 * 1024) return true;
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> limits;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = limits[{dev, fn}];
    if (bytes <= cur) return true;
    if (!cuda_ok(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(bytes)),
                 "shared memory size")) {
        return false;
    }
    cur = bytes;
    return true;
}

static std::atomic<uint64_t> g_launches{0};
void note_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t launches() { return g_launches.load(std::memory_order_relaxed); }

std::mutex& global_mutex()
{
    static std::mutex m;
    return m;
}

GpuTape::~GpuTape()
{
    if (d_clauses) cudaFree(d_clauses);
    if (d_cpool) cudaFree(d_cpool);
    if (d_wide) cudaFree(d_wide);
    if (d_pslot) cudaFree(d_pslot);
    jit_release(*this);
}

bool GpuTape::ensure_wide()
{
    std::lock_guard<std::mutex> lock(mu);
    if (wide_ready) return true;
    std::vector<WideEntry> w;
    std::string err;
    if (!build_wide_list(reg, w, wide_root, &err)) {
        set_error(LFB_E_UNSUPPORTED, err);
        return false;
    }
    const size_t bytes = std::max<size_t>(w.size(), 1) * sizeof(WideEntry);
    if (!cuda_ok(cudaMalloc(&d_wide, bytes), "level-ordered tape alloc")) return false;
    if (!w.empty() &&
        !cuda_ok(cudaMemcpy(d_wide, w.data(), w.size() * sizeof(WideEntry),
                            cudaMemcpyHostToDevice), "level-ordered tape upload")) {
        return false;
    }
    wide_ready = true;
    return true;
}

DevTape GpuTape::dev() const
{
    DevTape d;
    d.clauses = d_clauses;
    d.n = static_cast<uint32_t>(reg.clauses.size());
    d.cpool = d_cpool;
    d.n_cpool = static_cast<uint32_t>(reg.cpool.size());
    d.n_const = reg.n_const;
    d.n_regs = reg.n_regs;
    d.n_choices = reg.n_choices;
    d.root_kind = reg.root_kind;
    d.root = reg.root;
    return d;
}

bool GpuTape::upload_cpool()
{
    if (reg.cpool.empty()) return true;
    return cuda_ok(cudaMemcpy(d_cpool, reg.cpool.data(),
                              reg.cpool.size() * sizeof(float),
                              cudaMemcpyHostToDevice),
                   "upload constants");
}

bool GpuTape::pull_vars()
{
    if (!vars_on_device) return true;
    if (reg.n_vars &&
        (!cuda_ok(cudaDeviceSynchronize(), "variable download") ||
         !cuda_ok(cudaMemcpy(reg.cpool.data() + reg.n_const, d_cpool + reg.n_const,
                             reg.n_vars * sizeof(float), cudaMemcpyDeviceToHost),
                  "variable download"))) {
        return false;
    }
    vars_on_device = false;
    return true;
}

bool GpuTape::set_vars(const void* const* ids, const float* values,
                       uint32_t n)
{
    bool changed = false;
    for (uint32_t i = 0; i < n; ++i) {
        for (uint32_t k = 0; k < reg.n_vars; ++k) {
            if (reg.var_nodes[k] == ids[i]) {
                float& slot = reg.cpool[reg.n_const + k];
                if (slot != values[i]) {
                    changed = true;
                }
                slot = values[i];
            }
        }
    }
    return changed;
}

std::shared_ptr<GpuTape> make_tape(const Tree& t)
{
    if (!require_device()) {
        return nullptr;
    }
    if (!t.is_valid()) {
        set_error(LFB_E_INVALID, "invalid tree");
        return nullptr;
    }
    auto g = std::make_shared<GpuTape>();
    g->tree = t;
    if (!cuda_ok(cudaGetDevice(&g->device), "cudaGetDevice")) return nullptr;
    std::string err;
    if (!build_slot_tape(t, g->slot, &err) ||
        !build_reg_tape(g->slot, g->reg, &err)) {
        set_error(LFB_E_UNSUPPORTED, err);
        return nullptr;
    }
    // an even clause count: the batched interpreters copy the tape to shared
    // memory in 16-byte multiples
    const size_t nc = std::max<size_t>(2, (g->reg.clauses.size() + 1) & ~size_t(1));
    const size_t np = std::max<size_t>(1, g->reg.cpool.size());
    if (!cuda_ok(cudaMalloc(&g->d_clauses, nc * sizeof(RegClause)), "tape alloc") ||
        !cuda_ok(cudaMalloc(&g->d_cpool, np * sizeof(float)), "tape alloc")) {
        return nullptr;
    }
    if (!g->reg.clauses.empty() &&
        !cuda_ok(cudaMemcpy(g->d_clauses, g->reg.clauses.data(),
                            g->reg.clauses.size() * sizeof(RegClause),
                            cudaMemcpyHostToDevice),
                 "tape upload")) {
        return nullptr;
    }
    if (!g->upload_cpool()) {
        return nullptr;
    }
    return g;
}

static std::mutex g_cache_mu;
static std::unordered_map<const Node*, std::shared_ptr<GpuTape>> g_cache;

bool GpuTape::on_current_device() const
{
    int cur = -1;
    if (!cuda_ok(cudaGetDevice(&cur), "cudaGetDevice")) return false;
    if (cur != device) {
        set_error(LFB_E_INVALID, "the tape was made on CUDA device " + std::to_string(device) +
                                     " but device " + std::to_string(cur) + " is current");
        return false;
    }
    return true;
}

std::shared_ptr<GpuTape> cached_tape(const Node* root)
{
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) cur = -1;
    {
        std::lock_guard<std::mutex> lock(g_cache_mu);
        auto it = g_cache.find(root);
        // a tape made on another device is replaced by one on this device
        if (it != g_cache.end() && it->second->device == cur) {
            return it->second;
        }
    }
    auto g = make_tape(Tree(root));
    if (g) {
        std::lock_guard<std::mutex> lock(g_cache_mu);
        if (g_cache.size() > 4096) {
            g_cache.clear();
        }
        g_cache[root] = g;
    }
    return g;
}

void invalidate_cached(const Node* root)
{
    std::lock_guard<std::mutex> lock(g_cache_mu);
    g_cache.erase(root);
}

DevBuf::~DevBuf()
{
    if (!ptr) return;
    if (ordered) cudaFreeAsync(ptr, stream);
    else cudaFree(ptr);
}

void keep_pool_memory(uint64_t bytes)
{
    static std::mutex mu;
    static uint64_t done = 0;   // one bit per device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 64 && ((done >> dev) & 1)) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &bytes);
    }
    cudaGetLastError();
    if (dev < 64) done |= 1ull << dev;
}

DebugHooks& debug_hooks()
{
    static DebugHooks h;
    return h;
}

void note_device_oom() { t_device_oom = true; }

bool take_device_oom()
{
    const bool r = t_device_oom;
    t_device_oom = false;
    return r;
}

bool debug_alloc_allowed()
{
    auto& h = debug_hooks().fail_alloc_after;
    int64_t left = h.load();
    while (left > 0) {
        if (h.compare_exchange_weak(left, left - 1)) {
            if (left == 1) {
                set_error(LFB_E_CUDA, "scratch alloc: out of memory (failure injected by lfb_debug_set)");
                return false;
            }
            return true;
        }
    }
    return true;
}

bool DevBuf::reserve(size_t n)
{
    if (n <= bytes) return true;
    if (ptr) {
        if (ordered) cudaFreeAsync(ptr, stream);
        else cudaFree(ptr);
    }
    ptr = nullptr;
    bytes = 0;
    const size_t want = std::max<size_t>(n, 256);
    if (!debug_alloc_allowed()) return false;
    const cudaError_t e = ordered ? cudaMallocAsync(&ptr, want, stream) : cudaMalloc(&ptr, want);
    if (e == cudaErrorMemoryAllocation) t_device_oom = true;
    if (!cuda_ok(e, "scratch alloc")) {
        return false;
    }
    bytes = want;
    return true;
}

}  // namespace lfb
