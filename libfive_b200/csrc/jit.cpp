#include "jit.hpp"

#include <cuda.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "opcode.hpp"
#include "tape.hpp"

namespace lfb {

int device_sm_count();   // eval_kernels.cu

namespace {

/// NVRTC and the driver's module calls, looked up at run time so that the
/// library loads (and its interpreter runs) where either is missing.
struct Api {
    bool ok = false;
    nvrtcResult (*create)(nvrtcProgram*, const char*, const char*, int, const char* const*,
                          const char* const*) = nullptr;
    nvrtcResult (*compile)(nvrtcProgram, int, const char* const*) = nullptr;
    nvrtcResult (*cubin_size)(nvrtcProgram, size_t*) = nullptr;
    nvrtcResult (*cubin)(nvrtcProgram, char*) = nullptr;
    nvrtcResult (*destroy)(nvrtcProgram*) = nullptr;
    CUresult (*load)(CUmodule*, const void*) = nullptr;
    CUresult (*function)(CUfunction*, CUmodule, const char*) = nullptr;
    CUresult (*unload)(CUmodule) = nullptr;
    CUresult (*launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                       unsigned, CUstream, void**, void**) = nullptr;
};

const Api& api()
{
    static const Api a = [] {
        Api r;
        const char* e = std::getenv("LFB_JIT");
        if (e && e[0] == '0') return r;
        void* rtc = dlopen("libnvrtc.so.12", RTLD_NOW | RTLD_LOCAL);
        if (!rtc) rtc = dlopen("/usr/local/cuda/lib64/libnvrtc.so.12", RTLD_NOW | RTLD_LOCAL);
        void* drv = dlopen("libcuda.so.1", RTLD_NOW | RTLD_LOCAL);
        if (!rtc || !drv) return r;
        auto get = [](void* h, const char* name, auto& fn) {
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
            return fn != nullptr;
        };
        r.ok = get(rtc, "nvrtcCreateProgram", r.create) &&
               get(rtc, "nvrtcCompileProgram", r.compile) &&
               get(rtc, "nvrtcGetCUBINSize", r.cubin_size) &&
               get(rtc, "nvrtcGetCUBIN", r.cubin) &&
               get(rtc, "nvrtcDestroyProgram", r.destroy) &&
               get(drv, "cuModuleLoadData", r.load) &&
               get(drv, "cuModuleGetFunction", r.function) &&
               get(drv, "cuModuleUnload", r.unload) &&
               get(drv, "cuLaunchKernel", r.launch);
        return r;
    }();
    return a;
}

/// The value expression of one opcode, written with the same separately
/// rounded operations as dv_value; empty for opcodes left to the
/// interpreter.
std::string expr(uint8_t o, const std::string& a, const std::string& b)
{
    switch (o) {
        case op::ADD: return "__fadd_rn(" + a + ", " + b + ")";
        case op::SUB: return "__fsub_rn(" + a + ", " + b + ")";
        case op::MUL: return "__fmul_rn(" + a + ", " + b + ")";
        case op::DIV: return "__fdiv_rn(" + a + ", " + b + ")";
        case op::MIN: return "((" + b + ") < (" + a + ") ? (" + b + ") : (" + a + "))";
        case op::MAX: return "((" + a + ") < (" + b + ") ? (" + b + ") : (" + a + "))";
        case op::SQUARE: return "__fmul_rn(" + a + ", " + a + ")";
        case op::SQRT: return "__fsqrt_rn(" + a + ")";
        case op::NEG: return "(-(" + a + "))";
        case op::LOG: return "logf(" + a + ")";
        case op::EXP: return "expf(" + a + ")";
        case op::ABS: return "fabsf(" + a + ")";
        case op::RECIP: return "__fdiv_rn(1.0f, " + a + ")";
        case op::CONST_VAR: return "(" + a + ")";
        default: return std::string();
    }
}

std::string operand(const RegTape& t, uint32_t kind, uint32_t idx)
{
    if (kind == OPND_REG) return "r" + std::to_string(idx);
    if (kind == OPND_VAR) return "__ldg(cp + " + std::to_string(idx) + ")";
    uint32_t bits;
    std::memcpy(&bits, &t.cpool[idx], 4);
    char buf[40];
    std::snprintf(buf, sizeof(buf), "__uint_as_float(0x%08xu)", bits);
    return buf;
}

/// CUDA source of the tape's value kernel, or empty when an opcode has no
/// compiled form.  Registers of the tape become local variables; constants
/// are literals (bit patterns), free variables are read from the constant
/// pool so that they can change without recompiling.
std::string source(const RegTape& t)
{
    std::string s;
    s.reserve(64 * t.clauses.size() + 1024);
    s += "extern \"C\" __global__ void __launch_bounds__(256)\n"
         "lfb_tape_values(const float* __restrict__ X, const float* __restrict__ Y,\n"
         "                const float* __restrict__ Z, float* __restrict__ out,\n"
         "                unsigned long long n, const float* __restrict__ cp)\n{\n"
         "    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;\n"
         "    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + "
         "threadIdx.x;\n         i < n; i += stride) {\n"
         "        float r0 = X[i], r1 = Y[i], r2 = Z[i];\n";
    for (uint32_t r = 3; r < t.n_regs; ++r) {
        s += "        float r" + std::to_string(r) + " = 0.0f;\n";
    }
    for (const RegClause& c : t.clauses) {
        const std::string a = operand(t, c.kinds & 3, c.a);
        const std::string b = operand(t, (c.kinds >> 2) & 3, c.b);
        const std::string e = expr(c.op, a, b);
        if (e.empty()) return std::string();
        s += "        r" + std::to_string(c.out) + " = " + e + ";\n";
    }
    s += "        out[i] = " + operand(t, t.root_kind, t.root) + ";\n    }\n}\n";
    return s;
}

bool build(GpuTape& g)
{
    const Api& A = api();
    if (!A.ok || g.reg.clauses.size() > kJitMaxClauses) return false;
    const std::string src = source(g.reg);
    if (src.empty()) return false;
    nvrtcProgram prog = nullptr;
    if (A.create(&prog, src.c_str(), "lfb_tape.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
        return false;
    }
    const char* opts[] = {"--gpu-architecture=sm_100a", "-fmad=false", "--std=c++17"};
    bool ok = A.compile(prog, 3, opts) == NVRTC_SUCCESS;
    std::vector<char> cubin;
    size_t size = 0;
    ok = ok && A.cubin_size(prog, &size) == NVRTC_SUCCESS && size > 0;
    if (ok) {
        cubin.resize(size);
        ok = A.cubin(prog, cubin.data()) == NVRTC_SUCCESS;
    }
    A.destroy(&prog);
    if (!ok) return false;
    CUmodule mod = nullptr;
    CUfunction fn = nullptr;
    if (A.load(&mod, cubin.data()) != CUDA_SUCCESS) return false;
    if (A.function(&fn, mod, "lfb_tape_values") != CUDA_SUCCESS) {
        A.unload(mod);
        return false;
    }
    g.jit_module = mod;
    g.jit_function = fn;
    return true;
}

}  // namespace

bool jit_values(GpuTape& g, uint64_t n, const float* x, const float* y, const float* z,
                float* out, cudaStream_t s)
{
    {
        std::lock_guard<std::mutex> lock(g.mu);
        if (g.jit_state == 0) g.jit_state = build(g) ? 1 : -1;
        if (g.jit_state != 1) return false;
    }
    if (n == 0) return true;
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256,
                                               static_cast<uint64_t>(device_sm_count()) * 16);
    unsigned long long nn = n;
    const float* cp = g.d_cpool;
    void* args[] = {&x, &y, &z, &out, &nn, &cp};
    if (api().launch(static_cast<CUfunction>(g.jit_function), static_cast<unsigned>(blocks), 1,
                     1, 256, 1, 1, 0, reinterpret_cast<CUstream>(s), args,
                     nullptr) != CUDA_SUCCESS) {
        return false;
    }
    note_launches(1);
    return true;
}

void jit_release(GpuTape& g)
{
    if (g.jit_module && api().ok) api().unload(static_cast<CUmodule>(g.jit_module));
    g.jit_module = nullptr;
    g.jit_function = nullptr;
}

}  // namespace lfb
