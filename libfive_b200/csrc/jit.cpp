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

// The headers run-time compiled kernels include (generated by build.py).
extern const int kJitHeaderCount;
extern const char* const kJitHeaderNames[];
extern const char* const kJitHeaderSources[];

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
    nvrtcResult (*log_size)(nvrtcProgram, size_t*) = nullptr;
    nvrtcResult (*log)(nvrtcProgram, char*) = nullptr;
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
        auto get = [](void* h, const char* name, auto& fn) {
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
            return fn != nullptr;
        };
        void* rtc = dlopen("libnvrtc.so.12", RTLD_NOW | RTLD_LOCAL);
        if (!rtc) rtc = dlopen("/usr/local/cuda/lib64/libnvrtc.so.12", RTLD_NOW | RTLD_LOCAL);
        if (!rtc) return r;
        const bool rtc_ok = get(rtc, "nvrtcCreateProgram", r.create) &&
                            get(rtc, "nvrtcCompileProgram", r.compile) &&
                            get(rtc, "nvrtcGetCUBINSize", r.cubin_size) &&
                            get(rtc, "nvrtcGetCUBIN", r.cubin) &&
                            get(rtc, "nvrtcDestroyProgram", r.destroy) &&
                            get(rtc, "nvrtcGetProgramLogSize", r.log_size) &&
                            get(rtc, "nvrtcGetProgramLog", r.log);
        if (!rtc_ok) {
            r.create = nullptr;
            return r;
        }
        // The driver's module calls: only on a machine with a GPU driver
        // (compilation alone works without one).
        void* drv = dlopen("libcuda.so.1", RTLD_NOW | RTLD_LOCAL);
        r.ok = drv && get(drv, "cuModuleLoadData", r.load) &&
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
        default:
            // the remaining opcodes through the interpreter's own function
            if (op::arity(o) < 1) return std::string();
            return "dv_value(" + std::to_string(o) + ", " + a + ", " + b + ")";
    }
}

/// Common start of every generated source: the point and interval rules of
/// the interpreters (dev_point.cuh, dev_interval.cuh), included from text
/// built into the library.
const char* kPrelude =
    "typedef unsigned char uint8_t;\ntypedef unsigned short uint16_t;\n"
    "typedef unsigned int uint32_t;\ntypedef unsigned long long uint64_t;\n"
    "typedef int int32_t;\ntypedef long long int64_t;\n"
    "#include \"dev_point.cuh\"\n#include \"dev_interval.cuh\"\nusing namespace lfb;\n";

/// Second operand of a clause: unary clauses get a zero (their rules never
/// read it).
uint32_t b_kind(const RegClause& c) { return op::arity(c.op) == 2 ? (c.kinds >> 2) & 3 : 99u; }

std::string operand(const RegTape& t, uint32_t kind, uint32_t idx)
{
    if (kind == 99u) return "0.0f";
    if (kind == OPND_REG) return "r" + std::to_string(idx);
    if (kind == OPND_VAR) return "__ldg(cp + " + std::to_string(idx) + ")";
    uint32_t bits;
    std::memcpy(&bits, &t.cpool[idx], 4);
    char buf[40];
    std::snprintf(buf, sizeof(buf), "__uint_as_float(0x%08xu)", bits);
    return buf;
}

/// Tangent c (0 = d/dx, 1 = d/dy, 2 = d/dz) of an operand: constants and
/// free variables have none.
std::string tangent(uint32_t kind, uint32_t idx, int c)
{
    if (kind != OPND_REG) return "0.0f";
    return "r" + std::to_string(idx) + "_" + "xyz"[c];
}

const char* kHead =
    "    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;\n"
    "    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + "
    "threadIdx.x;\n         i < n; i += stride) {\n";

/// CUDA source of the tape's value kernel, or empty when an opcode has no
/// compiled form.  Registers of the tape become local variables; constants
/// are literals (bit patterns), free variables are read from the constant
/// pool so that they can change without recompiling.
std::string values_source(const RegTape& t)
{
    std::string s;
    s.reserve(64 * t.clauses.size() + 1024);
    s += kPrelude;
    s += "extern \"C\" __global__ void __launch_bounds__(256)\n"
         "lfb_tape_values(const float* __restrict__ X, const float* __restrict__ Y,\n"
         "                const float* __restrict__ Z, float* __restrict__ out,\n"
         "                unsigned long long n, const float* __restrict__ cp)\n{\n";
    s += kHead;
    s += "        float r0 = X[i], r1 = Y[i], r2 = Z[i];\n";
    for (uint32_t r = 3; r < t.n_regs; ++r) {
        s += "        float r" + std::to_string(r) + " = 0.0f;\n";
    }
    for (const RegClause& c : t.clauses) {
        const std::string a = operand(t, c.kinds & 3, c.a);
        const std::string b = operand(t, b_kind(c), c.b);
        const std::string e = expr(c.op, a, b);
        if (e.empty()) return std::string();
        s += "        r" + std::to_string(c.out) + " = " + e + ";\n";
    }
    s += "        out[i] = " + operand(t, t.root_kind, t.root) + ";\n    }\n}\n";
    return s;
}

/// One clause of the derivative kernel: value and the three tangents by the
/// rules of dv_deriv (clear_vars off), through temporaries so that an output
/// register may also be an operand.  Empty for opcodes without a compiled form.
std::string deriv_clause(const RegTape& t, const RegClause& c)
{
    const uint32_t ka = c.kinds & 3, kb = b_kind(c);
    std::string s = "        {\n            const float a = " + operand(t, ka, c.a) +
                    ", b = " + operand(t, kb, c.b) + ";\n";
    for (int k = 0; k < 3; ++k) {
        s += std::string("            const float a") + "xyz"[k] + " = " + tangent(ka, c.a, k) +
             ", b" + "xyz"[k] + " = " + tangent(kb, c.b, k) + ";\n";
    }
    std::string v, d[3];
    std::string pre;
    switch (c.op) {
        case op::ADD:
            v = "__fadd_rn(a, b)";
            for (int k = 0; k < 3; ++k) d[k] = std::string("__fadd_rn(a") + "xyz"[k] + ", b" + "xyz"[k] + ")";
            break;
        case op::SUB:
            v = "__fsub_rn(a, b)";
            for (int k = 0; k < 3; ++k) d[k] = std::string("__fsub_rn(a") + "xyz"[k] + ", b" + "xyz"[k] + ")";
            break;
        case op::MUL:
            v = "__fmul_rn(a, b)";
            for (int k = 0; k < 3; ++k) {
                d[k] = std::string("__fadd_rn(__fmul_rn(b") + "xyz"[k] + ", a), __fmul_rn(a" +
                       "xyz"[k] + ", b))";
            }
            break;
        case op::DIV:
            pre = "            const float den = __fmul_rn(b, b);\n";
            v = "__fdiv_rn(a, b)";
            for (int k = 0; k < 3; ++k) {
                d[k] = std::string("__fdiv_rn(__fsub_rn(__fmul_rn(a") + "xyz"[k] +
                       ", b), __fmul_rn(b" + "xyz"[k] + ", a)), den)";
            }
            break;
        case op::MIN:
            v = "((b) < (a) ? (b) : (a))";
            for (int k = 0; k < 3; ++k) d[k] = std::string("(a < b ? a") + "xyz"[k] + " : b" + "xyz"[k] + ")";
            break;
        case op::MAX:
            v = "((a) < (b) ? (b) : (a))";
            for (int k = 0; k < 3; ++k) d[k] = std::string("(a < b ? b") + "xyz"[k] + " : a" + "xyz"[k] + ")";
            break;
        case op::SQUARE:
            v = "__fmul_rn(a, a)";
            for (int k = 0; k < 3; ++k) d[k] = std::string("__fmul_rn(__fmul_rn(a") + "xyz"[k] + ", a), 2.0f)";
            break;
        case op::SQRT:
            pre = "            const float ov = __fsqrt_rn(a);\n"
                  "            const float den = __fmul_rn(2.0f, ov);\n";
            v = "ov";
            for (int k = 0; k < 3; ++k) {
                const std::string t_ = std::string("a") + "xyz"[k];
                d[k] = "((a < 0 || " + t_ + " == 0) ? 0.0f : __fdiv_rn(" + t_ + ", den))";
            }
            break;
        case op::NEG:
            v = "(-a)";
            for (int k = 0; k < 3; ++k) d[k] = std::string("(-a") + "xyz"[k] + ")";
            break;
        case op::LOG:
            v = "logf(a)";
            for (int k = 0; k < 3; ++k) d[k] = std::string("__fdiv_rn(a") + "xyz"[k] + ", a)";
            break;
        case op::EXP:
            pre = "            const float e = expf(a);\n";
            v = "e";
            for (int k = 0; k < 3; ++k) d[k] = std::string("__fmul_rn(a") + "xyz"[k] + ", e)";
            break;
        case op::ABS:
            v = "fabsf(a)";
            for (int k = 0; k < 3; ++k) d[k] = std::string("(a > 0 ? a") + "xyz"[k] + " : -a" + "xyz"[k] + ")";
            break;
        case op::RECIP:
            pre = "            const float den = -__fmul_rn(a, a);\n";
            v = "__fdiv_rn(1.0f, a)";
            for (int k = 0; k < 3; ++k) d[k] = std::string("__fdiv_rn(a") + "xyz"[k] + ", den)";
            break;
        case op::CONST_VAR:
            v = "a";
            for (int k = 0; k < 3; ++k) d[k] = std::string("a") + "xyz"[k];
            break;
        default:
            // the remaining opcodes through the interpreter's own rules
            if (op::arity(c.op) < 1) return std::string();
            pre = "            const D4 dd = dv_deriv_all(" + std::to_string(c.op) +
                  ", D4{a, ax, ay, az}, D4{b, bx, by, bz}, false);\n";
            v = "dd.v";
            d[0] = "dd.dx";
            d[1] = "dd.dy";
            d[2] = "dd.dz";
            break;
    }
    const std::string o = "r" + std::to_string(c.out);
    s += pre;
    s += "            " + o + " = " + v + ";\n";
    for (int k = 0; k < 3; ++k) s += "            " + o + "_" + "xyz"[k] + " = " + d[k] + ";\n";
    s += "        }\n";
    return s;
}

/// CUDA source of the tape's value + derivative kernel (or empty).
std::string derivs_source(const RegTape& t)
{
    std::string s;
    s.reserve(400 * t.clauses.size() + 2048);
    s += kPrelude;
    s += "extern \"C\" __global__ void __launch_bounds__(256)\n"
         "lfb_tape_derivs(const float* __restrict__ X, const float* __restrict__ Y,\n"
         "                const float* __restrict__ Z, float* __restrict__ ov,\n"
         "                float* __restrict__ odx, float* __restrict__ ody,\n"
         "                float* __restrict__ odz, unsigned long long n,\n"
         "                const float* __restrict__ cp)\n{\n";
    s += kHead;
    s += "        float r0 = X[i], r0_x = 1.0f, r0_y = 0.0f, r0_z = 0.0f;\n"
         "        float r1 = Y[i], r1_x = 0.0f, r1_y = 1.0f, r1_z = 0.0f;\n"
         "        float r2 = Z[i], r2_x = 0.0f, r2_y = 0.0f, r2_z = 1.0f;\n";
    for (uint32_t r = 3; r < t.n_regs; ++r) {
        const std::string n = "r" + std::to_string(r);
        s += "        float " + n + " = 0.0f, " + n + "_x = 0.0f, " + n + "_y = 0.0f, " + n +
             "_z = 0.0f;\n";
    }
    for (const RegClause& c : t.clauses) {
        const std::string cl = deriv_clause(t, c);
        if (cl.empty()) return std::string();
        s += cl;
    }
    const uint32_t rk = t.root_kind, ri = t.root;
    s += "        ov[i] = " + operand(t, rk, ri) + ";\n";
    s += "        if (odx) odx[i] = " + tangent(rk, ri, 0) + ";\n";
    s += "        if (ody) ody[i] = " + tangent(rk, ri, 1) + ";\n";
    s += "        if (odz) odz[i] = " + tangent(rk, ri, 2) + ";\n    }\n}\n";
    return s;
}

/// Reverse mode.  The slot table (slot | kind << 28) and the partial rules
/// are those of grad_kernels.cu: kind 0 fixed by the opcode, 1 a min/max
/// choice, 2 one partial, 3 two partials.
enum : uint32_t { RK_CONST = 0, RK_CHOICE = 1, RK_ONE = 2, RK_TWO = 3 };

/// Partials d out / d a, d out / d b of one clause as expressions of its
/// operand values `a`, `b` (and temporaries declared in `pre`), the results
/// of DerivArrayEvaluator's rules for unit tangents; false for opcodes
/// without a compiled form.
bool partial_exprs(uint8_t o, std::string* v, std::string* pa, std::string* pb, std::string* pre)
{
    *pb = "0.0f";
    switch (o) {
        case op::ADD: *v = "__fadd_rn(a, b)"; *pa = "1.0f"; *pb = "1.0f"; return true;
        case op::SUB: *v = "__fsub_rn(a, b)"; *pa = "1.0f"; *pb = "-1.0f"; return true;
        case op::NEG: *v = "(-a)"; *pa = "-1.0f"; return true;
        case op::CONST_VAR: *v = "a"; *pa = "1.0f"; return true;
        case op::MUL:
            *v = "__fmul_rn(a, b)";
            *pa = "__fadd_rn(__fmul_rn(0.0f, a), __fmul_rn(1.0f, b))";
            *pb = "__fadd_rn(__fmul_rn(1.0f, a), __fmul_rn(0.0f, b))";
            return true;
        case op::MIN: *v = "((b) < (a) ? (b) : (a))"; *pa = "(a < b ? 1.0f : 0.0f)"; return true;
        case op::MAX: *v = "((a) < (b) ? (b) : (a))"; *pa = "(a < b ? 0.0f : 1.0f)"; return true;
        case op::SQUARE: *v = "__fmul_rn(a, a)"; *pa = "__fmul_rn(a, 2.0f)"; return true;
        case op::ABS: *v = "fabsf(a)"; *pa = "(a > 0 ? 1.0f : -1.0f)"; return true;
        case op::SQRT:
            *pre = "const float ov = __fsqrt_rn(a); ";
            *v = "ov";
            *pa = "(a < 0 ? 0.0f : __fdiv_rn(1.0f, __fmul_rn(2.0f, ov)))";
            return true;
        case op::LOG: *v = "logf(a)"; *pa = "__fdiv_rn(1.0f, a)"; return true;
        case op::EXP:
            *pre = "const float e = expf(a); ";
            *v = "e";
            *pa = "__fmul_rn(1.0f, e)";
            return true;
        case op::RECIP:
            *v = "__fdiv_rn(1.0f, a)";
            *pa = "__fdiv_rn(1.0f, -__fmul_rn(a, a))";
            return true;
        case op::DIV:
            *pre = "const float den = __fmul_rn(b, b); ";
            *v = "__fdiv_rn(a, b)";
            *pa = "__fdiv_rn(__fsub_rn(__fmul_rn(1.0f, b), __fmul_rn(0.0f, a)), den)";
            *pb = "__fdiv_rn(__fsub_rn(__fmul_rn(0.0f, b), __fmul_rn(1.0f, a)), den)";
            return true;
        default:
            // the remaining opcodes through the interpreter's own rules
            if (op::arity(o) < 1) return false;
            *pre = "const D4 dd = dv_deriv_all(" + std::to_string(o) +
                   ", D4{a, 1.0f, 0.0f, 0.0f}, D4{b, 0.0f, 1.0f, 0.0f}, false); ";
            *v = "dd.v";
            *pa = "dd.dx";
            *pb = "dd.dy";
            return true;
    }
}

/// Forward pass of the reverse mode: values in registers, the partials the
/// slot table keeps written per point.
std::string partials_source(const RegTape& t, const std::vector<uint32_t>& slots)
{
    std::string s;
    s.reserve(160 * t.clauses.size() + 1024);
    s += kPrelude;
    s += "extern \"C\" __global__ void __launch_bounds__(256)\n"
         "lfb_tape_partials(const float* __restrict__ X, const float* __restrict__ Y,\n"
         "                  const float* __restrict__ Z, float* __restrict__ P,\n"
         "                  float* __restrict__ f, unsigned m, const float* __restrict__ cp)\n{\n"
         "    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;\n"
         "    if (i >= m) return;\n"
         "    float* const Pi = P + i;\n"
         "    float r0 = X[i], r1 = Y[i], r2 = Z[i];\n";
    for (uint32_t r = 3; r < t.n_regs; ++r) s += "    float r" + std::to_string(r) + " = 0.0f;\n";
    for (size_t c = 0; c < t.clauses.size(); ++c) {
        const RegClause& cl = t.clauses[c];
        std::string v, pa, pb, pre;
        if (!partial_exprs(cl.op, &v, &pa, &pb, &pre)) return std::string();
        const uint32_t kind = slots[c] >> 28, slot = slots[c] & 0x0fffffffu;
        s += "    { const float a = " + operand(t, cl.kinds & 3, cl.a) + ", b = " +
             operand(t, b_kind(cl), cl.b) + "; " + pre;
        if (kind != RK_CONST) {
            s += "Pi[(size_t)" + std::to_string(slot) + " * m] = " + pa + "; ";
            if (kind == RK_TWO) s += "Pi[(size_t)" + std::to_string(slot + 1) + " * m] = " + pb + "; ";
        }
        s += "r" + std::to_string(cl.out) + " = " + v + "; }\n";
    }
    s += "    if (f) f[i] = " + operand(t, t.root_kind, t.root) + ";\n}\n";
    return s;
}

/// Backward pass: one adjoint per tape register, clauses in reverse, the
/// same products and sums as the interpreted backward pass; variable
/// adjoints are summed over the warp, then over the block in shared memory.
std::string backward_source(const RegTape& t, const std::vector<uint32_t>& slots)
{
    std::string s;
    s.reserve(200 * t.clauses.size() + 2048);
    s += "__device__ __forceinline__ void lfb_add_var(float* Gv, unsigned k, float g)\n{\n"
         "    for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);\n"
         "    if ((threadIdx.x & 31) == 0 && g != 0.0f) atomicAdd(Gv + k, g);\n}\n"
         "extern \"C\" __global__ void __launch_bounds__(256)\n"
         "lfb_tape_backward(const float* __restrict__ P, const float* __restrict__ seed,\n"
         "                  float* __restrict__ gx, float* __restrict__ gy,\n"
         "                  float* __restrict__ gz, float* __restrict__ gvars, unsigned m,\n"
         "                  unsigned n_vars, int block_cv)\n{\n"
         "    extern __shared__ float Gv[];\n"
         "    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;\n"
         "    const bool ok = i < m;\n"
         "    const bool gv = gvars != nullptr;\n"
         "    if (gv) {\n"
         "        for (unsigned k = threadIdx.x; k < n_vars; k += blockDim.x) Gv[k] = 0.0f;\n"
         "        __syncthreads();\n    }\n"
         "    const float* const Pi = P + (ok ? i : 0);\n";
    for (uint32_t r = 0; r < t.n_regs; ++r) s += "    float a" + std::to_string(r) + " = 0.0f;\n";
    s += "    const float s0 = ok ? (seed ? seed[i] : 1.0f) : 0.0f;\n";
    if (t.root_kind == OPND_REG) {
        s += "    a" + std::to_string(t.root) + " = s0;\n";
    } else if (t.root_kind == OPND_VAR) {
        s += "    if (gv) lfb_add_var(Gv, " + std::to_string(t.root - t.n_const) + ", s0);\n";
    }
    // register adjoints: one fused multiply-add per operand (as the
    // interpreter); variable adjoints: the product, summed per warp
    auto contribution = [&](uint32_t kind, uint32_t idx, const std::string& pd) {
        if (kind == OPND_REG) {
            const std::string a = "a" + std::to_string(idx);
            return a + " = __fmaf_rn(adj, " + pd + ", " + a + "); ";
        }
        if (kind == OPND_VAR) {
            return "if (gv) lfb_add_var(Gv, " + std::to_string(idx - t.n_const) + ", adj * " + pd +
                   "); ";
        }
        return std::string();
    };
    for (size_t c = t.clauses.size(); c-- > 0;) {
        const RegClause& cl = t.clauses[c];
        const uint32_t kind = slots[c] >> 28, slot = slots[c] & 0x0fffffffu;
        const uint32_t ka = cl.kinds & 3, kb = (cl.kinds >> 2) & 3;
        const bool binary = op::arity(cl.op) == 2;
        const std::string o = "a" + std::to_string(cl.out);
        std::string pdx, pdy = "0.0f";
        switch (kind) {
            case RK_CONST:
                switch (cl.op) {
                    case op::ADD: pdx = "1.0f"; pdy = "1.0f"; break;
                    case op::SUB: pdx = "1.0f"; pdy = "-1.0f"; break;
                    case op::NEG: pdx = "-1.0f"; break;
                    case op::CONST_VAR: pdx = "(block_cv ? 0.0f : 1.0f)"; break;
                    default: pdx = "1.0f"; break;
                }
                break;
            case RK_CHOICE:
                pdx = "p0";
                pdy = "(ok ? 1.0f - p0 : 0.0f)";
                break;
            case RK_ONE: pdx = "p0"; break;
            default: pdx = "p0"; pdy = "p1"; break;
        }
        s += "    { const float adj = " + o + "; " + o + " = 0.0f; ";
        if (kind != RK_CONST) {
            s += "const float p0 = ok ? Pi[(size_t)" + std::to_string(slot) + " * m] : 0.0f; ";
            if (kind == RK_TWO) {
                s += "const float p1 = ok ? Pi[(size_t)" + std::to_string(slot + 1) +
                     " * m] : 0.0f; ";
            }
        }
        s += contribution(ka, cl.a, pdx);
        if (binary) s += contribution(kb, cl.b, pdy);
        s += "}\n";
    }
    s += "    if (ok) {\n"
         "        if (gx) gx[i] = a0;\n        if (gy) gy[i] = a1;\n        if (gz) gz[i] = a2;\n"
         "    }\n"
         "    if (gv) {\n        __syncthreads();\n"
         "        for (unsigned k = threadIdx.x; k < n_vars; k += blockDim.x) {\n"
         "            if (Gv[k] != 0.0f) atomicAdd(gvars + k, Gv[k]);\n        }\n    }\n}\n";
    return s;
}

////////////////////////////////////////////////////////////////////////////////
// Segmented kernels for long tapes, and the checkpointed reverse mode.
//
// A straight-line kernel's compile time grows much faster than its length
// (register allocation over one huge function), so long tapes are cut into
// segments of kJitSegClauses clauses, each a function of its own; the tape
// registers pass between segments through a per-thread array in local
// memory.  Inside a segment every clause result gets its own name (single
// assignment), so that the reverse pass of a segment can use all of them.
//
// Checkpointed reverse mode: the forward kernel stores, per point, only the
// registers each segment reads from earlier segments (its checkpoint); the
// backward kernel runs the segments last to first, each recomputing its
// clauses from its checkpoint and sweeping their adjoints back, so the
// stored data per point is the checkpoints instead of every clause's local
// partials.  The recomputed values, partials and products are the same
// expressions as the partials / backward kernels', in the same order.

constexpr uint32_t kJitSegClauses = 192;
/// Threads per block of the checkpointed forward and backward kernels.
constexpr unsigned kCkptFwdBlock = 256;
constexpr unsigned kCkptBwdBlock = 256;

struct JitSeg {
    uint32_t c0 = 0, c1 = 0;
    std::vector<uint32_t> live_in;   // registers read before they are written here
    std::vector<uint32_t> written;   // registers written here (each once)
    uint32_t ck_base = 0;            // first checkpoint slot of live_in
};

std::vector<JitSeg> jit_segments(const RegTape& t, uint32_t* ck_total)
{
    std::vector<JitSeg> out;
    uint32_t base = 0;
    const uint32_t n = static_cast<uint32_t>(t.clauses.size());
    std::vector<uint8_t> st(t.n_regs);
    for (uint32_t c0 = 0; c0 < n; c0 += kJitSegClauses) {
        JitSeg s;
        s.c0 = c0;
        s.c1 = std::min(n, c0 + kJitSegClauses);
        s.ck_base = base;
        std::fill(st.begin(), st.end(), 0);   // 0 untouched, 1 read first, 2 written
        for (uint32_t c = s.c0; c < s.c1; ++c) {
            const RegClause& cl = t.clauses[c];
            auto read = [&](uint32_t kind, uint32_t r) {
                if (kind != OPND_REG) return;
                if (st[r] == 0) {
                    st[r] = 1;
                    s.live_in.push_back(r);
                }
            };
            read(cl.kinds & 3, cl.a);
            read(b_kind(cl), cl.b);
            if (st[cl.out] != 2) {
                if (std::find(s.written.begin(), s.written.end(), cl.out) == s.written.end()) {
                    s.written.push_back(cl.out);
                }
                st[cl.out] = 2;
            }
        }
        base += static_cast<uint32_t>(s.live_in.size());
        out.push_back(std::move(s));
    }
    if (ck_total) *ck_total = base;
    return out;
}

/// Operand of a clause inside a segment: the latest name of a register
/// (a single-assignment name, or its live-in value), a literal or a free
/// variable.
std::string seg_operand(const RegTape& t, uint32_t kind, uint32_t idx,
                        const std::vector<std::string>& name)
{
    if (kind == OPND_REG) return name[idx];
    return operand(t, kind, idx);
}

/// Forward segment function: live-ins from R (and, with ckpt, stored to
/// the checkpoint column Ci), the clauses in single assignment, the
/// registers it writes back to R.
std::string fseg_source(const RegTape& t, const JitSeg& sg, uint32_t k, bool ckpt)
{
    std::string s = "__device__ __noinline__ void fseg" + std::to_string(k) +
                    "(float* __restrict__ R, float* __restrict__ Ci, unsigned m, "
                    "const float* __restrict__ cp, int ok)\n{\n";
    std::vector<std::string> name(t.n_regs);
    for (size_t j = 0; j < sg.live_in.size(); ++j) {
        const uint32_t r = sg.live_in[j];
        name[r] = "v" + std::to_string(r);
        s += "    const float " + name[r] + " = R[" + std::to_string(r) + "];\n";
        if (ckpt) {
            s += "    if (ok) Ci[(size_t)" + std::to_string(sg.ck_base + j) + " * m] = " + name[r] +
                 ";\n";
        }
    }
    for (uint32_t c = sg.c0; c < sg.c1; ++c) {
        const RegClause& cl = t.clauses[c];
        const std::string a = seg_operand(t, cl.kinds & 3, cl.a, name);
        const std::string b = seg_operand(t, b_kind(cl), cl.b, name);
        const std::string e = expr(cl.op, a, b);
        if (e.empty()) return std::string();
        const std::string o = "s" + std::to_string(c);
        s += "    const float " + o + " = " + e + ";\n";
        name[cl.out] = o;
    }
    for (uint32_t r : sg.written) s += "    R[" + std::to_string(r) + "] = " + name[r] + ";\n";
    s += "}\n";
    return s;
}

/// Root operand after all segments (the register array or a literal).
std::string root_from_R(const RegTape& t)
{
    if (t.root_kind == OPND_REG) return "R[" + std::to_string(t.root) + "]";
    return operand(t, t.root_kind, t.root);
}

/// Value kernel of a long tape (same signature as values_source's).
std::string values_source_segmented(const RegTape& t)
{
    const auto segs = jit_segments(t, nullptr);
    std::string s = kPrelude;
    for (uint32_t k = 0; k < segs.size(); ++k) {
        const std::string f = fseg_source(t, segs[k], k, false);
        if (f.empty()) return std::string();
        s += f;
    }
    s += "extern \"C\" __global__ void __launch_bounds__(256)\n"
         "lfb_tape_values(const float* __restrict__ X, const float* __restrict__ Y,\n"
         "                const float* __restrict__ Z, float* __restrict__ out,\n"
         "                unsigned long long n, const float* __restrict__ cp)\n{\n";
    s += kHead;
    s += "        float R[" + std::to_string(t.n_regs) + "];\n"
         "        for (int r = 3; r < " + std::to_string(t.n_regs) + "; ++r) R[r] = 0.0f;\n"
         "        R[0] = X[i]; R[1] = Y[i]; R[2] = Z[i];\n";
    for (uint32_t k = 0; k < segs.size(); ++k) {
        s += "        fseg" + std::to_string(k) + "(R, nullptr, 0u, cp, 0);\n";
    }
    s += "        out[i] = " + root_from_R(t) + ";\n    }\n}\n";
    return s;
}

/// Checkpointed reverse mode, forward kernel: f and the checkpoints.
std::string ckpt_forward_source(const RegTape& t)
{
    const auto segs = jit_segments(t, nullptr);
    std::string s = kPrelude;
    for (uint32_t k = 0; k < segs.size(); ++k) {
        const std::string f = fseg_source(t, segs[k], k, true);
        if (f.empty()) return std::string();
        s += f;
    }
    s += "extern \"C\" __global__ void __launch_bounds__(" + std::to_string(kCkptFwdBlock) + ")\n"
         "lfb_tape_ckpt_fwd(const float* __restrict__ X, const float* __restrict__ Y,\n"
         "                  const float* __restrict__ Z, float* __restrict__ C,\n"
         "                  float* __restrict__ f, unsigned m, const float* __restrict__ cp)\n{\n"
         "    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;\n"
         "    const int ok = i < m;\n"
         "    const unsigned ii = ok ? i : 0u;\n";
    s += "    float R[" + std::to_string(t.n_regs) + "];\n"
         "    for (int r = 3; r < " + std::to_string(t.n_regs) + "; ++r) R[r] = 0.0f;\n"
         "    R[0] = X[ii]; R[1] = Y[ii]; R[2] = Z[ii];\n";
    for (uint32_t k = 0; k < segs.size(); ++k) {
        s += "    fseg" + std::to_string(k) + "(R, C + ii, m, cp, ok);\n";
    }
    s += "    if (ok && f) f[i] = " + root_from_R(t) + ";\n}\n";
    return s;
}

/// Backward segment function: live-ins from the checkpoint, the clauses
/// and their local partials recomputed, adjoints swept back; A holds the
/// adjoint of every register at the segment's end on entry and at its
/// start on return.
std::string bseg_source(const RegTape& t, const JitSeg& sg, uint32_t k,
                        std::vector<uint32_t>* vidx)
{
    std::string s = "__device__ __noinline__ void bseg" + std::to_string(k) +
                    "(float* __restrict__ A, const float* __restrict__ Ci, unsigned m, "
                    "const float* __restrict__ cp, float* Gv, int gv, int block_cv, int ok)\n{\n";
    std::vector<std::string> name(t.n_regs);
    for (size_t j = 0; j < sg.live_in.size(); ++j) {
        const uint32_t r = sg.live_in[j];
        name[r] = "v" + std::to_string(r);
        s += "    const float " + name[r] + " = Ci[(size_t)" + std::to_string(sg.ck_base + j) +
             " * m];\n";
    }
    // recompute: value and local partials of every clause
    struct Ref {
        uint32_t kind;      // OPND_REG / OPND_VAR / other
        std::string adj;    // adjoint variable receiving the contribution
        uint32_t var;       // variable index (OPND_VAR)
    };
    std::vector<Ref> ra(sg.c1 - sg.c0), rb(sg.c1 - sg.c0);
    std::vector<uint8_t> is_written(t.n_regs, 0), is_live(t.n_regs, 0);
    for (uint32_t r : sg.written) is_written[r] = 1;
    for (uint32_t r : sg.live_in) is_live[r] = 1;
    std::vector<std::string> adjname(t.n_regs);   // current adjoint variable of each register
    for (uint32_t r : sg.live_in) adjname[r] = "gi" + std::to_string(r);
    for (uint32_t c = sg.c0; c < sg.c1; ++c) {
        const RegClause& cl = t.clauses[c];
        std::string v, pa, pb, pre;
        if (!partial_exprs(cl.op, &v, &pa, &pb, &pre)) return std::string();
        if (cl.op == op::CONST_VAR) pa = "(block_cv ? 0.0f : 1.0f)";
        // a min / max passes the adjoint to the chosen side: b gets 1 - pa
        if (cl.op == op::MIN || cl.op == op::MAX) pb = "1.0f - pa" + std::to_string(c);
        const uint32_t ka = cl.kinds & 3, kb = b_kind(cl);
        const std::string c_ = std::to_string(c);
        s += "    float s" + c_ + ", pa" + c_ + ", pb" + c_ + ";\n";
        s += "    { const float a = " + seg_operand(t, ka, cl.a, name) + ", b = " +
             seg_operand(t, kb, cl.b, name) + "; " + pre + "s" + c_ + " = " + v + "; pa" + c_ +
             " = " + pa + "; pb" + c_ + " = " + pb + "; }\n";
        const uint32_t i = c - sg.c0;
        ra[i] = {ka, ka == OPND_REG ? adjname[cl.a] : std::string(),
                 ka == OPND_VAR ? cl.a - t.n_const : 0u};
        if (kb != 99u) {
            rb[i] = {kb, kb == OPND_REG ? adjname[cl.b] : std::string(),
                     kb == OPND_VAR ? cl.b - t.n_const : 0u};
        } else {
            rb[i] = {99u, std::string(), 0u};
        }
        name[cl.out] = "s" + c_;
        adjname[cl.out] = "g" + c_;
    }
    // adjoint variables: clause results (the last definition of a register
    // starts from the register's adjoint after the segment), live-ins (those
    // not written here pass the adjoint after the segment through)
    std::vector<uint8_t> last_def(sg.c1 - sg.c0, 0);
    {
        std::vector<uint8_t> seen(t.n_regs, 0);
        for (uint32_t c = sg.c1; c-- > sg.c0;) {
            const uint32_t o = t.clauses[c].out;
            if (!seen[o]) {
                seen[o] = 1;
                last_def[c - sg.c0] = 1;
            }
        }
    }
    for (uint32_t c = sg.c0; c < sg.c1; ++c) {
        const uint32_t o = t.clauses[c].out;
        s += "    float g" + std::to_string(c) + " = " +
             (last_def[c - sg.c0] ? "A[" + std::to_string(o) + "]" : std::string("0.0f")) + ";\n";
    }
    for (uint32_t r : sg.live_in) {
        s += "    float gi" + std::to_string(r) + " = " +
             (is_written[r] ? std::string("0.0f") : "A[" + std::to_string(r) + "]") + ";\n";
    }
    // Variable adjoints: summed per thread over the segment, then over the
    // warp 32 variables at a time (lfb_flush32) into the block's sums.
    std::vector<uint32_t> seg_vars;
    auto var_slot = [&](uint32_t v) {
        auto it = std::find(seg_vars.begin(), seg_vars.end(), v);
        if (it != seg_vars.end()) return static_cast<uint32_t>(it - seg_vars.begin());
        seg_vars.push_back(v);
        s += "    float va" + std::to_string(seg_vars.size() - 1) + " = 0.0f;\n";
        return static_cast<uint32_t>(seg_vars.size() - 1);
    };
    for (uint32_t c = sg.c0; c < sg.c1; ++c) {
        const uint32_t i = c - sg.c0;
        if (ra[i].kind == OPND_VAR) var_slot(ra[i].var);
        if (rb[i].kind == OPND_VAR) var_slot(rb[i].var);
    }
    // register adjoints: one fused multiply-add per operand (as the
    // interpreter); variable sums: product then sum
    auto contrib = [&](const Ref& rf, const std::string& g, const std::string& p) -> std::string {
        if (rf.kind == OPND_REG) {
            return "    " + rf.adj + " = __fmaf_rn(" + g + ", " + p + ", " + rf.adj + ");\n";
        }
        if (rf.kind == OPND_VAR) {
            return "    va" + std::to_string(var_slot(rf.var)) + " += " + g + " * " + p + ";\n";
        }
        return std::string();
    };
    for (uint32_t c = sg.c1; c-- > sg.c0;) {
        const std::string c_ = std::to_string(c);
        const uint32_t i = c - sg.c0;
        s += contrib(ra[i], "g" + c_, "pa" + c_);
        if (rb[i].kind != 99u) s += contrib(rb[i], "g" + c_, "pb" + c_);
    }
    for (size_t g0 = 0; g0 < seg_vars.size(); g0 += 32) {
        const size_t base = vidx->size();
        s += "    if (gv) { float v[32] = {";
        for (size_t j = 0; j < 32; ++j) {
            const size_t q = g0 + j;
            s += j ? ", " : "";
            s += q < seg_vars.size() ? "ok ? va" + std::to_string(q) + " : 0.0f" : "0.0f";
            vidx->push_back(q < seg_vars.size() ? seg_vars[q] : 0xffffu);
        }
        s += "}; lfb_flush32(v, Gv, " + std::to_string(base) + "u); }\n";
    }
    for (uint32_t r : sg.live_in) s += "    A[" + std::to_string(r) + "] = gi" + std::to_string(r) + ";\n";
    for (uint32_t r : sg.written) {
        if (!is_live[r]) s += "    A[" + std::to_string(r) + "] = 0.0f;\n";
    }
    s += "}\n";
    return s;
}

/// Checkpointed reverse mode, backward kernel (arguments as the backward
/// kernel's, plus the checkpoints and the constant pool).
std::string ckpt_backward_source(const RegTape& t)
{
    const auto segs = jit_segments(t, nullptr);
    std::string body;
    std::vector<uint32_t> vidx;
    for (uint32_t k = 0; k < segs.size(); ++k) {
        const std::string b = bseg_source(t, segs[k], k, &vidx);
        if (b.empty()) return std::string();
        body += b;
    }
    std::string s = kPrelude;
    s += "__device__ __forceinline__ void lfb_add_var(float* Gv, unsigned k, float g)\n{\n"
         "    for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);\n"
         "    if ((threadIdx.x & 31) == 0 && g != 0.0f) atomicAdd(Gv + k, g);\n}\n";
    // variable of each flushed slot (0xffff: none)
    s += "__device__ const unsigned short lfb_vidx[" + std::to_string(std::max<size_t>(vidx.size(), 1)) +
         "] = {";
    for (size_t j = 0; j < vidx.size(); ++j) s += (j ? "," : "") + std::to_string(vidx[j]);
    if (vidx.empty()) s += "0";
    s += "};\n";
    // 32 per-thread sums -> lane l holds slot l's sum over the warp
    // (recursive halving: 31 shuffles for 32 variables)
    s += "__device__ __forceinline__ void lfb_flush32(float (&v)[32], float* Gv, unsigned base)\n{\n"
         "    const unsigned lane = threadIdx.x & 31;\n"
         "#pragma unroll\n"
         "    for (int w = 16; w >= 1; w >>= 1) {\n"
         "#pragma unroll\n"
         "        for (int i = 0; i < w; ++i) {\n"
         "            const bool up = lane & w;\n"
         "            const float send = up ? v[i] : v[i + w];\n"
         "            const float keep = up ? v[i + w] : v[i];\n"
         "            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, w);\n"
         "        }\n    }\n"
         "    const unsigned k = lfb_vidx[base + lane];\n"
         "    if (k != 0xffffu && v[0] != 0.0f) atomicAdd(Gv + k, v[0]);\n}\n";
    s += body;
    // at most 64 registers a thread: four blocks of 256 threads on an SM.
    // (One 1024-thread block with a barrier before each segment, so that
    // an SM's warps share a segment's instruction fetches, was measured
    // slower: the barriers cost more than the fetch stalls they saved.)
    s += "extern \"C\" __global__ void __launch_bounds__(" + std::to_string(kCkptBwdBlock) +
         ", 4)\n"
         "lfb_tape_ckpt_bwd(const float* __restrict__ C, const float* __restrict__ seed,\n"
         "                  float* __restrict__ gx, float* __restrict__ gy,\n"
         "                  float* __restrict__ gz, float* __restrict__ gvars, unsigned m,\n"
         "                  unsigned n_vars, int block_cv, const float* __restrict__ cp,\n"
         "                  float sscale)\n{\n"
         "    extern __shared__ float Gv[];\n"
         "    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;\n"
         "    const int ok = i < m;\n"
         "    const int gv = gvars != nullptr;\n"
         "    if (gv) {\n"
         "        for (unsigned k = threadIdx.x; k < n_vars; k += blockDim.x) Gv[k] = 0.0f;\n"
         "        __syncthreads();\n    }\n"
         "    const float* const Ci = C + (ok ? i : 0);\n";
    s += "    float A[" + std::to_string(t.n_regs) + "];\n"
         "    for (int r = 0; r < " + std::to_string(t.n_regs) + "; ++r) A[r] = 0.0f;\n"
         "    const float s0 = ok ? (seed ? seed[i] : 1.0f) * sscale : 0.0f;\n";
    if (t.root_kind == OPND_REG) {
        s += "    A[" + std::to_string(t.root) + "] = s0;\n";
    } else if (t.root_kind == OPND_VAR) {
        s += "    if (gv) lfb_add_var(Gv, " + std::to_string(t.root - t.n_const) + ", s0);\n";
    }
    for (uint32_t k = static_cast<uint32_t>(segs.size()); k-- > 0;) {
        s += "    bseg" + std::to_string(k) + "(A, Ci, m, cp, Gv, gv, block_cv, ok);\n";
    }
    s += "    if (ok) {\n"
         "        if (gx) gx[i] = A[0];\n        if (gy) gy[i] = A[1];\n        if (gz) gz[i] = A[2];\n"
         "    }\n"
         "    if (gv) {\n        __syncthreads();\n"
         "        for (unsigned k = threadIdx.x; k < n_vars; k += blockDim.x) {\n"
         "            if (Gv[k] != 0.0f) atomicAdd(gvars + k, Gv[k]);\n        }\n    }\n}\n";
    return s;
}

/// Interval operand: registers are kept as Iv values; constants and free
/// variables become degenerate intervals as the interpreter's fetch does.
std::string iv_operand(const RegTape& t, uint32_t kind, uint32_t idx)
{
    if (kind == OPND_REG) return "r" + std::to_string(idx);
    const std::string v = operand(t, kind, idx);
    return "iv_make(" + v + ", " + v + ")";
}

/// Opcodes the interval kernel compiles: every unary and binary one.
bool iv_supported(uint8_t o)
{
    return op::arity(o) >= 1;
}

/// Compiles `src` and loads its kernel `name` into slot k; false when
/// anything is unavailable or fails.
bool build(GpuTape& g, int k, const std::string& src, const char* name)
{
    const Api& A = api();
    if (!A.ok || src.empty()) return false;
    std::vector<char> cubin;
    if (!jit_compile(src, &cubin, nullptr)) return false;
    CUmodule mod = nullptr;
    CUfunction fn = nullptr;
    if (A.load(&mod, cubin.data()) != CUDA_SUCCESS) return false;
    if (A.function(&fn, mod, name) != CUDA_SUCCESS) {
        A.unload(mod);
        return false;
    }
    g.jit[k].module = mod;
    g.jit[k].function = fn;
    return true;
}

/// The kernel of slot k (0 values, 1 derivatives, 2 reverse-mode
/// partials, 3 reverse-mode backward pass), compiled on first use.
void* kernel(GpuTape& g, int k, const std::vector<uint32_t>* slots = nullptr)
{
    std::lock_guard<std::mutex> lock(g.mu);
    GpuTape::JitKernel& j = g.jit[k];
    if (j.state == 0) {
        const size_t n = g.reg.clauses.size();
        bool ok = api().ok && n <= (k == 4 ? kJitMaxIntervalClauses
                                    : (k == 0 || k >= 5) ? kJitMaxSegmentedClauses
                                                         : kJitMaxClauses);
        if (ok) {
            switch (k) {
                case 0:
                    ok = build(g, 0, n <= kJitMaxClauses ? values_source(g.reg)
                                                         : values_source_segmented(g.reg),
                               "lfb_tape_values");
                    break;
                case 5: ok = build(g, 5, ckpt_forward_source(g.reg), "lfb_tape_ckpt_fwd"); break;
                case 6: ok = build(g, 6, ckpt_backward_source(g.reg), "lfb_tape_ckpt_bwd"); break;
                case 1: ok = build(g, 1, derivs_source(g.reg), "lfb_tape_derivs"); break;
                case 2: ok = build(g, 2, partials_source(g.reg, *slots), "lfb_tape_partials"); break;
                case 3: ok = build(g, 3, backward_source(g.reg, *slots), "lfb_tape_backward"); break;
                default: ok = build(g, 4, jit_interval_source(g.reg), "lfb_tape_intervals"); break;
            }
        }
        j.state = ok ? 1 : -1;
    }
    return j.state == 1 ? j.function : nullptr;
}

bool launch_1d(void* fn, uint32_t m, void** args, unsigned smem, cudaStream_t s,
               unsigned block = 256)
{
    const unsigned blocks = (m + block - 1) / block;
    if (api().launch(static_cast<CUfunction>(fn), blocks, 1, 1, block, 1, 1, smem,
                     reinterpret_cast<CUstream>(s), args, nullptr) != CUDA_SUCCESS) {
        return false;
    }
    note_launches(1);
    return true;
}

bool launch(void* fn, uint64_t n, void** args, cudaStream_t s)
{
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256,
                                               static_cast<uint64_t>(device_sm_count()) * 16);
    if (api().launch(static_cast<CUfunction>(fn), static_cast<unsigned>(blocks), 1, 1, 256, 1,
                     1, 0, reinterpret_cast<CUstream>(s), args, nullptr) != CUDA_SUCCESS) {
        return false;
    }
    note_launches(1);
    return true;
}

}  // namespace

bool jit_values(GpuTape& g, uint64_t n, const float* x, const float* y, const float* z,
                float* out, cudaStream_t s)
{
    void* fn = kernel(g, 0);
    if (!fn) return false;
    if (n == 0) return true;
    unsigned long long nn = n;
    const float* cp = g.d_cpool;
    void* args[] = {&x, &y, &z, &out, &nn, &cp};
    return launch(fn, n, args, s);
}

bool jit_derivs(GpuTape& g, uint64_t n, const float* x, const float* y, const float* z,
                float* v, float* dx, float* dy, float* dz, cudaStream_t s)
{
    void* fn = kernel(g, 1);
    if (!fn) return false;
    if (n == 0) return true;
    unsigned long long nn = n;
    const float* cp = g.d_cpool;
    void* args[] = {&x, &y, &z, &v, &dx, &dy, &dz, &nn, &cp};
    return launch(fn, n, args, s);
}

bool jit_derivs_if_loaded(GpuTape& g, uint64_t n, const float* x, const float* y,
                          const float* z, float* v, float* dx, float* dy, float* dz,
                          cudaStream_t s)
{
    {
        std::lock_guard<std::mutex> lock(g.mu);
        if (g.jit[1].state != 1) return false;
    }
    return jit_derivs(g, n, x, y, z, v, dx, dy, dz, s);
}

bool jit_partials(GpuTape& g, const uint32_t* slots, uint32_t m, const float* x,
                  const float* y, const float* z, float* P, float* f, cudaStream_t s)
{
    std::vector<uint32_t> table;
    {
        std::lock_guard<std::mutex> lock(g.mu);
        if (g.jit[2].state == 0) table.assign(slots, slots + g.reg.clauses.size());
    }
    void* fn = kernel(g, 2, &table);
    if (!fn) return false;
    if (m == 0) return true;
    const float* cp = g.d_cpool;
    void* args[] = {&x, &y, &z, &P, &f, &m, &cp};
    return launch_1d(fn, m, args, 0, s);
}

bool jit_backward(GpuTape& g, const uint32_t* slots, uint32_t m, const float* P,
                  const float* seed, float* gx, float* gy, float* gz, float* gvars,
                  int block_cv, cudaStream_t s)
{
    uint32_t n_vars = g.reg.n_vars;
    const unsigned smem = gvars ? n_vars * 4 : 0;
    if (smem > 48 * 1024) return false;
    std::vector<uint32_t> table;
    {
        std::lock_guard<std::mutex> lock(g.mu);
        if (g.jit[3].state == 0) table.assign(slots, slots + g.reg.clauses.size());
    }
    void* fn = kernel(g, 3, &table);
    if (!fn) return false;
    if (m == 0) return true;
    void* args[] = {&P, &seed, &gx, &gy, &gz, &gvars, &m, &n_vars, &block_cv};
    return launch_1d(fn, m, args, smem, s);
}

uint32_t jit_ckpt_prepare(GpuTape& g)
{
    if (!kernel(g, 5) || !kernel(g, 6)) return 0;
    std::lock_guard<std::mutex> lock(g.mu);
    if (!g.ckpt_floats) {
        uint32_t total = 0;
        jit_segments(g.reg, &total);
        g.ckpt_floats = std::max<uint32_t>(total, 1);
    }
    return g.ckpt_floats;
}

bool jit_ckpt_forward(GpuTape& g, uint32_t m, const float* x, const float* y, const float* z,
                      float* C, float* f, cudaStream_t s)
{
    void* fn = kernel(g, 5);
    if (!fn) return false;
    if (m == 0) return true;
    const float* cp = g.d_cpool;
    void* args[] = {&x, &y, &z, &C, &f, &m, &cp};
    return launch_1d(fn, m, args, 0, s, kCkptFwdBlock);
}

bool jit_ckpt_backward(GpuTape& g, uint32_t m, const float* C, const float* seed, float* gx,
                       float* gy, float* gz, float* gvars, int block_cv, cudaStream_t s,
                       float seed_scale)
{
    uint32_t n_vars = g.reg.n_vars;
    const unsigned smem = gvars ? n_vars * 4 : 0;
    if (smem > 48 * 1024) return false;
    void* fn = kernel(g, 6);
    if (!fn) return false;
    if (m == 0) return true;
    const float* cp = g.d_cpool;
    void* args[] = {&C, &seed, &gx, &gy, &gz, &gvars, &m, &n_vars, &block_cv, &cp, &seed_scale};
    return launch_1d(fn, m, args, smem, s, kCkptBwdBlock);
}

bool jit_compile(const std::string& src, std::vector<char>* cubin, std::string* log)
{
    const Api& A = api();
    if (!A.create) return false;
    nvrtcProgram prog = nullptr;
    if (A.create(&prog, src.c_str(), "lfb_tape.cu", kJitHeaderCount, kJitHeaderSources,
                 kJitHeaderNames) != NVRTC_SUCCESS) {
        return false;
    }
    const char* opts[] = {"--gpu-architecture=sm_100a", "-fmad=false", "--std=c++17"};
    bool ok = A.compile(prog, 3, opts) == NVRTC_SUCCESS;
    if (log && A.log_size && A.log) {
        size_t n = 0;
        if (A.log_size(prog, &n) == NVRTC_SUCCESS && n > 1) {
            log->resize(n);
            A.log(prog, &(*log)[0]);
        }
    }
    size_t size = 0;
    ok = ok && A.cubin_size(prog, &size) == NVRTC_SUCCESS && size > 0;
    if (ok) {
        cubin->resize(size);
        ok = A.cubin(prog, cubin->data()) == NVRTC_SUCCESS;
    }
    A.destroy(&prog);
    return ok;
}

std::string jit_interval_source(const RegTape& t)
{
    std::string s;
    s.reserve(96 * t.clauses.size() + 1024);
    s += kPrelude;
    s += "extern \"C\" __global__ void __launch_bounds__(256)\n"
         "lfb_tape_intervals(const float* __restrict__ xlo, const float* __restrict__ xhi,\n"
         "                   const float* __restrict__ ylo, const float* __restrict__ yhi,\n"
         "                   const float* __restrict__ zlo, const float* __restrict__ zhi,\n"
         "                   float* __restrict__ olo, float* __restrict__ ohi,\n"
         "                   unsigned char* __restrict__ onan, unsigned long long n,\n"
         "                   const float* __restrict__ cp)\n{\n";
    s += kHead;
    s += "        Iv r0 = iv_make(xlo[i], xhi[i]), r1 = iv_make(ylo[i], yhi[i]),\n"
         "           r2 = iv_make(zlo[i], zhi[i]);\n";
    for (uint32_t r = 3; r < t.n_regs; ++r) {
        s += "        Iv r" + std::to_string(r) + " = {0.0f, 0.0f, false};\n";
    }
    for (const RegClause& c : t.clauses) {
        if (!iv_supported(c.op)) return std::string();
        const std::string a = iv_operand(t, c.kinds & 3, c.a);
        const bool binary = op::arity(c.op) == 2;
        const std::string b = binary ? iv_operand(t, (c.kinds >> 2) & 3, c.b) : "ia";
        s += "        { const Iv ia = " + a + "; const Iv ib = " + b + "; r" +
             std::to_string(c.out) + " = iv_apply(" + std::to_string(c.op) + ", ia, ib); }\n";
    }
    const std::string root = iv_operand(t, t.root_kind, t.root);
    s += "        { const Iv r = " + root + "; olo[i] = r.lo; ohi[i] = r.hi; onan[i] = r.nan; }\n"
         "    }\n}\n";
    return s;
}

bool jit_intervals(GpuTape& g, uint64_t n, const float* xlo, const float* xhi,
                   const float* ylo, const float* yhi, const float* zlo, const float* zhi,
                   float* olo, float* ohi, uint8_t* onan, cudaStream_t s)
{
    void* fn = kernel(g, 4);
    if (!fn) return false;
    if (n == 0) return true;
    unsigned long long nn = n;
    const float* cp = g.d_cpool;
    void* args[] = {&xlo, &xhi, &ylo, &yhi, &zlo, &zhi, &olo, &ohi, &onan, &nn, &cp};
    return launch(fn, n, args, s);
}

void jit_release(GpuTape& g)
{
    for (auto& j : g.jit) {
        if (j.module && api().ok) api().unload(static_cast<CUmodule>(j.module));
        j.module = nullptr;
        j.function = nullptr;
    }
}

}  // namespace lfb
