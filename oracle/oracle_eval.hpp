// CPU oracle evaluators (TEST INFRASTRUCTURE ONLY; see oracle.hpp).
#pragma once
#include <functional>
#include <memory>
#include <vector>

#include "oracle.hpp"

namespace ora {

// Opcode values of libfive/include/libfive/tree/opcode.hpp (unpacked).
enum {
    OP_CONST_VAR = 6, OP_SQUARE = 7, OP_SQRT = 8, OP_NEG = 9, OP_SIN = 10,
    OP_COS = 11, OP_TAN = 12, OP_ASIN = 13, OP_ACOS = 14, OP_ATAN = 15,
    OP_EXP = 16, OP_ADD = 17, OP_MUL = 18, OP_MIN = 19, OP_MAX = 20,
    OP_SUB = 21, OP_DIV = 22, OP_ATAN2 = 23, OP_POW = 24, OP_NTH_ROOT = 25,
    OP_MOD = 26, OP_NANFILL = 27, OP_ABS = 28, OP_RECIP = 29, OP_LOG = 30,
    OP_COMPARE = 31,
};

constexpr int NB = 256;   // LIBFIVE_EVAL_ARRAY_SIZE

int op_arity(int op);

// Library-call results of the point evaluators: 0 = host C library,
// 1 = host library and record every (opcode << 32 | input bits) key,
// 2 = replay from the table of libm_set_table (misses use the host library
// and are recorded).  Switching mode clears what was recorded.
void libm_set_mode(int mode);
void libm_set_table(const uint64_t* keys, const uint32_t* vals, uint64_t n);
uint64_t libm_take(uint64_t* out, uint64_t max);
uint64_t libm_misses();
float value_op(int op, float a, float b);
void deriv_op(int op, float av, float bv, float ov, const float* ad,
              const float* bd, float* od, bool clear_vars);

struct BI;
struct Iv;
Iv iv_make(float lo, float hi);

struct Vec3 {
    float x[3];
};

struct Feature {
    Vec3 deriv{{0, 0, 0}};
    std::vector<Vec3> eps;
    bool check(const Vec3& e, bool* dup = nullptr) const;
    bool push(const Vec3& e);
    bool push_all(const Feature& other);
};

using KeepFn = std::function<Keep(int, uint32_t, uint32_t, uint32_t)>;

const Tape* get_base(const Tape* tape, float x, float y, float z);

}  // namespace ora

// Interval definitions are needed by users of Evaluator::interval.
namespace ora {
struct BI {
    float lo, hi;
    static BI empty();
    static BI make(float l, float u);
    bool bad() const { return !(lo <= hi); }
};
struct Iv {
    BI i;
    bool nan;
};
}  // namespace ora

namespace ora {

class Evaluator {
public:
    explicit Evaluator(const Tape& base);

    std::shared_ptr<Tape> base;
    bool clear_vars = false;

    void set(float x, float y, float z, int index);
    const float* values(int count, const Tape& tape);
    /// out4[4*i + 0..2] = d/dx, d/dy, d/dz; out4[4*i + 3] = value
    void derivs(int count, const Tape& tape, float* out4);
    void ambiguous(int count, const Tape& tape, bool* out);
    Iv interval(float xl, float yl, float zl, float xu, float yu, float zu,
                const Tape& tape);
    std::shared_ptr<Tape> push_interval(const std::shared_ptr<Tape>& tape);
    std::shared_ptr<Tape> value_and_push(float x, float y, float z,
                                         const std::shared_ptr<Tape>& tape,
                                         float* value);
    bool is_inside(float x, float y, float z, const std::shared_ptr<Tape>& tape);
    std::vector<Vec3> features(float x, float y, float z,
                               const std::shared_ptr<Tape>& tape);
    void jacobian(float x, float y, float z, float* out);

private:
    std::shared_ptr<Tape> push(const std::shared_ptr<Tape>& tape,
                               const KeepFn& fn, int type);
    std::vector<Feature> feature_lists(const Tape& tape, uint32_t* root);

    std::vector<float> v;
    std::vector<float> d;
    std::vector<Iv> iv;
    std::vector<uint8_t> disabled;
    std::vector<uint32_t> remap;
};

}  // namespace ora
