// Device-side per-opcode semantics for the three forward evaluators.
//
//  * value:    ArrayEvaluator::operator()      (libfive/src/eval/eval_array.cpp:221-369)
//  * deriv:    DerivArrayEvaluator::operator() (libfive/src/eval/eval_deriv_array.cpp:119-256)
//  * interval: IntervalEvaluator::operator()   (libfive/src/eval/eval_interval.cpp:189-294)
//              with the Interval class rules (libfive/include/libfive/eval/interval.hpp:31-442)
//              and Boost.Interval's rounded arithmetic restated with the
//              directed-rounding intrinsics __f{add,sub,mul,div,sqrt}_{rd,ru}.
//
// All arithmetic is written with explicit _rn / _rd / _ru intrinsics so that
// no FMA contraction can change a result; value-mode results are therefore
// bit-identical to a scalar IEEE evaluation of the same clause for every
// exactly-rounded opcode (+ - * / sqrt neg abs square min max recip ...).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "opcode.hpp"
#include "scalar_ops.h"
#include "dev_tape.h"
#include "tape.hpp"
#include "dev_interval.cuh"
#include "dev_point.cuh"

namespace lfb {



}  // namespace lfb
