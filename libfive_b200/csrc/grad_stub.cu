#include "eval_api.hpp"
#include "libfive_b200.h"
namespace lfb {
int eval_jacobian(GpuTape&, uint64_t, const float*, const float*, const float*, float*, cudaStream_t, bool)
{ return set_error(LFB_E_UNSUPPORTED, "not built yet"); }
int eval_grad(GpuTape&, uint64_t, const float*, const float*, const float*, const float*, float*, float*, float*, float*, float*, cudaStream_t, bool)
{ return set_error(LFB_E_UNSUPPORTED, "not built yet"); }
}
