#include "eval_api.hpp"
#include "mesher.hpp"
namespace lfb {
int render_dc_mesh(GpuTape&, const libfive_region3&, double, double, MeshOut&, lfb_mesh_stats*)
{ return set_error(LFB_E_UNSUPPORTED, "mesher not built yet"); }
int eval_jacobian(GpuTape&, uint64_t, const float*, const float*, const float*, float*, cudaStream_t, bool)
{ return set_error(LFB_E_UNSUPPORTED, "not built yet"); }
int eval_grad(GpuTape&, uint64_t, const float*, const float*, const float*, const float*, float*, float*, float*, float*, float*, cudaStream_t, bool)
{ return set_error(LFB_E_UNSUPPORTED, "not built yet"); }
}
