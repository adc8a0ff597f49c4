// Height-map rendering on the GPU (Heightmap::render,
// libfive/src/render/discrete/heightmap.cpp:247-296) and the voxel grid it
// samples (Voxels, libfive/src/render/discrete/voxels.cpp:16-44).
#pragma once
#include <cstdint>
#include <vector>

#include "runtime.hpp"

namespace lfb {

/// Voxels: a region whose bounds are widened about their centre to a whole
/// number of voxels per axis, sampled at the voxel centres.  Computed in
/// float arithmetic exactly as the reference's Eigen expressions.
struct VoxelGrid {
    float lower[3], upper[3];
    std::vector<float> pts[3];
};
VoxelGrid make_voxel_grid(const float lower[3], const float upper[3], const float res[3]);

/// Depth (rows x cols, row-major: the highest z sample at which the shape
/// is filled, -inf where no sample is) and, when `norm` is not null, packed
/// normals (0xAABBGGRR of the normalised gradient mapped to 0..255; pixels
/// at the top of the region 0xffff7f7f, empty pixels 0).  depth and norm are
/// host arrays.  Returns 0 or a negative LFB_E* code.
int render_heightmap(GpuTape& g, const VoxelGrid& V, float* depth, uint32_t* norm);

}  // namespace lfb
