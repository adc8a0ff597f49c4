// CPU oracle for height-map rendering: TEST INFRASTRUCTURE ONLY.
#pragma once
#include <cstdint>

#include "oracle.hpp"

namespace ora {

/// Image size of a voxel region (Voxels, voxels.cpp:23-44):
/// dims = {cols, rows, depth samples}.
void voxel_dims(const float lower[3], const float upper[3], const float res[3],
                uint32_t dims[3]);

/// Voxel sample positions along one axis (dims[axis] floats).
void voxel_pts(const float lower[3], const float upper[3], const float res[3], int axis,
               float* out);

/// Heightmap::render (heightmap.cpp:247-296) with `workers` initial regions:
/// depth and norm are rows x cols, row-major; norm may be null.
void render_heightmap(const Tape& base, const float lower[3], const float upper[3],
                      const float res[3], int workers, float* depth, uint32_t* norm);

}  // namespace ora
