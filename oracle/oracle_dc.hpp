// CPU oracle dual-contouring mesher (TEST INFRASTRUCTURE ONLY).
#pragma once
#include <cstdint>
#include <vector>

#include "oracle.hpp"

namespace ora {

/// Mesh::render with DUAL_CONTOURING on the CPU; returns the octree depth.
int render_mesh(const Tape& tape, const float lo[3], const float hi[3],
                double min_feature, double max_err, int threads,
                std::vector<float>& verts, std::vector<uint32_t>& tris);

}  // namespace ora
