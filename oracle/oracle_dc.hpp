// CPU oracle dual-contouring mesher (TEST INFRASTRUCTURE ONLY).
#pragma once
#include <cstdint>
#include <vector>

#include "oracle.hpp"

namespace ora {

/// Mesh::render with DUAL_CONTOURING on the CPU; returns the octree depth.
/// With threads > 1 the octree build and the dual walk run as task pools
/// (cells five levels below the root) on that many threads.  sample_stride
/// > 1 builds only every sample_stride-th task and stops (timing samples);
/// phase_s (or null) receives the seconds of the serial top levels, the
/// parallel tasks, and the collapse + dual walk.
int render_mesh(const Tape& tape, const float lo[3], const float hi[3],
                double min_feature, double max_err, int threads,
                std::vector<float>& verts, std::vector<uint32_t>& tris, int sample_stride,
                double* phase_s);

}  // namespace ora
