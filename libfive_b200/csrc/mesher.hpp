// Dual-contouring mesher driver (GPU) and STL writer.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "libfive.h"
#include "libfive_b200.h"
#include "runtime.hpp"

namespace lfb {

struct MeshOut {
    std::vector<float> verts;      // xyz triples; verts[0..2] is the dummy
    std::vector<uint32_t> tris;    // index triples (indices start at 1)
};

/// Mesh::render with DUAL_CONTOURING (libfive/src/render/brep/mesh.cpp:48-72)
/// for one tree; returns 0 or a negative LFB_E* code.
int render_dc_mesh(GpuTape& g, const libfive_region3& R, double min_feature,
                   double max_err, MeshOut& out, lfb_mesh_stats* stats);

/// Binary STL in the reference's layout (mesh.cpp:139-194): 80-byte header,
/// uint32 triangle count, then per triangle a zero normal, three vertices
/// and a zero attribute word.
bool save_stl(const char* path, const std::vector<libfive_mesh*>& meshes);

}  // namespace lfb
