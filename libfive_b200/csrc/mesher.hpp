// Dual-contouring mesher driver (GPU) and STL writer.
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "libfive.h"
#include "libfive_b200.h"
#include "runtime.hpp"

namespace lfb {

/// What render_dc_mesh returns for the triangles: the indexed mesh
/// (libfive_mesh), the vertices with 4 coordinate indices per triangle
/// (a, b, c, -1: libfive_mesh_coords, libfive.cpp:354-395), or binary STL
/// records (mesh.cpp:139-194) packed on the device and streamed to a file.
enum class MeshFormat { Indexed, Coords, Stl };

/// Mesh arrays in host memory from host_alloc (freed with host_free); the
/// C API hands them to the caller's libfive_mesh without a copy.
struct MeshOut {
    libfive_vec3* verts = nullptr;   // verts[0] is the dummy vertex
    libfive_tri* tris = nullptr;     // indices start at 1 (Indexed only)
    uint32_t vert_count = 0;
    uint32_t tri_count = 0;
    MeshFormat format = MeshFormat::Indexed;
    int32_t* coords = nullptr;       // Coords: 4 * tri_count, host_alloc'd
    const char* stl_path = nullptr;  // Stl: the file written (header, count,
                                     // records) once the triangles are known;
                                     // verts then holds the dummy vertex only
    MeshOut() = default;
    MeshOut(const MeshOut&) = delete;
    MeshOut& operator=(const MeshOut&) = delete;
    ~MeshOut();
    /// Moves the arrays into a new libfive_mesh (freed by libfive_mesh_delete).
    libfive_mesh* release();
};

/// Mesh arrays in page-locked host memory, recycled between meshes (a freed
/// block serves the next allocation of up to twice its size; at most 1 GiB
/// of idle blocks is kept), so that a mesh downloads in one direct copy.
/// Falls back to pageable memory when page-locked memory is unavailable.
void* host_alloc(size_t bytes);
void host_free(void* p);

/// Mesh::render with DUAL_CONTOURING (libfive/src/render/brep/mesh.cpp:48-72)
/// for one tree; returns 0 or a negative LFB_E* code.
/// cancel (or null) is polled between stages (lfb_mesh_settings::cancel).
int render_dc_mesh(GpuTape& g, const libfive_region3& R, double min_feature,
                   double max_err, MeshOut& out, lfb_mesh_stats* stats,
                   const volatile int32_t* cancel = nullptr);

/// One mesh of a batch (render_dc_meshes).
struct MeshJob {
    GpuTape* g = nullptr;
    libfive_region3 R{};
    double min_feature = 0.0;
    double max_err = 0.0;
    const volatile int32_t* cancel = nullptr;
    bool want_stats = false;
    MeshOut out;
    lfb_mesh_stats stats{};
    int rc = 1;            // 1 until rendered, then 0 or a negative LFB_E* code
    std::string err;       // the failure's message
};

/// Renders n meshes with up to `workers` of them in flight at once, each on
/// its own CUDA stream and scratch context, longest (tape length x 4^depth)
/// first; large meshes go one at a time through one context while the
/// others render the small ones.  A mesh that runs out of device memory is
/// rendered again alone.  Returns 0 when every job succeeded, else the first
/// failing job's code (with its message set as this thread's error).
int render_dc_meshes(MeshJob* jobs, size_t n, unsigned workers);

/// Binary STL in the reference's layout (mesh.cpp:139-194): 80-byte header,
/// uint32 triangle count, then per triangle a zero normal, three vertices
/// and a zero attribute word.
bool save_stl(const char* path, const std::vector<libfive_mesh*>& meshes);

/// Opens `path` and writes the STL header and triangle count, with the
/// reference's messages for a name without ".stl" and a failed open; null
/// when the file cannot be opened.
std::FILE* stl_begin(const char* path, uint32_t count);

}  // namespace lfb
