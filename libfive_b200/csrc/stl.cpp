#include <cstdio>
#include <cstring>
#include <string>

#include "mesher.hpp"

namespace lfb {

bool save_stl(const char* path, const std::vector<libfive_mesh*>& meshes)
{
    if (!path) return false;
    const std::string name(path);
    if (name.size() < 4 ||
        (name.compare(name.size() - 4, 4, ".stl") != 0 &&
         name.compare(name.size() - 4, 4, ".STL") != 0)) {
        std::fprintf(stderr, "Mesh::saveSTL: filename \"%s\" does not end in .stl\n",
                     path);
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        std::fprintf(stderr, "Mesh::saveSTL: could not open %s\n", path);
        return false;
    }
    char header[80];
    std::memset(header, ' ', sizeof(header));
    const char* text = "This is a binary STL exported from libfive.";
    std::memcpy(header, text, std::strlen(text));
    std::fwrite(header, 1, sizeof(header), f);
    uint32_t count = 0;
    for (auto m : meshes) count += m->tri_count;
    std::fwrite(&count, sizeof(count), 1, f);
    for (auto m : meshes) {
        for (uint32_t i = 0; i < m->tri_count; ++i) {
            unsigned char rec[50];
            std::memset(rec, 0, sizeof(rec));
            const uint32_t idx[3] = {m->tris[i].a, m->tris[i].b, m->tris[i].c};
            for (int k = 0; k < 3; ++k) {
                const libfive_vec3& v = m->verts[idx[k]];
                const float xyz[3] = {v.x, v.y, v.z};
                std::memcpy(rec + 12 + 12 * k, xyz, 12);
            }
            std::fwrite(rec, 1, sizeof(rec), f);
        }
    }
    const bool ok = std::ferror(f) == 0;
    std::fclose(f);
    return ok;
}

}  // namespace lfb
