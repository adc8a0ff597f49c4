#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "contours.hpp"
#include "mesher.hpp"

namespace lfb {

std::FILE* stl_begin(const char* path, uint32_t count)
{
    if (!path) return nullptr;
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
        return nullptr;
    }
    char header[80];
    std::memset(header, ' ', sizeof(header));
    const char* text = "This is a binary STL exported from libfive.";
    std::memcpy(header, text, std::strlen(text));
    std::fwrite(header, 1, sizeof(header), f);
    std::fwrite(&count, sizeof(count), 1, f);
    return f;
}

bool save_stl(const char* path, const std::vector<libfive_mesh*>& meshes)
{
    uint32_t count = 0;
    for (auto m : meshes) count += m->tri_count;
    FILE* f = stl_begin(path, count);
    if (!f) return false;
    // Records are packed into one buffer by a few threads and written with
    // one call per mesh (a write per 50-byte record is the slow part of a
    // large file).
    std::vector<unsigned char> body;
    for (auto m : meshes) {
        const size_t n = m->tri_count;
        body.assign(n * 50, 0);
        auto pack = [&](size_t lo, size_t hi) {
            for (size_t i = lo; i < hi; ++i) {
                unsigned char* rec = body.data() + 50 * i;
                const uint32_t idx[3] = {m->tris[i].a, m->tris[i].b, m->tris[i].c};
                for (int k = 0; k < 3; ++k) {
                    const libfive_vec3& v = m->verts[idx[k]];
                    const float xyz[3] = {v.x, v.y, v.z};
                    std::memcpy(rec + 12 + 12 * k, xyz, 12);
                }
            }
        };
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const size_t n_threads = std::min<size_t>(std::min(hw, 8u), std::max<size_t>(1, n >> 16));
        const size_t part = (n + n_threads - 1) / n_threads;
        std::vector<std::thread> pool;
        for (size_t t = 1; t < n_threads; ++t) {
            pool.emplace_back(pack, std::min(n, t * part), std::min(n, (t + 1) * part));
        }
        pack(0, std::min(n, part));
        for (auto& th : pool) th.join();
        if (n) std::fwrite(body.data(), 1, body.size(), f);
    }
    const bool ok = std::ferror(f) == 0;
    std::fclose(f);
    return ok;
}

/// Contours::saveSVG (contours.cpp:51-116): one path per contour, y
/// flipped into the bounding box, "Z" closing a contour whose last point
/// repeats its first; numbers in the stream's default format (%g).
bool save_svg(const char* path, const ContoursOut& cs, const double lo[2], const double hi[2])
{
    const std::string name(path);
    const auto ends_with = [&](const char* suf) {
        const size_t n = std::strlen(suf);
        if (name.size() < n) return false;
        for (size_t k = 0; k < n; ++k) {
            const char a = name[name.size() - n + k];
            if (std::tolower(static_cast<unsigned char>(a)) != suf[k]) return false;
        }
        return true;
    };
    if (!ends_with(".svg")) {
        std::fprintf(stderr, "Contours::saveSVG: filename \"%s\" does not end in .svg\n", path);
    }
    FILE* f = std::fopen(path, "w");
    if (!f) {
        std::printf("Contours::saveSVG: could not open %s\n", path);
        return false;
    }
    std::fprintf(f,
                 "<?xml version=\"1.0\" encoding=\"UTF-8\" standalone=\"no\"?>\n"
                 "<svg xmlns=\"http://www.w3.org/2000/svg\" version=\"1.1\"\n"
                 " width=\"%g\" height=\"%g\" id=\"libfive\">\n",
                 hi[0] - lo[0], hi[1] - lo[1]);
    size_t k = 0;
    for (uint32_t n : cs.counts) {
        const float* p = cs.pts.data() + 2 * k;
        k += n;
        std::fprintf(f, "<path d=\"");
        const bool closed = n > 0 && p[0] == p[2 * (n - 1)] && p[1] == p[2 * (n - 1) + 1];
        const uint32_t end = closed ? n - 1 : n;
        for (uint32_t j = 0; j < end; ++j) {
            std::fprintf(f, "%s %g %g ", j == 0 ? "M" : "L", static_cast<double>(p[2 * j]) - lo[0],
                         hi[1] - static_cast<double>(p[2 * j + 1]));
        }
        if (closed) std::fprintf(f, "Z");
        std::fprintf(f, "\"\nfill=\"none\" stroke=\"black\" stroke-width=\"0.01\"/>");
    }
    std::fprintf(f, "\n</svg>");
    const bool ok = std::ferror(f) == 0;
    return std::fclose(f) == 0 && ok;
}

}  // namespace lfb
