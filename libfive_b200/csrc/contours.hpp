// 2D contours of a slice (Contours::render) on the GPU.
#pragma once
#include <cstdint>
#include <utility>
#include <vector>

#include "runtime.hpp"

namespace lfb {

/// Contours as polylines: counts[i] points of contour i, x and y
/// interleaved in pts; a closed contour repeats its first point at the end.
struct ContoursOut {
    std::vector<float> pts;
    std::vector<uint32_t> counts;
};

/// Contours::render (libfive/src/render/brep/contours.cpp:25-49) of the
/// tape over [lo, hi] at z = perp, with BRepSettings' min_feature and
/// max_err; 0 or a negative LFB_E* code.
int render_contours(GpuTape& g, const double lo[2], const double hi[2], double z,
                    double min_feature, double max_err, ContoursOut& out);

/// Contours::collect's welding of directed segments into polylines
/// (contours.cpp:118-184), in segment order.
void weld_segments(const std::vector<std::pair<uint32_t, uint32_t>>& segs,
                   std::vector<std::vector<uint32_t>>& out);

/// Contours::saveSVG (contours.cpp:51-116).
bool save_svg(const char* path, const ContoursOut& cs, const double lo[2], const double hi[2]);

}  // namespace lfb
