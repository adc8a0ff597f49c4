// CPU oracle for height-map rendering: TEST INFRASTRUCTURE ONLY.
//
// Restates libfive's Voxels (libfive/src/render/discrete/voxels.cpp:16-44,
// include/libfive/render/discrete/voxels.hpp:50-110) and Heightmap::render
// (libfive/src/render/discrete/heightmap.cpp:22-296) on top of the oracle
// evaluators: the image is split on X/Y into up to eight regions, each
// region is reduced recursively (skip when every pixel is already above it,
// evaluate pixel by pixel at <= 256 voxels, else interval-evaluate, fill
// when filled, split on the largest axis and recurse into the upper half
// first when ambiguous), and normals are taken from derivatives at the
// surface voxels.  The regions are processed one after another here; they
// cover disjoint pixels, so the order does not change the result.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <list>
#include <memory>
#include <vector>

#include "oracle_eval.hpp"
#include "oracle_heightmap.hpp"

using namespace ora;

namespace {

struct Voxels {
    float lower[3], upper[3];
    std::vector<float> pts[3];
};

// voxels.cpp:23-44, in float arithmetic as Eigen does it.
Voxels make_voxels(const float lo[3], const float hi[3], const float res[3])
{
    Voxels v;
    for (int a = 0; a < 3; ++a) {
        const float span = hi[a] - lo[a];
        const float sz = std::max(std::ceil(res[a] * span), 1.0f);
        const int size = static_cast<int>(sz);
        const float extra = res[a] > 0 ? static_cast<float>(size) / res[a] - span : 0.0f;
        v.lower[a] = lo[a] - extra / 2;
        v.upper[a] = hi[a] + extra / 2;
        for (int i = 0; i < size; ++i) {
            const float frac = static_cast<float>((i + 0.5) / size);
            v.pts[a].push_back(v.lower[a] * (1 - frac) + v.upper[a] * frac);
        }
    }
    return v;
}

struct View {
    float lower[3], upper[3];
    int size[3];
    int corner[3];
    const float* pts[3];

    size_t voxels() const
    {
        return static_cast<size_t>(size[0]) * size[1] * size[2];
    }

    // Voxels::View::split<A> (voxels.hpp:63-99): the largest allowed axis
    // (first one on ties), the lower part rounded up.
    void split(unsigned axes, View* lo, View* hi) const
    {
        int axis = 0, best = -1;
        for (int a = 0; a < 3; ++a) {
            const int s = (axes & (1u << a)) ? size[a] : 0;
            if (s > best) {
                best = s;
                axis = a;
            }
        }
        const int size_upper = size[axis] / 2;
        const int size_lower = size[axis] - size_upper;
        const float frac = size_lower / static_cast<float>(size[axis]);
        const float middle = (upper[axis] * frac) + (lower[axis] * (1 - frac));
        *lo = *this;
        *hi = *this;
        lo->upper[axis] = middle;
        lo->size[axis] = size_lower;
        hi->lower[axis] = middle;
        hi->size[axis] = size_upper;
        hi->pts[axis] += size_lower;
        hi->corner[axis] += size_lower;
    }
};

constexpr int kArray = 256;   // ArrayEvaluator::N

struct Heightmap {
    int rows, cols;
    std::vector<float> depth;      // row-major [y][x]
    std::vector<uint32_t> norm;

    float& d(int y, int x) { return depth[static_cast<size_t>(y) * cols + x]; }
    uint32_t& n(int y, int x) { return norm[static_cast<size_t>(y) * cols + x]; }
};

// The packing of heightmap.cpp:40-52: Eigen's normalized() (squared norm
// reduced as x^2 + (y^2 + z^2) by its unrolled reduction, no division when
// it is zero), mapped to 0..255 and truncated, alpha 0xff.
uint32_t pack_normal(float dx, float dy, float dz)
{
    const float sq = dx * dx + (dy * dy + dz * dz);
    float n[3] = {dx, dy, dz};
    if (sq > 0) {
        const float s = std::sqrt(sq);
        for (float& c : n) c = c / s;
    }
    uint32_t out = 0xffu << 24;
    for (int a = 0; a < 3; ++a) {
        const float f = 255.0f * (n[a] / 2 + 0.5f);
        // cvttss2si: NaN and out-of-range values give INT_MIN
        const int32_t i = (f >= -2147483648.0f && f < 2147483648.0f)
                              ? static_cast<int32_t>(f)
                              : std::numeric_limits<int32_t>::min();
        out |= static_cast<uint32_t>(i) << (8 * a);
    }
    return out;
}

struct Normals {
    Evaluator* e;
    const Tape* tape;
    const View& r;
    Heightmap& hm;
    int xs[kArray], ys[kArray];
    int count = 0;

    void run()
    {
        std::vector<float> d4(4 * count);
        e->derivs(count, *tape, d4.data());
        for (int i = 0; i < count; ++i) {
            hm.n(ys[i], xs[i]) = pack_normal(d4[4 * i], d4[4 * i + 1], d4[4 * i + 2]);
        }
        count = 0;
    }
    void flush()
    {
        if (count > 0) run();
    }
    void push(int i, int j, float z)
    {
        xs[count] = r.corner[0] + i;
        ys[count] = r.corner[1] + j;
        e->set(r.pts[0][i], r.pts[1][j], z, count++);
        if (count == kArray) run();
    }
};

// heightmap.cpp:96-151
void pixels(Evaluator* e, const Tape& tape, const View& r, Heightmap& hm)
{
    const float ztop = r.pts[2][r.size[2] - 1];
    int index = 0;
    for (int i = 0; i < r.size[0]; ++i) {
        for (int j = 0; j < r.size[1]; ++j) {
            if (hm.d(r.corner[1] + j, r.corner[0] + i) < ztop) {
                for (int k = 0; k < r.size[2]; ++k) {
                    e->set(r.pts[0][i], r.pts[1][j], r.pts[2][r.size[2] - k - 1], index++);
                }
            }
        }
    }
    const float* out = e->values(index, tape);
    std::vector<float> vals(out, out + index);
    index = 0;
    Normals nr{e, &tape, r, hm};
    for (int i = 0; i < r.size[0]; ++i) {
        for (int j = 0; j < r.size[1]; ++j) {
            if (!(hm.d(r.corner[1] + j, r.corner[0] + i) < ztop)) continue;
            for (int k = 0; k < r.size[2]; ++k) {
                if (vals[index++] < 0) {
                    const float z = r.pts[2][r.size[2] - k - 1];
                    float& d = hm.d(r.corner[1] + j, r.corner[0] + i);
                    if (d < z) {
                        d = z;
                        nr.push(i, j, z);
                    }
                    index += r.size[2] - k - 1;
                    break;
                }
            }
        }
    }
    nr.flush();
}

// heightmap.cpp:159-188
void fill(Evaluator* e, const Tape& tape, const View& r, Heightmap& hm)
{
    const float z = r.pts[2][r.size[2] - 1];
    Normals nr{e, &tape, r, hm};
    for (int i = 0; i < r.size[0]; ++i) {
        for (int j = 0; j < r.size[1]; ++j) {
            float& d = hm.d(r.corner[1] + j, r.corner[0] + i);
            if (d < z) {
                d = z;
                nr.push(i, j, z);
            }
        }
    }
    nr.flush();
}

// heightmap.cpp:194-245
void recurse(Evaluator* e, const std::shared_ptr<Tape>& tape, const View& r, Heightmap& hm)
{
    const float ztop = r.pts[2][r.size[2] - 1];
    bool all_above = true;
    for (int j = 0; j < r.size[1] && all_above; ++j) {
        for (int i = 0; i < r.size[0]; ++i) {
            if (!(hm.d(r.corner[1] + j, r.corner[0] + i) >= ztop)) {
                all_above = false;
                break;
            }
        }
    }
    if (all_above) return;
    if (r.voxels() <= static_cast<size_t>(kArray)) {
        pixels(e, *tape, r, hm);
        return;
    }
    const Iv out = e->interval(r.lower[0], r.lower[1], r.lower[2],
                               r.upper[0], r.upper[1], r.upper[2], *tape);
    const auto pushed = e->push_interval(tape);
    if (out.i.hi < 0) {
        fill(e, *tape, r, hm);
    } else if (!(out.i.lo > 0)) {
        View lo, hi;
        r.split(7, &lo, &hi);
        recurse(e, pushed, hi, hm);
        recurse(e, pushed, lo, hm);
    }
}

}  // namespace

namespace ora {

/// Image size of a voxel region: dims = {cols, rows, depth samples}.
void voxel_dims(const float lower[3], const float upper[3], const float res[3],
                    uint32_t dims[3])
{
    const Voxels v = make_voxels(lower, upper, res);
    for (int a = 0; a < 3; ++a) dims[a] = static_cast<uint32_t>(v.pts[a].size());
}

/// Voxel sample positions along one axis (pts[axis], dims[axis] floats).
void voxel_pts(const float lower[3], const float upper[3], const float res[3],
                   int axis, float* out)
{
    const Voxels v = make_voxels(lower, upper, res);
    std::memcpy(out, v.pts[axis].data(), v.pts[axis].size() * sizeof(float));
}

/// Heightmap::render with `workers` initial regions (the reference's default
/// is 8): depth and norm are rows x cols, row-major.
void render_heightmap(const Tape& base, const float lower[3], const float upper[3],
                      const float res[3], int workers, float* depth, uint32_t* norm)
{
    const Voxels v = make_voxels(lower, upper, res);
    Heightmap hm;
    hm.cols = static_cast<int>(v.pts[0].size());
    hm.rows = static_cast<int>(v.pts[1].size());
    hm.depth.assign(static_cast<size_t>(hm.rows) * hm.cols,
                    -std::numeric_limits<float>::infinity());
    hm.norm.assign(static_cast<size_t>(hm.rows) * hm.cols, 0);

    View root;
    for (int a = 0; a < 3; ++a) {
        root.lower[a] = v.lower[a];
        root.upper[a] = v.upper[a];
        root.size[a] = static_cast<int>(v.pts[a].size());
        root.corner[a] = 0;
        root.pts[a] = v.pts[a].data();
    }
    // heightmap.cpp:264-276: split on X/Y until there is a region per worker
    std::list<View> rs = {root};
    while (static_cast<int>(rs.size()) < workers &&
           std::min(rs.front().size[0], rs.front().size[1]) > 1) {
        View f = rs.front();
        rs.pop_front();
        View lo, hi;
        f.split(3, &lo, &hi);
        rs.push_back(lo);
        rs.push_back(hi);
    }
    for (const View& r : rs) {
        Evaluator e(base);
        recurse(&e, e.base, r, hm);
    }
    const float ztop = v.pts[2].back();
    for (size_t i = 0; i < hm.depth.size(); ++i) {
        if (hm.depth[i] == ztop) hm.norm[i] = 0xffff7f7fu;
    }
    std::memcpy(depth, hm.depth.data(), hm.depth.size() * sizeof(float));
    if (norm) std::memcpy(norm, hm.norm.data(), hm.norm.size() * sizeof(uint32_t));
}

}  // namespace ora
