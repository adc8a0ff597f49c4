// Height maps on the GPU.
//
// The reference reduces each image region depth-first (heightmap.cpp:194-
// 245): skip it when every pixel is already above it, fill it when its
// interval is negative, evaluate its voxels when it holds at most 256 of
// them, else split it and recurse, upper half first.  Its result is, per
// pixel, the highest z sample whose voxel is inside (value < 0): a filled
// region's voxels are all inside, an empty region's all outside, so the
// order of the recursion does not change the image.  This driver computes
// the same image breadth-first:
//
//   1. the image is cut into 16 x 16 pixel tiles and the z range into slabs
//      of 16 samples; one interval evaluation per (tile, slab) box over the
//      box's sample points classifies it filled (upper < 0, as isFilled,
//      interval.hpp:64), empty (lower > 0) or ambiguous;
//   2. per tile, the highest filled slab sets a depth floor (its top
//      sample) and the ambiguous slabs above it are the only ones that can
//      raise it;
//   3. those slabs are processed top slab first, one round per slab depth,
//      skipping tiles whose pixels are all above the slab: each selected
//      box is refined into 4 x 4 x 4 sub-boxes, classified by interval
//      again (a filled sub-box raises its pixels to its top sample), and
//      only the ambiguous sub-boxes are evaluated voxel by voxel; depths
//      rise by an atomic max on an order-preserving integer key;
//   4. normals are the normalised gradient at (x, y, depth) of each pixel
//      (DerivArrayEvaluator, as NormalRenderer does, heightmap.cpp:35-53).
//
// The image matches the reference's wherever the shape has no NaN values:
// the reference's fill test ignores the interval's maybe-NaN flag, so a
// region it fills may contain voxels whose value is NaN, which voxel
// evaluation here counts as outside.
#include "heightmap.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "eval_api.hpp"
#include "libfive_b200.h"

namespace lfb {

VoxelGrid make_voxel_grid(const float lo[3], const float hi[3], const float res[3])
{
    // voxels.cpp:23-44: size = max(ceil(res * span), 1); the bounds grow by
    // half the excess on each side; samples at (i + 0.5) / size, the
    // fraction divided in double and rounded to float.
    VoxelGrid v;
    for (int a = 0; a < 3; ++a) {
        const float span = hi[a] - lo[a];
        const float sz = std::max(std::ceil(res[a] * span), 1.0f);
        const int size = static_cast<int>(sz);
        const float extra = res[a] > 0 ? static_cast<float>(size) / res[a] - span : 0.0f;
        v.lower[a] = lo[a] - extra / 2;
        v.upper[a] = hi[a] + extra / 2;
        v.pts[a].reserve(size);
        for (int i = 0; i < size; ++i) {
            const float frac = static_cast<float>((i + 0.5) / size);
            v.pts[a].push_back(v.lower[a] * (1 - frac) + v.upper[a] * frac);
        }
    }
    return v;
}

namespace {

constexpr uint32_t kTile = 16;   // pixels per tile side
constexpr uint32_t kSlab = 16;   // z samples per slab

/// Float -> unsigned key with the same order (for atomicMax on depths).
__device__ __forceinline__ uint32_t depth_key(float f)
{
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_depth(uint32_t k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

struct Grid {
    const float* px;
    const float* py;
    const float* pz;
    uint32_t W, H, D;       // cols, rows, z samples
    uint32_t ntx, nty, ns;  // tiles across, tiles down, slabs
    uint32_t tz;            // z samples per slab (kSlab, or D when smaller)
};

// z-sample index range of slab s (s = 0 is the top slab): [k0, k1)
__device__ __forceinline__ void slab_range(const Grid& g, uint32_t s, uint32_t* k0, uint32_t* k1)
{
    const uint32_t top = g.D - s * g.tz;   // exclusive
    *k1 = top;
    *k0 = top > g.tz ? top - g.tz : 0;
}

/// Bounding box of each (tile, slab)'s sample points; box b = tile * ns + s.
__global__ void k_hm_boxes(Grid g, float* xlo, float* xhi, float* ylo, float* yhi,
                           float* zlo, float* zhi)
{
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= g.ntx * g.nty * g.ns) return;
    const uint32_t s = b % g.ns, t = b / g.ns;
    const uint32_t tx = t % g.ntx, ty = t / g.ntx;
    const uint32_t x0 = tx * kTile, x1 = min(g.W, x0 + kTile);
    const uint32_t y0 = ty * kTile, y1 = min(g.H, y0 + kTile);
    uint32_t k0, k1;
    slab_range(g, s, &k0, &k1);
    auto span = [](const float* p, uint32_t i0, uint32_t i1, float* lo, float* hi) {
        const float a = p[i0], c = p[i1 - 1];
        *lo = a < c ? a : c;
        *hi = a < c ? c : a;
    };
    span(g.px, x0, x1, xlo + b, xhi + b);
    span(g.py, y0, y1, ylo + b, yhi + b);
    span(g.pz, k0, k1, zlo + b, zhi + b);
}

/// Per tile, top slab first: the first filled slab sets the tile's depth
/// floor; the ambiguous slabs above it are marked for voxel evaluation.
__global__ void k_hm_classify(Grid g, const float* lo, const float* hi, uint8_t* need,
                              uint32_t* floor_key)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.ntx * g.nty) return;
    uint32_t key = depth_key(-INFINITY);
    for (uint32_t s = 0; s < g.ns; ++s) {
        const uint32_t b = t * g.ns + s;
        need[b] = 0;
        if (hi[b] < 0) {
            uint32_t k0, k1;
            slab_range(g, s, &k0, &k1);
            key = depth_key(g.pz[k1 - 1]);
            for (uint32_t r = s + 1; r < g.ns; ++r) need[t * g.ns + r] = 0;
            break;
        }
        if (!(lo[b] > 0)) need[b] = 1;
    }
    floor_key[t] = key;
}

/// Boxes of slab s to evaluate this round: marked, and with a pixel of the
/// tile still below the slab's top sample.  One warp per tile.
__global__ void k_hm_select(Grid g, uint32_t s, const uint8_t* need, const uint32_t* pix_key,
                            uint32_t* list, uint32_t* count)
{
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const uint32_t lane = threadIdx.x & 31;
    if (warp >= g.ntx * g.nty) return;
    const uint32_t t = warp;
    if (!need[t * g.ns + s]) return;
    uint32_t k0, k1;
    slab_range(g, s, &k0, &k1);
    const uint32_t top = depth_key(g.pz[k1 - 1]);
    const uint32_t tx = t % g.ntx, ty = t / g.ntx;
    bool below = false;
    for (uint32_t p = lane; p < kTile * kTile; p += 32) {
        const uint32_t x = tx * kTile + p % kTile, y = ty * kTile + p / kTile;
        if (x < g.W && y < g.H && pix_key[static_cast<size_t>(y) * g.W + x] < top) below = true;
    }
    if (__any_sync(0xffffffffu, below) && lane == 0) {
        list[atomicAdd(count, 1u)] = t * g.ns + s;
    }
}

/// Each selected box is refined into sub-boxes of 4 x 4 pixels x 4 z samples
/// (fewer at the image edge and in short slabs) before any voxel is
/// evaluated: sub-box j of a box covers pixel columns 4 (j % 4), rows
/// 4 ((j / 4) % 4) of its tile and the j / 16-th group of 4 z samples from
/// the top of its slab.
constexpr uint32_t kSub = 4;

struct SubRange {
    uint32_t x0, x1, y0, y1, z0, z1;
    bool valid;
};

__device__ __forceinline__ uint32_t sub_depth(const Grid& g)
{
    return min(kSub, g.tz);
}

__device__ SubRange sub_range(const Grid& g, uint32_t b, uint32_t j)
{
    const uint32_t s = b % g.ns, t = b / g.ns;
    const uint32_t tx = t % g.ntx, ty = t / g.ntx;
    uint32_t k0, k1;
    slab_range(g, s, &k0, &k1);
    const uint32_t sd = sub_depth(g);
    SubRange r;
    r.x0 = tx * kTile + (j % 4) * kSub;
    r.x1 = min(g.W, r.x0 + kSub);
    r.y0 = ty * kTile + ((j / 4) % 4) * kSub;
    r.y1 = min(g.H, r.y0 + kSub);
    const uint32_t dz = (j / 16) * sd;
    r.valid = r.x0 < r.x1 && r.y0 < r.y1 && dz < k1 - k0;
    r.z1 = r.valid ? k1 - dz : k1;
    r.z0 = (r.z1 - k0 > sd) ? r.z1 - sd : k0;
    if (!r.valid) {
        r.x0 = r.y0 = 0;
        r.x1 = r.y1 = 1;
    }
    return r;
}

/// Bounds of the sub-boxes of boxes list[0..n), nsub per box (invalid
/// sub-boxes get the first voxel's bounds; classification skips them).
__global__ void k_hm_subboxes(Grid g, const uint32_t* list, uint32_t n, uint32_t nsub,
                              float* xlo, float* xhi, float* ylo, float* yhi, float* zlo,
                              float* zhi)
{
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n * nsub) return;
    const SubRange r = sub_range(g, list[q / nsub], q % nsub);
    auto span = [](const float* p, uint32_t i0, uint32_t i1, float* lo, float* hi) {
        const float a = p[i0], c = p[i1 - 1];
        *lo = a < c ? a : c;
        *hi = a < c ? c : a;
    };
    span(g.px, r.x0, r.x1, xlo + q, xhi + q);
    span(g.py, r.y0, r.y1, ylo + q, yhi + q);
    span(g.pz, r.z0, r.z1, zlo + q, zhi + q);
}

/// Filled sub-boxes raise their pixels to the sub-box's top sample; the
/// ambiguous ones with a pixel still below that sample are listed for
/// voxel evaluation (entry = q, the sub-box's index in this chunk).
__global__ void k_hm_subclassify(Grid g, const uint32_t* list, uint32_t n, uint32_t nsub,
                                 const float* lo, const float* hi, uint32_t* pix_key,
                                 uint32_t* amb, uint32_t* n_amb)
{
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n * nsub) return;
    const SubRange r = sub_range(g, list[q / nsub], q % nsub);
    if (!r.valid) return;
    const uint32_t top = depth_key(g.pz[r.z1 - 1]);
    if (hi[q] < 0) {
        for (uint32_t y = r.y0; y < r.y1; ++y) {
            for (uint32_t x = r.x0; x < r.x1; ++x) {
                atomicMax(pix_key + static_cast<size_t>(y) * g.W + x, top);
            }
        }
        return;
    }
    if (lo[q] > 0) return;
    bool below = false;
    for (uint32_t y = r.y0; y < r.y1; ++y) {
        for (uint32_t x = r.x0; x < r.x1; ++x) {
            below |= pix_key[static_cast<size_t>(y) * g.W + x] < top;
        }
    }
    if (below) amb[atomicAdd(n_amb, 1u)] = q;
}

/// Voxel v of listed sub-box e: column v % 4, row (v / 4) % 4, z sample
/// v / 16 from the sub-box's bottom; false past its edge.
__device__ __forceinline__ bool sub_voxel(const Grid& g, const uint32_t* list, uint32_t nsub,
                                          uint32_t e, uint32_t v, uint32_t* xi, uint32_t* yi,
                                          uint32_t* zi)
{
    const SubRange r = sub_range(g, list[e / nsub], e % nsub);
    const uint32_t x = r.x0 + v % kSub, y = r.y0 + (v / kSub) % kSub;
    const uint32_t z = r.z0 + v / (kSub * kSub);
    *xi = min(x, r.x1 - 1);
    *yi = min(y, r.y1 - 1);
    *zi = min(z, r.z1 - 1);
    return x < r.x1 && y < r.y1 && z < r.z1;
}

/// Sample points of the listed sub-boxes amb[0..n), vps points each.
__global__ void k_hm_points(Grid g, const uint32_t* list, uint32_t nsub, const uint32_t* amb,
                            uint32_t n, uint32_t vps, float* x, float* y, float* z)
{
    const uint64_t q = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<uint64_t>(n) * vps) return;
    uint32_t xi, yi, zi;
    sub_voxel(g, list, nsub, amb[q / vps], q % vps, &xi, &yi, &zi);
    x[q] = g.px[xi];
    y[q] = g.py[yi];
    z[q] = g.pz[zi];
}

/// Raises each pixel's depth to every inside voxel's z.
__global__ void k_hm_reduce(Grid g, const uint32_t* list, uint32_t nsub, const uint32_t* amb,
                            uint32_t n, uint32_t vps, const float* f, uint32_t* pix_key)
{
    const uint64_t q = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<uint64_t>(n) * vps) return;
    if (!(f[q] < 0)) return;
    uint32_t xi, yi, zi;
    if (!sub_voxel(g, list, nsub, amb[q / vps], q % vps, &xi, &yi, &zi)) return;
    atomicMax(pix_key + static_cast<size_t>(yi) * g.W + xi, depth_key(g.pz[zi]));
}

/// Final depth: the voxel result or the tile's filled-slab floor, whichever
/// is higher.  Normals start at 0, or 0xffff7f7f for pixels at the top
/// sample (heightmap.cpp:289-292).
__global__ void k_hm_finalize(Grid g, const uint32_t* pix_key, const uint32_t* floor_key,
                              float* depth, uint32_t* norm)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= g.W * g.H) return;
    const uint32_t x = p % g.W, y = p / g.W;
    const uint32_t t = (y / kTile) * g.ntx + x / kTile;
    const float d = key_depth(max(pix_key[p], floor_key[t]));
    depth[p] = d;
    if (norm) norm[p] = (d == g.pz[g.D - 1]) ? 0xffff7f7fu : 0u;
}

/// Pixels that need a normal (a finite depth below the top sample), with
/// the point at which their gradient is taken.
__global__ void k_hm_normal_points(Grid g, const float* depth, uint32_t* list, uint32_t* count,
                                   float* x, float* y, float* z)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= g.W * g.H) return;
    const float d = depth[p];
    if (d == -INFINITY || d == g.pz[g.D - 1]) return;
    const uint32_t i = atomicAdd(count, 1u);
    list[i] = p;
    x[i] = g.px[p % g.W];
    y[i] = g.py[p / g.W];
    z[i] = d;
}

/// heightmap.cpp:40-52: Eigen's normalized() (the squared norm reduced as
/// x^2 + (y^2 + z^2) by its unrolled sum; no division when it is zero),
/// each component mapped to 255 * (n / 2 + 0.5) and truncated the way x86
/// converts (NaN and out-of-range values give INT_MIN), alpha 0xff.
__device__ uint32_t pack_normal(float dx, float dy, float dz)
{
    const float sq = __fadd_rn(__fmul_rn(dx, dx), __fadd_rn(__fmul_rn(dy, dy), __fmul_rn(dz, dz)));
    float n[3] = {dx, dy, dz};
    if (sq > 0) {
        const float s = __fsqrt_rn(sq);
        for (float& c : n) c = __fdiv_rn(c, s);
    }
    uint32_t out = 0xff000000u;
    for (int a = 0; a < 3; ++a) {
        const float f = __fmul_rn(255.0f, __fadd_rn(__fdiv_rn(n[a], 2.0f), 0.5f));
        const int32_t i = (f >= -2147483648.0f && f < 2147483648.0f) ? __float2int_rz(f)
                                                                      : INT32_MIN;
        out |= static_cast<uint32_t>(i) << (8 * a);
    }
    return out;
}

__global__ void k_hm_pack(const uint32_t* list, uint32_t n, const float* dx, const float* dy,
                          const float* dz, uint32_t* norm)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    norm[list[i]] = pack_normal(dx[i], dy[i], dz[i]);
}

__global__ void k_hm_fill(uint32_t* p, uint64_t n, uint32_t v)
{
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

/// Device buffers of the height-map driver, grow-only, reused across calls.
struct HmBuffers {
    std::mutex mu;
    DevBuf b[26];
    template <class T>
    T* get(int k, size_t count)
    {
        return b[k].reserve(std::max<size_t>(count, 1) * sizeof(T)) ? b[k].as<T>() : nullptr;
    }
};
HmBuffers& hm_buffers()
{
    static HmBuffers* h = new HmBuffers;
    return *h;
}

uint32_t blocks_for(uint64_t n, uint32_t threads)
{
    return static_cast<uint32_t>((n + threads - 1) / threads);
}

}  // namespace

int render_heightmap(GpuTape& g, const VoxelGrid& V, float* depth, uint32_t* norm)
{
    if (!require_device()) return LFB_E_CUDA;
    const uint64_t W = V.pts[0].size(), H = V.pts[1].size(), D = V.pts[2].size();
    if (W == 0 || H == 0 || D == 0) return 0;
    if (W * H >= (1ull << 31) || D >= (1ull << 30)) {
        return set_error(LFB_E_CAPACITY, "height map too large");
    }
    HmBuffers& B = hm_buffers();
    std::lock_guard<std::mutex> lock(B.mu);
    cudaStream_t s = 0;

    Grid gr{};
    gr.W = static_cast<uint32_t>(W);
    gr.H = static_cast<uint32_t>(H);
    gr.D = static_cast<uint32_t>(D);
    gr.ntx = (gr.W + kTile - 1) / kTile;
    gr.nty = (gr.H + kTile - 1) / kTile;
    gr.tz = std::min<uint32_t>(kSlab, gr.D);
    gr.ns = (gr.D + gr.tz - 1) / gr.tz;
    const uint64_t n_tiles = static_cast<uint64_t>(gr.ntx) * gr.nty;
    const uint64_t nb = n_tiles * gr.ns;
    const uint64_t npix = W * H;
    // Sub-boxes per box and voxels per sub-box; boxes are refined 1024 at a
    // time, ambiguous sub-boxes evaluated up to 2^22 voxels at a time.
    const uint32_t sub_d = std::min(4u, gr.tz);
    const uint32_t nsub = 16 * ((gr.tz + sub_d - 1) / sub_d);
    const uint32_t vps = 16 * sub_d;
    const uint32_t chunk_boxes = 1024;
    const uint64_t n_sub = static_cast<uint64_t>(chunk_boxes) * nsub;
    const uint32_t chunk_amb = (1u << 22) / vps;
    const uint64_t chunk = static_cast<uint64_t>(chunk_amb) * vps;

    float* px = B.get<float>(0, W);
    float* py = B.get<float>(1, H);
    float* pz = B.get<float>(2, D);
    float* box = B.get<float>(3, 6 * nb);
    float* ilo = B.get<float>(4, nb);
    float* ihi = B.get<float>(5, nb);
    uint8_t* inan = B.get<uint8_t>(6, nb);
    uint8_t* need = B.get<uint8_t>(7, nb);
    uint32_t* floor_key = B.get<uint32_t>(8, n_tiles);
    uint32_t* pix_key = B.get<uint32_t>(9, npix);
    uint32_t* list = B.get<uint32_t>(10, std::max<uint64_t>(n_tiles, npix));
    uint32_t* count = B.get<uint32_t>(11, 2);
    float* cx = B.get<float>(12, std::max<uint64_t>(chunk, npix));
    float* cy = B.get<float>(13, std::max<uint64_t>(chunk, npix));
    float* cz = B.get<float>(14, std::max<uint64_t>(chunk, npix));
    float* cf = B.get<float>(15, std::max<uint64_t>(chunk, npix));
    float* sbox = B.get<float>(21, 6 * n_sub);
    float* slo = B.get<float>(22, n_sub);
    float* shi = B.get<float>(23, n_sub);
    uint8_t* snan = B.get<uint8_t>(24, n_sub);
    uint32_t* amb = B.get<uint32_t>(25, n_sub);
    float* d_depth = B.get<float>(16, npix);
    uint32_t* d_norm = norm ? B.get<uint32_t>(17, npix) : nullptr;
    float* gdx = norm ? B.get<float>(18, npix) : nullptr;
    float* gdy = norm ? B.get<float>(19, npix) : nullptr;
    float* gdz = norm ? B.get<float>(20, npix) : nullptr;
    if (!px || !py || !pz || !box || !ilo || !ihi || !inan || !need || !floor_key ||
        !pix_key || !list || !count || !cx || !cy || !cz || !cf || !d_depth || !sbox ||
        !slo || !shi || !snan || !amb ||
        (norm && (!d_norm || !gdx || !gdy || !gdz))) {
        return LFB_E_CUDA;
    }
    gr.px = px;
    gr.py = py;
    gr.pz = pz;
    if (!cuda_ok(cudaMemcpyAsync(px, V.pts[0].data(), W * 4, cudaMemcpyHostToDevice, s), "copy") ||
        !cuda_ok(cudaMemcpyAsync(py, V.pts[1].data(), H * 4, cudaMemcpyHostToDevice, s), "copy") ||
        !cuda_ok(cudaMemcpyAsync(pz, V.pts[2].data(), D * 4, cudaMemcpyHostToDevice, s), "copy")) {
        return LFB_E_CUDA;
    }
    uint64_t launches = 0;

    // 1-2. Classify every (tile, slab) box.
    float* xlo = box;
    float* xhi = box + nb;
    float* ylo = box + 2 * nb;
    float* yhi = box + 3 * nb;
    float* zlo = box + 4 * nb;
    float* zhi = box + 5 * nb;
    k_hm_boxes<<<blocks_for(nb, 256), 256, 0, s>>>(gr, xlo, xhi, ylo, yhi, zlo, zhi);
    int rc = eval_intervals_device(g, nb, xlo, xhi, ylo, yhi, zlo, zhi, ilo, ihi, inan, s);
    if (rc) return rc;
    k_hm_classify<<<blocks_for(n_tiles, 128), 128, 0, s>>>(gr, ilo, ihi, need, floor_key);
    k_hm_fill<<<blocks_for(npix, 256), 256, 0, s>>>(pix_key, npix, 0x007fffffu);   // -inf
    launches += 3;

    // 3. Voxels of the ambiguous slabs, top slab first.
    for (uint32_t sl = 0; sl < gr.ns; ++sl) {
        cudaMemsetAsync(count, 0, sizeof(uint32_t), s);
        k_hm_select<<<blocks_for(n_tiles * 32, 256), 256, 0, s>>>(gr, sl, need, pix_key, list,
                                                                    count);
        ++launches;
        uint32_t n = 0;
        cudaMemcpyAsync(&n, count, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if (!cuda_ok(cudaStreamSynchronize(s), "height map slab selection")) return LFB_E_CUDA;
        for (uint32_t c0 = 0; c0 < n; c0 += chunk_boxes) {
            const uint32_t m = std::min(chunk_boxes, n - c0);
            const uint32_t q = m * nsub;
            const uint32_t* lc = list + c0;
            k_hm_subboxes<<<blocks_for(q, 256), 256, 0, s>>>(gr, lc, m, nsub, sbox, sbox + n_sub,
                                                             sbox + 2 * n_sub, sbox + 3 * n_sub,
                                                             sbox + 4 * n_sub, sbox + 5 * n_sub);
            rc = eval_intervals_device(g, q, sbox, sbox + n_sub, sbox + 2 * n_sub,
                                       sbox + 3 * n_sub, sbox + 4 * n_sub, sbox + 5 * n_sub,
                                       slo, shi, snan, s);
            if (rc) return rc;
            cudaMemsetAsync(count + 1, 0, sizeof(uint32_t), s);
            k_hm_subclassify<<<blocks_for(q, 256), 256, 0, s>>>(gr, lc, m, nsub, slo, shi,
                                                                pix_key, amb, count + 1);
            launches += 2;
            uint32_t na = 0;
            cudaMemcpyAsync(&na, count + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
            if (!cuda_ok(cudaStreamSynchronize(s), "height map refinement")) return LFB_E_CUDA;
            for (uint32_t a0 = 0; a0 < na; a0 += chunk_amb) {
                const uint32_t ma = std::min(chunk_amb, na - a0);
                const uint64_t nv = static_cast<uint64_t>(ma) * vps;
                k_hm_points<<<blocks_for(nv, 256), 256, 0, s>>>(gr, lc, nsub, amb + a0, ma, vps,
                                                                cx, cy, cz);
                rc = eval_values_device(g, nv, cx, cy, cz, cf, s);
                if (rc) return rc;
                k_hm_reduce<<<blocks_for(nv, 256), 256, 0, s>>>(gr, lc, nsub, amb + a0, ma, vps,
                                                                cf, pix_key);
                launches += 2;
            }
        }
    }
    k_hm_finalize<<<blocks_for(npix, 256), 256, 0, s>>>(gr, pix_key, floor_key, d_depth, d_norm);
    ++launches;

    // 4. Normals.
    if (norm) {
        cudaMemsetAsync(count, 0, sizeof(uint32_t), s);
        k_hm_normal_points<<<blocks_for(npix, 256), 256, 0, s>>>(gr, d_depth, list, count, cx,
                                                                  cy, cz);
        ++launches;
        uint32_t n = 0;
        cudaMemcpyAsync(&n, count, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if (!cuda_ok(cudaStreamSynchronize(s), "height map normals")) return LFB_E_CUDA;
        if (n) {
            rc = eval_derivs_device(g, n, cx, cy, cz, cf, gdx, gdy, gdz, s);
            if (rc) return rc;
            k_hm_pack<<<blocks_for(n, 256), 256, 0, s>>>(list, n, gdx, gdy, gdz, d_norm);
            ++launches;
        }
        if (!cuda_ok(cudaMemcpyAsync(norm, d_norm, npix * 4, cudaMemcpyDeviceToHost, s),
                     "height map download")) {
            return LFB_E_CUDA;
        }
    }
    if (!cuda_ok(cudaMemcpyAsync(depth, d_depth, npix * 4, cudaMemcpyDeviceToHost, s),
                 "height map download") ||
        !cuda_ok(cudaStreamSynchronize(s), "height map") ||
        !cuda_ok(cudaGetLastError(), "height map kernels")) {
        return LFB_E_CUDA;
    }
    note_launches(launches);
    return 0;
}

}  // namespace lfb
