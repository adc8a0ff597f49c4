// C entry points of the CPU oracle for ctypes (TEST INFRASTRUCTURE ONLY).
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "oracle_eval.hpp"
#include "oracle_heightmap.hpp"

using namespace ora;

namespace {

struct Handle {
    Tape tape;
};

template <class F>
void parallel_chunks(uint64_t n, int threads, F fn)
{
    if (threads <= 1 || n < 4096) {
        fn(0, n);
        return;
    }
    std::vector<std::thread> ts;
    const uint64_t per = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        const uint64_t lo = t * per, hi = std::min(n, lo + per);
        if (lo >= hi) break;
        ts.emplace_back([=] { fn(lo, hi); });
    }
    for (auto& t : ts) t.join();
}

}  // namespace

extern "C" {

void* ora_tape_new(uint32_t num_clauses, uint32_t n_tape, const int32_t* clauses,
                   uint32_t n_const, const uint32_t* cslots, const float* cvals,
                   uint32_t n_vars, const uint32_t* vslots, const float* vvals,
                   uint32_t X, uint32_t Y, uint32_t Z, uint32_t root)
{
    auto h = new Handle;
    Tape& t = h->tape;
    t.num_clauses = num_clauses;
    t.X = X;
    t.Y = Y;
    t.Z = Z;
    t.root = root;
    for (uint32_t i = 0; i < n_tape; ++i) {
        t.t.push_back({clauses[4 * i], static_cast<uint32_t>(clauses[4 * i + 1]),
                       static_cast<uint32_t>(clauses[4 * i + 2]),
                       static_cast<uint32_t>(clauses[4 * i + 3])});
    }
    for (uint32_t i = 0; i < n_const; ++i) t.constants.push_back({cslots[i], cvals[i]});
    for (uint32_t i = 0; i < n_vars; ++i) {
        t.vars.push_back({vslots[i], vvals ? vvals[i] : 0.0f});
    }
    return h;
}

void ora_tape_delete(void* h) { delete static_cast<Handle*>(h); }

void ora_values(void* h_, uint64_t n, const float* x, const float* y,
                const float* z, float* out, int threads)
{
    auto h = static_cast<Handle*>(h_);
    parallel_chunks(n, threads, [&](uint64_t lo, uint64_t hi) {
        Evaluator e(h->tape);
        for (uint64_t i = lo; i < hi; i += NB) {
            const int c = static_cast<int>(std::min<uint64_t>(NB, hi - i));
            for (int k = 0; k < c; ++k) e.set(x[i + k], y[i + k], z[i + k], k);
            const float* r = e.values(c, *e.base);
            std::memcpy(out + i, r, c * sizeof(float));
        }
    });
}

void ora_derivs(void* h_, uint64_t n, const float* x, const float* y,
                const float* z, float* v, float* dx, float* dy, float* dz,
                int threads)
{
    auto h = static_cast<Handle*>(h_);
    parallel_chunks(n, threads, [&](uint64_t lo, uint64_t hi) {
        Evaluator e(h->tape);
        std::vector<float> out4(4 * NB);
        for (uint64_t i = lo; i < hi; i += NB) {
            const int c = static_cast<int>(std::min<uint64_t>(NB, hi - i));
            for (int k = 0; k < c; ++k) e.set(x[i + k], y[i + k], z[i + k], k);
            e.derivs(c, *e.base, out4.data());
            for (int k = 0; k < c; ++k) {
                v[i + k] = out4[4 * k + 3];
                dx[i + k] = out4[4 * k + 0];
                dy[i + k] = out4[4 * k + 1];
                dz[i + k] = out4[4 * k + 2];
            }
        }
    });
}

void ora_ambiguous(void* h_, uint64_t n, const float* x, const float* y,
                   const float* z, uint8_t* out)
{
    auto h = static_cast<Handle*>(h_);
    Evaluator e(h->tape);
    bool amb[NB];
    for (uint64_t i = 0; i < n; i += NB) {
        const int c = static_cast<int>(std::min<uint64_t>(NB, n - i));
        for (int k = 0; k < c; ++k) e.set(x[i + k], y[i + k], z[i + k], k);
        e.values(c, *e.base);
        e.ambiguous(c, *e.base, amb);
        for (int k = 0; k < c; ++k) out[i + k] = amb[k];
    }
}

void ora_intervals(void* h_, uint64_t n, const float* xlo, const float* xhi,
                   const float* ylo, const float* yhi, const float* zlo,
                   const float* zhi, float* lo, float* hi, uint8_t* nan,
                   int threads)
{
    auto h = static_cast<Handle*>(h_);
    parallel_chunks(n, threads, [&](uint64_t a, uint64_t b) {
        Evaluator e(h->tape);
        for (uint64_t i = a; i < b; ++i) {
            const Iv r = e.interval(xlo[i], ylo[i], zlo[i], xhi[i], yhi[i],
                                    zhi[i], *e.base);
            lo[i] = r.i.lo;
            hi[i] = r.i.hi;
            nan[i] = r.nan;
        }
    });
}

/// Length of the tape after an interval push over the box (tape.cpp:23-160).
uint32_t ora_pushed_size(void* h_, float xl, float yl, float zl, float xu,
                         float yu, float zu)
{
    auto h = static_cast<Handle*>(h_);
    Evaluator e(h->tape);
    e.interval(xl, yl, zl, xu, yu, zu, *e.base);
    auto t = e.push_interval(e.base);
    return static_cast<uint32_t>(t->t.size());
}

void ora_jacobian(void* h_, uint64_t n, const float* x, const float* y,
                  const float* z, float* out, int threads)
{
    auto h = static_cast<Handle*>(h_);
    const size_t nv = h->tape.vars.size();
    parallel_chunks(n, threads, [&](uint64_t a, uint64_t b) {
        Evaluator e(h->tape);
        for (uint64_t i = a; i < b; ++i) {
            e.jacobian(x[i], y[i], z[i], out + i * nv);
        }
    });
}

int ora_is_inside(void* h_, float x, float y, float z)
{
    auto h = static_cast<Handle*>(h_);
    Evaluator e(h->tape);
    return e.is_inside(x, y, z, e.base) ? 1 : 0;
}

int ora_features(void* h_, float x, float y, float z, float* out, int max)
{
    auto h = static_cast<Handle*>(h_);
    Evaluator e(h->tape);
    const auto fs = e.features(x, y, z, e.base);
    int i = 0;
    for (const auto& f : fs) {
        if (i >= max) break;
        out[3 * i + 0] = f.x[0];
        out[3 * i + 1] = f.x[1];
        out[3 * i + 2] = f.x[2];
        ++i;
    }
    return static_cast<int>(fs.size());
}

void ora_voxel_dims(const float lower[3], const float upper[3], const float res[3],
                    uint32_t dims[3])
{
    voxel_dims(lower, upper, res, dims);
}

void ora_voxel_pts(const float lower[3], const float upper[3], const float res[3], int axis,
                   float* out)
{
    voxel_pts(lower, upper, res, axis, out);
}

void ora_render_heightmap(void* h_, const float lower[3], const float upper[3],
                          const float res[3], int workers, float* depth, uint32_t* norm)
{
    render_heightmap(static_cast<Handle*>(h_)->tape, lower, upper, res, workers, depth, norm);
}

}  // extern "C"

// Library-call record / replay (see libm in oracle_eval.cpp).
extern "C" {
void ora_libm_mode(int mode) { ora::libm_set_mode(mode); }
void ora_libm_table(const uint64_t* keys, const uint32_t* vals, uint64_t n)
{
    ora::libm_set_table(keys, vals, n);
}
uint64_t ora_libm_take(uint64_t* out, uint64_t max) { return ora::libm_take(out, max); }
uint64_t ora_libm_misses() { return ora::libm_misses(); }
}

// The mesher's FP64 QEF routines (qef.h), for checks against an independent
// eigensolver.
#include "qef.h"
extern "C" {
void ora_sym3_eigen(const double s[6], double eval[3], double evec[9])
{
    double U[3][3];
    lfb::sym3_eigen(s, eval, U);
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) evec[3 * r + c] = U[r][c];
    }
}
int ora_qef_rank(const double ata[6])
{
    lfb::Qef q;
    lfb::qef_zero(q);
    for (int i = 0; i < 6; ++i) q.ata[i] = ata[i];
    return lfb::qef_rank(q);
}
double ora_qef_vertex(const double ata[6], const double atb[3], double btb,
                      const double mass[4], double v[3], int* rank)
{
    lfb::Qef q;
    for (int i = 0; i < 6; ++i) q.ata[i] = ata[i];
    for (int i = 0; i < 3; ++i) q.atb[i] = atb[i];
    q.btb = btb;
    for (int i = 0; i < 4; ++i) q.mass[i] = mass[i];
    return lfb::qef_vertex(q, v, rank);
}
/// The quadtree form: q = {ata xx, xy, yy, atb x, y, btb, mass x, y, count}.
double ora_qef2_vertex(const double q9[9], double v[2], int* rank)
{
    lfb::Qef2 q;
    for (int i = 0; i < 3; ++i) q.ata[i] = q9[i];
    for (int i = 0; i < 2; ++i) q.atb[i] = q9[3 + i];
    q.btb = q9[5];
    for (int i = 0; i < 3; ++i) q.mass[i] = q9[6 + i];
    return lfb::qef2_vertex(q, v, rank);
}
}

// The mesher's constant tables (dc_tables.hpp), for checks against the
// reference's own table tests.
#include "dc_tables.hpp"
extern "C" {
const void* ora_dc_tables(uint64_t* bytes)
{
    static const lfb::DcTables* t = [] {
        auto* p = new lfb::DcTables;
        lfb::build_dc_tables(*p);
        return p;
    }();
    if (bytes) *bytes = sizeof(lfb::DcTables);
    return t;
}
}
