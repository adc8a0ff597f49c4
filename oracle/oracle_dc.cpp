// CPU oracle dual-contouring mesher (TEST INFRASTRUCTURE ONLY).
//
// A depth-first restatement of the reference mesher:
//   WorkerPool::build/run      libfive/src/render/brep/worker_pool.inl:35-255
//   DCTree::evalInterval       libfive/src/render/brep/dc/dc_tree.inl:94-128
//   DCTree::evalLeaf           dc_tree.inl:131-552 (no neighbour sharing:
//                              every cell evaluates its own corners/edges)
//   DCTree::collectChildren    dc_tree.inl:581-735, dc_tree3.cpp:16-109
//   Dual<3>::work/face3/edge3  libfive/include/libfive/render/brep/dual.hpp:126-203
//   DCMesher::load             libfive/src/render/brep/dc/dc_mesher.cpp:18-169
// It shares two pieces with the product library because the reference's own
// implementations of them cannot be built here: the constant tables
// (dc_tables.hpp, generated by the reference's algorithm) and the FP64 QEF
// solve (qef.h, replacing Eigen's SelfAdjointEigenSolver).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <array>
#include <atomic>
#include <chrono>
#include <thread>
#include <vector>

#include "dc_tables.hpp"
#include "oracle_dc.hpp"
#include "oracle_eval.hpp"
#include "qef.h"

namespace ora {

using lfb::Qef;

static const lfb::DcTables& tables()
{
    static lfb::DcTables t;
    static bool init = [] { lfb::build_dc_tables(t); return true; }();
    (void)init;
    return t;
}

enum { UNKNOWN = -1, EMPTY = 0, FILLED = 1, AMBIGUOUS = 2 };

struct Leaf {
    double verts[4][3] = {};
    uint8_t corner_mask = 0;
    int vertex_count = 0;
    bool manifold = false;
    int rank = 0;
    int level = 0;
    Qef q{};                         // AtA / AtB / BtB and mass point
    uint32_t index[4] = {0, 0, 0, 0};
};

struct Cell {
    double lo[3], hi[3];
    int level;                       // region level: 0 at the leaves
    int type = UNKNOWN;
    std::unique_ptr<Cell> child[8];
    std::unique_ptr<Leaf> leaf;
    bool branch() const { return child[0] != nullptr; }
    const Cell* kid(int i) const { return branch() ? child[i].get() : this; }
};

namespace {

struct Builder {
    Evaluator eval;
    double max_err;
    explicit Builder(const Tape& t, double me) : eval(t), max_err(me) {}

    int corner_state(const Cell* c, int i) const
    {
        if (c->type == AMBIGUOUS) return (c->leaf->corner_mask >> i) & 1 ? FILLED : EMPTY;
        return c->type;
    }
    bool is_manifold(const Cell* c) const
    {
        return c->type == AMBIGUOUS ? c->leaf->manifold : true;
    }
    int rank_of(const Cell* c) const { return c->type == AMBIGUOUS ? c->leaf->rank : 0; }

    void corner(const Cell* c, int i, double out[3]) const
    {
        for (int a = 0; a < 3; ++a) out[a] = (i & (1 << a)) ? c->hi[a] : c->lo[a];
    }

    // -- DCTree::evalInterval ------------------------------------------------
    std::shared_ptr<Tape> eval_interval(Cell* c, const std::shared_ptr<Tape>& tape)
    {
        const Iv r = eval.interval(static_cast<float>(c->lo[0]), static_cast<float>(c->lo[1]),
                                   static_cast<float>(c->lo[2]), static_cast<float>(c->hi[0]),
                                   static_cast<float>(c->hi[1]), static_cast<float>(c->hi[2]),
                                   *tape);
        auto pushed = eval.push_interval(tape);
        if (r.nan) {
            c->type = AMBIGUOUS;
            return tape;
        }
        if (r.i.lo > 0) c->type = EMPTY;
        else if (r.i.hi < 0) c->type = FILLED;
        else c->type = AMBIGUOUS;
        return pushed;
    }

    // -- DCTree::evalLeaf ------------------------------------------------------
    void eval_leaf(Cell* c, const std::shared_ptr<Tape>& tape)
    {
        const auto& T = tables();
        int corners[8];
        float pos[8][3];
        for (int i = 0; i < 8; ++i) {
            double p[3];
            corner(c, i, p);
            for (int a = 0; a < 3; ++a) pos[i][a] = static_cast<float>(p[a]);
            eval.set(pos[i][0], pos[i][1], pos[i][2], i);
        }
        const float* vs = eval.values(8, *tape);
        float vals[8];
        std::memcpy(vals, vs, sizeof(vals));
        bool ambig[8];
        eval.ambiguous(8, *tape, ambig);
        int zeros[8], nz = 0;
        for (int i = 0; i < 8; ++i) {
            if (vals[i] > 0 || std::isnan(vals[i])) { corners[i] = EMPTY; ambig[i] = false; }
            else if (vals[i] < 0) { corners[i] = FILLED; ambig[i] = false; }
            else if (!ambig[i]) zeros[nz++] = i;
        }
        if (nz) {
            for (int k = 0; k < nz; ++k) eval.set(pos[zeros[k]][0], pos[zeros[k]][1], pos[zeros[k]][2], k);
            std::vector<float> d4(4 * nz);
            eval.derivs(nz, *tape, d4.data());
            for (int k = 0; k < nz; ++k) {
                corners[zeros[k]] = (d4[4 * k] != 0 || d4[4 * k + 1] != 0 || d4[4 * k + 2] != 0)
                    ? FILLED : EMPTY;
            }
        }
        for (int i = 0; i < 8; ++i) {
            if (ambig[i]) {
                corners[i] = eval.is_inside(pos[i][0], pos[i][1], pos[i][2], tape) ? FILLED : EMPTY;
            }
        }
        bool all_full = true, all_empty = true;
        for (int i = 0; i < 8; ++i) {
            all_full &= corners[i] == FILLED;
            all_empty &= corners[i] == EMPTY;
        }
        c->type = all_empty ? EMPTY : all_full ? FILLED : AMBIGUOUS;
        if (c->type != AMBIGUOUS) return;

        c->leaf.reset(new Leaf);
        Leaf& L = *c->leaf;
        for (int i = 0; i < 8; ++i) L.corner_mask |= (corners[i] == FILLED) << i;
        L.manifold = T.manifold[L.corner_mask];

        // Intersections by directed edge id (one object per edge of this cell)
        struct Inter { Qef q; bool used = false; };
        Inter inter[24];
        for (auto& it : inter) lfb::qef_zero(it.q);

        const int npatch = T.npatch[L.corner_mask];
        for (int patch = 0; patch < npatch; ++patch) {
            const int ne = T.nedge[L.corner_mask][patch];
            int edges[12];
            double targets[12][2][3];
            for (int k = 0; k < ne; ++k) {
                const int a = T.v[L.corner_mask][patch][k][0];
                const int b = T.v[L.corner_mask][patch][k][1];
                edges[k] = T.e[a][b];
                corner(c, a, targets[k][0]);
                corner(c, b, targets[k][1]);
            }
            // Edges already evaluated by an earlier patch keep their samples
            // (in the reference, this is the intersection pointer reuse).
            int eval_idx[12], ne_eval = 0;
            for (int k = 0; k < ne; ++k) {
                if (!inter[edges[k]].used) eval_idx[ne_eval++] = k;
            }
            for (int s = 0; s < 4; ++s) {
                double ps[192][3];
                for (int q = 0; q < ne_eval; ++q) {
                    const int k = eval_idx[q];
                    for (int j = 0; j < 16; ++j) {
                        const double frac = j / (16 - 1.0);
                        const int i = j + q * 16;
                        for (int a = 0; a < 3; ++a) {
                            ps[i][a] = targets[k][0][a] * (1 - frac) + targets[k][1][a] * frac;
                        }
                        eval.set(static_cast<float>(ps[i][0]), static_cast<float>(ps[i][1]),
                                 static_cast<float>(ps[i][2]), i);
                    }
                }
                if (!ne_eval) continue;
                std::vector<float> out(16 * ne_eval);
                const float* r = eval.values(16 * ne_eval, *tape);
                std::memcpy(out.data(), r, out.size() * sizeof(float));
                for (int q = 0; q < ne_eval; ++q) {
                    const int k = eval_idx[q];
                    for (int j = 1; j < 16; ++j) {
                        const int i = j + q * 16;
                        if (out[i] > 0) {
                            std::memcpy(targets[k][0], ps[i - 1], sizeof(double) * 3);
                            std::memcpy(targets[k][1], ps[i], sizeof(double) * 3);
                            break;
                        } else if (out[i] == 0) {
                            if (!eval.is_inside(static_cast<float>(ps[i][0]),
                                                static_cast<float>(ps[i][1]),
                                                static_cast<float>(ps[i][2]), tape)) {
                                std::memcpy(targets[k][0], ps[i - 1], sizeof(double) * 3);
                                std::memcpy(targets[k][1], ps[i], sizeof(double) * 3);
                                break;
                            }
                        } else if (j == 15) {
                            std::memcpy(targets[k][0], ps[i - 1], sizeof(double) * 3);
                            std::memcpy(targets[k][1], ps[i], sizeof(double) * 3);
                            break;
                        }
                    }
                }
            }
            if (ne_eval) {
                for (int q = 0; q < ne_eval; ++q) {
                    const int k = eval_idx[q];
                    for (int side = 0; side < 2; ++side) {
                        eval.set(static_cast<float>(targets[k][side][0]),
                                 static_cast<float>(targets[k][side][1]),
                                 static_cast<float>(targets[k][side][2]), 2 * q + side);
                    }
                }
                std::vector<float> d4(4 * 2 * ne_eval);
                eval.derivs(2 * ne_eval, *tape, d4.data());
                bool amb[24];
                eval.ambiguous(2 * ne_eval, *tape, amb);
                for (int i = 0; i < 2 * ne_eval; ++i) {
                    const int k = eval_idx[i / 2];
                    const double* p = targets[k][i & 1];
                    Inter& it = inter[edges[k]];
                    if (!amb[i]) {
                        const double g[3] = {d4[4 * i], d4[4 * i + 1], d4[4 * i + 2]};
                        lfb::qef_push(it.q, p, g, static_cast<double>(d4[4 * i + 3]));
                        it.used = true;
                    } else {
                        const auto fs = eval.features(static_cast<float>(p[0]),
                                                      static_cast<float>(p[1]),
                                                      static_cast<float>(p[2]), tape);
                        for (const auto& f : fs) {
                            const double g[3] = {f.x[0], f.x[1], f.x[2]};
                            lfb::qef_push(it.q, p, g, static_cast<double>(d4[4 * i + 3]));
                            it.used = true;
                        }
                    }
                }
            }
            // Mass point from the max-rank intersections, then the QEF sums.
            Qef q;
            lfb::qef_zero(q);
            int max_rank = 0;
            for (int k = 0; k < ne; ++k) {
                if (inter[edges[k]].used) max_rank = std::max(max_rank, lfb::qef_rank(inter[edges[k]].q));
            }
            for (int k = 0; k < ne; ++k) {
                const Inter& it = inter[edges[k]];
                if (it.used && lfb::qef_rank(it.q) == max_rank) {
                    for (int a = 0; a < 3; ++a) q.mass[a] += it.q.mass[a] / it.q.mass[3];
                    q.mass[3] += 1.0;
                }
            }
            for (int k = 0; k < ne; ++k) {
                if (inter[edges[k]].used) lfb::qef_add(q, inter[edges[k]].q);
            }
            int rank = 0;
            lfb::qef_vertex(q, L.verts[patch], &rank);
            L.rank = rank;
            L.q = q;
            L.vertex_count = patch + 1;
        }
    }

    // -- DCTree::collectChildren ----------------------------------------------
    void collect(Cell* c, const std::shared_ptr<Tape>& tape)
    {
        for (int i = 0; i < 8; ++i) {
            if (c->child[i]->branch()) return;
        }
        bool all_empty = true, all_full = true;
        int corners[8];
        for (int i = 0; i < 8; ++i) {
            corners[i] = corner_state(c->child[i].get(), i);
            all_empty &= c->child[i]->type == EMPTY;
            all_full &= c->child[i]->type == FILLED;
        }
        if (all_empty || all_full) {
            c->type = all_empty ? EMPTY : FILLED;
            for (auto& k : c->child) k.reset();
            return;
        }
        uint8_t mask = 0;
        for (int i = 0; i < 8; ++i) mask |= (corners[i] == FILLED) << i;
        bool manifold = tables().manifold[mask];
        for (int i = 0; i < 8; ++i) manifold = manifold && is_manifold(c->child[i].get());
        manifold = manifold && leafs_manifold(c, corners);
        if (!manifold) return;

        std::unique_ptr<Leaf> L(new Leaf);
        L->manifold = true;
        L->corner_mask = mask;
        for (int i = 0; i < 8; ++i) L->rank = std::max(L->rank, rank_of(c->child[i].get()));
        Qef q;
        lfb::qef_zero(q);
        for (int i = 0; i < 8; ++i) {
            const Cell* k = c->child[i].get();
            if (k->type != AMBIGUOUS) continue;
            if (k->leaf->rank == L->rank) {
                for (int a = 0; a < 4; ++a) q.mass[a] += k->leaf->q.mass[a];
            }
            lfb::qef_add(q, k->leaf->q);
        }
        const double err = lfb::qef_vertex(q, L->verts[0], nullptr);
        L->q = q;
        L->vertex_count = 1;
        bool inside = true;
        for (int a = 0; a < 3; ++a) {
            inside = inside && L->verts[0][a] >= c->lo[a] - 1e-6 && L->verts[0][a] <= c->hi[a] + 1e-6;
        }
        if (err < max_err && inside) {
            const float vf[3] = {static_cast<float>(L->verts[0][0]),
                                 static_cast<float>(L->verts[0][1]),
                                 static_cast<float>(L->verts[0][2])};
            const Tape* t = get_base(tape.get(), vf[0], vf[1], vf[2]);
            eval.set(vf[0], vf[1], vf[2], 0);
            const float value = eval.values(1, *t)[0];
            if (std::fabs(value) < max_err) {
                L->level = c->level;
                c->leaf = std::move(L);
                c->type = AMBIGUOUS;
                for (auto& k : c->child) k.reset();
            }
        }
    }

    bool leafs_manifold(const Cell* c, const int corners[8]) const
    {
        auto cs = [&](int child, int corner) { return corner_state(c->child[child].get(), corner); };
        // Coarse edge midpoints (dc_tree3.cpp:27-56)
        const int E[12][2] = {{0, 4}, {0, 1}, {0, 2}, {1, 3}, {1, 5}, {2, 3},
                              {2, 6}, {3, 7}, {4, 5}, {4, 6}, {5, 7}, {6, 7}};
        for (auto& e : E) {
            const int m = cs(e[0], e[1]);
            if (!(m == corners[e[0]] || m == corners[e[1]])) return false;
        }
        // Coarse face centres (dc_tree3.cpp:58-87)
        const int F[6][6] = {{0, 5, 0, 1, 4, 5}, {0, 6, 0, 2, 4, 6}, {0, 3, 0, 2, 1, 3},
                             {7, 1, 1, 5, 3, 7}, {7, 2, 2, 6, 3, 7}, {7, 4, 4, 6, 5, 7}};
        for (auto& f : F) {
            const int m = cs(f[0], f[1]);
            if (!(m == corners[f[2]] || m == corners[f[3]] || m == corners[f[4]] ||
                  m == corners[f[5]])) return false;
        }
        // Cube centre (dc_tree3.cpp:89-97)
        const int m = cs(0, 7);
        for (int i = 0; i < 8; ++i) {
            if (m == corners[i]) return true;
        }
        return false;
    }

    // -- recursive build (WorkerPool::run) -------------------------------------
    void build(Cell* c, const std::shared_ptr<Tape>& tape)
    {
        if (c->level > 0) {
            auto next = eval_interval(c, tape);
            if (c->type != AMBIGUOUS) return;
            subdivide(c);
            for (int i = 0; i < 8; ++i) build(c->child[i].get(), next);
            collect(c, next);
        } else {
            eval_leaf(c, tape);
        }
    }

    /// The first `split` levels of build(): cells `split` levels below `c`
    /// become tasks (built later by any thread, in any order), and the cells
    /// above them are listed children-first for their collect() once every
    /// task is done.  Same tree, same arithmetic as build().
    struct Task {
        Cell* c;
        std::shared_ptr<Tape> tape;
    };
    void build_top(Cell* c, const std::shared_ptr<Tape>& tape, int split,
                   std::vector<Task>& tasks, std::vector<Task>& post)
    {
        if (split == 0 || c->level == 0) {
            tasks.push_back({c, tape});
            return;
        }
        auto next = eval_interval(c, tape);
        if (c->type != AMBIGUOUS) return;
        subdivide(c);
        for (int i = 0; i < 8; ++i) build_top(c->child[i].get(), next, split - 1, tasks, post);
        post.push_back({c, next});
    }

    void subdivide(Cell* c)
    {
        double mid[3];
        for (int a = 0; a < 3; ++a) mid[a] = (c->lo[a] + c->hi[a]) / 2;
        for (int i = 0; i < 8; ++i) {
            Cell* k = new Cell;
            for (int a = 0; a < 3; ++a) {
                const bool up = i & (1 << a);
                k->lo[a] = up ? mid[a] : c->lo[a];
                k->hi[a] = up ? c->hi[a] : mid[a];
            }
            k->level = c->level - 1;
            c->child[i].reset(k);
        }
    }
};

// -- Dual walk + DCMesher ----------------------------------------------------
struct Mesher {
    // Vertex ids come from a counter shared by the walking threads (ids from
    // 1, as BRep does, brep.hpp:25, per_thread_brep.hpp:33-42); each thread
    // keeps (id, position) records and its own triangles.
    std::atomic<uint32_t>* next_id;
    std::vector<std::pair<uint32_t, std::array<float, 3>>> vrecs;
    std::vector<uint32_t> tris;
    explicit Mesher(std::atomic<uint32_t>* n) : next_id(n) {}

    static int Q(int a) { return a == 1 ? 2 : a == 2 ? 4 : 1; }
    static int R(int a) { return a == 1 ? 4 : a == 2 ? 1 : 2; }

    void load(int A, const Cell* ts[4])
    {
        for (int i = 0; i < 4; ++i) {
            if (ts[i]->type != AMBIGUOUS) return;
        }
        int index = 0;
        for (int i = 1; i < 4; ++i) {
            if (ts[i]->leaf->level < ts[index]->leaf->level) index = i;
        }
        const int q = Q(A), r = R(A);
        const int corners[4] = {q | r, r, q, 0};
        const int a = (ts[index]->leaf->corner_mask >> corners[index]) & 1;
        const int b = (ts[index]->leaf->corner_mask >> (corners[index] | A)) & 1;
        if (a == b) return;
        const bool D = a == 1;
        const auto& T = tables();
        const int ev[4][2] = {{q | r, q | r | A}, {r, r | A}, {q, q | A}, {0, A}};
        uint32_t vs[4];
        float P[4][3];
        for (int i = 0; i < 4; ++i) {
            const int e = D ? T.e[ev[i][0]][ev[i][1]] : T.e[ev[i][1]][ev[i][0]];
            const int vi = ts[i]->leaf->level > 0 ? 0 : T.p[ts[i]->leaf->corner_mask][e];
            Leaf& L = *const_cast<Leaf*>(ts[i]->leaf.get());
            if (L.index[vi] == 0) {
                L.index[vi] = next_id->fetch_add(1);
                vrecs.push_back({L.index[vi], {static_cast<float>(L.verts[vi][0]),
                                               static_cast<float>(L.verts[vi][1]),
                                               static_cast<float>(L.verts[vi][2])}});
            }
            for (int k = 0; k < 3; ++k) P[i][k] = static_cast<float>(L.verts[vi][k]);
            vs[i] = L.index[vi];
        }
        if (!D) {
            std::swap(vs[1], vs[2]);
            for (int k = 0; k < 3; ++k) std::swap(P[1][k], P[2][k]);
        }
        float N[4][3];
        auto norm = [&](int a_, int b_, int c_) {
            const float u[3] = {P[b_][0] - P[a_][0], P[b_][1] - P[a_][1], P[b_][2] - P[a_][2]};
            const float w[3] = {P[c_][0] - P[a_][0], P[c_][1] - P[a_][1], P[c_][2] - P[a_][2]};
            float n[3];
            {
                const float p0 = u[1] * w[2], p1 = u[2] * w[1];
                const float p2 = u[2] * w[0], p3 = u[0] * w[2];
                const float p4 = u[0] * w[1], p5 = u[1] * w[0];
                n[0] = p0 - p1; n[1] = p2 - p3; n[2] = p4 - p5;
            }
            const float s0 = n[0] * n[0], s1 = n[1] * n[1], s2 = n[2] * n[2];
            const float z = (s0 + s1) + s2;
            if (z > 0) {
                const float sq = std::sqrt(z);
                for (auto& x : n) x = x / sq;
            }
            std::memcpy(N[a_], n, sizeof(n));
        };
        norm(0, 1, 2);
        norm(1, 3, 0);
        norm(2, 0, 3);
        norm(3, 2, 1);
        auto dot = [](const float* x, const float* y) {
            const float a0 = x[0] * y[0], a1 = x[1] * y[1], a2 = x[2] * y[2];
            return (a0 + a1) + a2;
        };
        auto push = [&](uint32_t x, uint32_t y, uint32_t z) {
            if (x != y && y != z && x != z) {
                tris.push_back(x);
                tris.push_back(y);
                tris.push_back(z);
            }
        };
        if (dot(N[0], N[3]) > dot(N[1], N[2])) {
            push(vs[0], vs[1], vs[2]);
            push(vs[2], vs[1], vs[3]);
        } else {
            push(vs[0], vs[1], vs[3]);
            push(vs[0], vs[3], vs[2]);
        }
    }

    void edge3(int A, const Cell* t0, const Cell* t1, const Cell* t2, const Cell* t3)
    {
        const Cell* ts[4] = {t0, t1, t2, t3};
        bool br = false;
        for (auto t : ts) br |= t->branch();
        const int q = Q(A), r = R(A);
        if (br) {
            edge3(A, t0->kid(q | r), t1->kid(r), t2->kid(q), t3->kid(0));
            edge3(A, t0->kid(q | r | A), t1->kid(r | A), t2->kid(q | A), t3->kid(A));
        } else {
            load(A, ts);
        }
    }

    void face3(int A, const Cell* t0, const Cell* t1)
    {
        if (!(t0->branch() || t1->branch())) return;
        const int q = Q(A), r = R(A);
        for (int k : {0, q, r, q | r}) face3(A, t0->kid(k | A), t1->kid(k));
        edge3(q, t0->kid(A), t0->kid(r | A), t1->kid(0), t1->kid(r));
        edge3(q, t0->kid(q | A), t0->kid(q | r | A), t1->kid(q), t1->kid(q | r));
        edge3(r, t0->kid(A), t1->kid(0), t0->kid(A | q), t1->kid(q));
        edge3(r, t0->kid(r | A), t1->kid(r), t0->kid(r | A | q), t1->kid(r | q));
    }

    void work(const Cell* t)
    {
        for (int A : {1, 2, 4}) {
            const int q = Q(A), r = R(A);
            face3(A, t->kid(0), t->kid(A));
            face3(A, t->kid(q), t->kid(q | A));
            face3(A, t->kid(r), t->kid(r | A));
            face3(A, t->kid(q | r), t->kid(q | r | A));
        }
        for (int A : {1, 2, 4}) {
            const int q = Q(A), r = R(A);
            for (int a : {0, A}) edge3(A, t->kid(a), t->kid(q | a), t->kid(r | a), t->kid(q | r | a));
        }
    }

    void walk(const Cell* t)
    {
        if (!t->branch()) return;
        for (auto& c : t->child) walk(c.get());
        work(t);
    }
};

/// Branch cells `split` levels below t become walk tasks; the branch cells
/// above them are listed children-first.  work() at a cell reads only that
/// cell's descendants, so the tasks' subtrees are independent, and the
/// cells above run after every task (Dual<3>::walk's order constraint,
/// dual.hpp:304-385).
void walk_top(const Cell* t, int split, std::vector<const Cell*>& tasks,
              std::vector<const Cell*>& post)
{
    if (!t->branch()) return;
    if (split == 0) {
        tasks.push_back(t);
        return;
    }
    for (auto& c : t->child) walk_top(c.get(), split - 1, tasks, post);
    post.push_back(t);
}

/// Runs fn(i) for i in [0, n) on `threads` threads taking the next index
/// from a shared counter (the reference's WorkerPool keeps every core busy
/// the same way, worker_pool.inl:35-90).  fn receives the thread number.
template <class F>
void pool(size_t n, int threads, F fn)
{
    std::atomic<size_t> next{0};
    std::vector<std::thread> ts;
    for (int k = 0; k < threads; ++k) {
        ts.emplace_back([&, k] {
            for (size_t i = next++; i < n; i = next++) fn(k, i);
        });
    }
    for (auto& t : ts) t.join();
}

}  // namespace

int render_mesh(const Tape& tape, const float lo[3], const float hi[3],
                double min_feature, double max_err, int threads,
                std::vector<float>& verts, std::vector<uint32_t>& tris, int sample_stride,
                double* phase_s)
{
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    auto root = std::make_unique<Cell>();
    double md = 1e300;
    for (int a = 0; a < 3; ++a) {
        root->lo[a] = lo[a];
        root->hi[a] = hi[a];
        md = std::min(md, root->hi[a] - root->lo[a]);
    }
    root->level = static_cast<int>(std::ceil(
        std::fmax(0.0f, logf(static_cast<float>(md / min_feature))) / logf(2.0f)));
    Builder b(tape, max_err);
    threads = std::max(1, threads);
    // Cells five levels below the root (up to 32768) are the parallel tasks.
    const int split = threads > 1 ? std::min(5, root->level) : 0;
    std::vector<Builder::Task> tasks, post;
    auto t1 = clk::now(), t2 = t1;
    if (split == 0) {
        b.build(root.get(), b.eval.base);
        t1 = t2 = clk::now();
    } else {
        b.build_top(root.get(), b.eval.base, split, tasks, post);
        t1 = clk::now();
        std::vector<std::unique_ptr<Builder>> bs(threads);
        pool(tasks.size(), threads, [&](int k, size_t i) {
            if (sample_stride > 1 && i % sample_stride != 0) return;
            if (!bs[k]) bs[k] = std::make_unique<Builder>(tape, max_err);
            bs[k]->build(tasks[i].c, tasks[i].tape);
        });
        t2 = clk::now();
        if (sample_stride > 1) {
            // a timing sample: only every sample_stride-th task was built
            if (phase_s) {
                phase_s[0] = std::chrono::duration<double>(t1 - t0).count();
                phase_s[1] = std::chrono::duration<double>(t2 - t1).count();
                phase_s[2] = 0.0;
            }
            return -1;
        }
        for (auto& p : post) b.collect(p.c, p.tape);
    }
    std::atomic<uint32_t> next_id{1};
    std::vector<std::unique_ptr<Mesher>> ms;
    if (split == 0) {
        ms.push_back(std::make_unique<Mesher>(&next_id));
        ms[0]->walk(root.get());
    } else {
        std::vector<const Cell*> wt, wpost;
        walk_top(root.get(), split, wt, wpost);
        ms.resize(threads + 1);
        pool(wt.size(), threads, [&](int k, size_t i) {
            if (!ms[k]) ms[k] = std::make_unique<Mesher>(&next_id);
            ms[k]->walk(wt[i]);
        });
        ms[threads] = std::make_unique<Mesher>(&next_id);
        for (const Cell* c : wpost) ms[threads]->work(c);
    }
    // BRep::collect (brep.hpp:51-107): vertex id -> position, vertex 0 the
    // placeholder at the origin.
    verts.assign(3 * static_cast<size_t>(next_id.load()), 0.0f);
    tris.clear();
    for (auto& m : ms) {
        if (!m) continue;
        for (auto& r : m->vrecs) {
            for (int k = 0; k < 3; ++k) verts[3 * static_cast<size_t>(r.first) + k] = r.second[k];
        }
        tris.insert(tris.end(), m->tris.begin(), m->tris.end());
    }
    if (phase_s) {
        phase_s[0] = std::chrono::duration<double>(t1 - t0).count();
        phase_s[1] = std::chrono::duration<double>(t2 - t1).count();
        phase_s[2] = std::chrono::duration<double>(clk::now() - t2).count();
    }
    return root->level;
}

}  // namespace ora

extern "C" {

int ora_render_mesh(void* h, float xl, float yl, float zl, float xu, float yu,
                    float zu, double min_feature, double max_err, int threads,
                    void** verts_out, uint32_t* nverts, void** tris_out,
                    uint32_t* ntris)
{
    const ora::Tape& t = *static_cast<ora::Tape*>(h);
    std::vector<float> v;
    std::vector<uint32_t> tr;
    const float lo[3] = {xl, yl, zl}, hi[3] = {xu, yu, zu};
    const int L = ora::render_mesh(t, lo, hi, min_feature, max_err, threads, v, tr, 1, nullptr);
    // raw storage, released by ora_free whatever the element type
    void* vo = ::operator new[](std::max<size_t>(v.size(), 1) * sizeof(float));
    std::memcpy(vo, v.data(), v.size() * sizeof(float));
    void* to = ::operator new[](std::max<size_t>(tr.size(), 1) * sizeof(uint32_t));
    std::memcpy(to, tr.data(), tr.size() * sizeof(uint32_t));
    *verts_out = vo;
    *tris_out = to;
    *nverts = static_cast<uint32_t>(v.size() / 3);
    *ntris = static_cast<uint32_t>(tr.size() / 3);
    return L;
}

void ora_free(void* p) { ::operator delete[](p); }

/// Timing of the oracle mesher's phases for the CPU baseline: phase_s[0] the
/// serial top levels, [1] the parallel octree tasks, [2] collapse of the top
/// levels and the dual walk.  With sample_stride > 1 only every
/// sample_stride-th octree task is built (a bounded sample of the same
/// work), no mesh is produced, phase_s[2] is 0 and -1 is returned.
int ora_time_mesh(void* h, float xl, float yl, float zl, float xu, float yu, float zu,
                  double min_feature, double max_err, int threads, int sample_stride,
                  double* phase_s, uint32_t* ntris)
{
    const ora::Tape& t = *static_cast<ora::Tape*>(h);
    std::vector<float> v;
    std::vector<uint32_t> tr;
    const float lo[3] = {xl, yl, zl}, hi[3] = {xu, yu, zu};
    const int L = ora::render_mesh(t, lo, hi, min_feature, max_err, threads, v, tr,
                                   sample_stride, phase_s);
    if (ntris) *ntris = static_cast<uint32_t>(tr.size() / 3);
    return L;
}

}  // extern "C"
