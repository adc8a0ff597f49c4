// CPU oracle contourer (TEST INFRASTRUCTURE ONLY).
//
// A single-threaded, depth-first restatement of the reference's 2D
// dual-contouring path:
//   Contours::render                   libfive/src/render/brep/contours.cpp:25-49
//   DCTree<2>::evalInterval            libfive/src/render/brep/dc/dc_tree.inl:94-128
//   DCTree<2>::evalLeaf                dc_tree.inl:131-552 with N = 2
//   DCTree<2>::collectChildren         dc_tree.inl:581-735; leafsAreManifold and
//                                      cornersAreManifold, dc_tree2.cpp:14-46
//   Dual<2>::work / edge2              libfive/include/libfive/render/brep/dual.hpp:82-110
//   DCContourer::load                  libfive/src/render/brep/dc/dc_contourer.cpp:16-104
//   Contours::collect                  contours.cpp:118-184
// Like the mesher oracle it shares the FP64 QEF solve (qef.h, the *2
// functions) and the generated tables (dc_tables.hpp, DcTables2) with the
// product library; both are pinned separately (numpy eigh, the reference's
// table tests).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <list>
#include <memory>
#include <vector>

#include "dc_tables.hpp"
#include "oracle_eval.hpp"
#include "qef.h"

namespace ora {

namespace {

using lfb::Qef2;

const lfb::DcTables2& tables2()
{
    static lfb::DcTables2 t;
    static bool init = [] { lfb::build_dc_tables2(t); return true; }();
    (void)init;
    return t;
}

enum { UNKNOWN = -1, EMPTY = 0, FILLED = 1, AMBIGUOUS = 2 };
constexpr int AX = 1, AY = 2;   // Axis::X, Axis::Y bits

struct Leaf2 {
    double verts[2][2] = {};
    uint8_t corner_mask = 0;
    int vertex_count = 0;
    bool manifold = false;
    int rank = 0;
    int level = 0;
    Qef2 q{};
    uint32_t index[2] = {0, 0};
};

struct Cell2 {
    double lo[2], hi[2];
    int level;
    int type = UNKNOWN;
    std::unique_ptr<Cell2> child[4];
    std::unique_ptr<Leaf2> leaf;
    bool branch() const { return child[0] != nullptr; }
    const Cell2* kid(int i) const { return branch() ? child[i].get() : this; }
};

struct Builder2 {
    Evaluator eval;
    double max_err;
    double perp;
    Builder2(const Tape& t, double me, double z) : eval(t), max_err(me), perp(z) {}

    static int corner_state(const Cell2* c, int i)
    {
        if (c->type == AMBIGUOUS && c->leaf) return (c->leaf->corner_mask >> i) & 1 ? FILLED : EMPTY;
        return c->type;
    }
    static bool is_manifold(const Cell2* c)
    {
        return c->type == AMBIGUOUS ? c->leaf->manifold : true;
    }
    static int rank_of(const Cell2* c) { return c->leaf ? c->leaf->rank : 0; }

    static void corner(const Cell2* c, int i, double out[2])
    {
        for (int a = 0; a < 2; ++a) out[a] = (i & (1 << a)) ? c->hi[a] : c->lo[a];
    }
    void set(const double p[2], int i)
    {
        eval.set(static_cast<float>(p[0]), static_cast<float>(p[1]), static_cast<float>(perp), i);
    }
    float pf() const { return static_cast<float>(perp); }

    // -- evalInterval ----------------------------------------------------------
    std::shared_ptr<Tape> eval_interval(Cell2* c, const std::shared_ptr<Tape>& tape)
    {
        const Iv r = eval.interval(static_cast<float>(c->lo[0]), static_cast<float>(c->lo[1]), pf(),
                                   static_cast<float>(c->hi[0]), static_cast<float>(c->hi[1]), pf(),
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

    // -- evalLeaf (N = 2) ------------------------------------------------------
    void eval_leaf(Cell2* c, const std::shared_ptr<Tape>& tape)
    {
        const auto& T = tables2();
        int corners[4];
        double pos[4][2];
        for (int i = 0; i < 4; ++i) {
            corner(c, i, pos[i]);
            set(pos[i], i);
        }
        float vals[4];
        std::memcpy(vals, eval.values(4, *tape), sizeof(vals));
        bool ambig[4];
        eval.ambiguous(4, *tape, ambig);
        int zeros[4], nz = 0;
        for (int i = 0; i < 4; ++i) {
            if (vals[i] > 0 || std::isnan(vals[i])) { corners[i] = EMPTY; ambig[i] = false; }
            else if (vals[i] < 0) { corners[i] = FILLED; ambig[i] = false; }
            else if (!ambig[i]) zeros[nz++] = i;
        }
        if (nz) {
            for (int k = 0; k < nz; ++k) set(pos[zeros[k]], k);
            std::vector<float> d4(4 * nz);
            eval.derivs(nz, *tape, d4.data());
            for (int k = 0; k < nz; ++k) {
                corners[zeros[k]] = (d4[4 * k] != 0 || d4[4 * k + 1] != 0 || d4[4 * k + 2] != 0)
                    ? FILLED : EMPTY;
            }
        }
        for (int i = 0; i < 4; ++i) {
            if (ambig[i]) {
                corners[i] = eval.is_inside(static_cast<float>(pos[i][0]),
                                            static_cast<float>(pos[i][1]), pf(), tape)
                    ? FILLED : EMPTY;
            }
        }
        bool all_full = true, all_empty = true;
        for (int i = 0; i < 4; ++i) {
            all_full &= corners[i] == FILLED;
            all_empty &= corners[i] == EMPTY;
        }
        c->type = all_empty ? EMPTY : all_full ? FILLED : AMBIGUOUS;
        if (c->type != AMBIGUOUS) return;

        c->leaf.reset(new Leaf2);
        Leaf2& L = *c->leaf;
        for (int i = 0; i < 4; ++i) L.corner_mask |= (corners[i] == FILLED) << i;
        L.manifold = T.manifold[L.corner_mask];

        struct Inter { Qef2 q; bool used = false; };
        Inter inter[8];
        for (auto& it : inter) lfb::qef2_zero(it.q);

        const int npatch = T.npatch[L.corner_mask];
        for (int patch = 0; patch < npatch; ++patch) {
            const int ne = T.nedge[L.corner_mask][patch];
            int edges[4];
            double targets[4][2][2];
            for (int k = 0; k < ne; ++k) {
                const int a = T.v[L.corner_mask][patch][k][0];
                const int b = T.v[L.corner_mask][patch][k][1];
                edges[k] = T.e[a][b];
                corner(c, a, targets[k][0]);
                corner(c, b, targets[k][1]);
            }
            // the search (dc_tree.inl:339-410): four rounds of 16 samples
            for (int s = 0; s < 4; ++s) {
                double ps[64][2];
                for (int k = 0; k < ne; ++k) {
                    for (int j = 0; j < 16; ++j) {
                        const double frac = j / (16 - 1.0);
                        const int i = j + k * 16;
                        for (int a = 0; a < 2; ++a) {
                            ps[i][a] = targets[k][0][a] * (1 - frac) + targets[k][1][a] * frac;
                        }
                        set(ps[i], i);
                    }
                }
                std::vector<float> out(16 * ne);
                std::memcpy(out.data(), eval.values(16 * ne, *tape), out.size() * sizeof(float));
                for (int k = 0; k < ne; ++k) {
                    for (int j = 1; j < 16; ++j) {
                        const int i = j + k * 16;
                        bool hit = false;
                        if (out[i] > 0) {
                            hit = true;
                        } else if (out[i] == 0) {
                            hit = !eval.is_inside(static_cast<float>(ps[i][0]),
                                                  static_cast<float>(ps[i][1]), pf(), tape);
                        } else if (j == 15) {
                            hit = true;
                        }
                        if (hit) {
                            std::memcpy(targets[k][0], ps[i - 1], sizeof(double) * 2);
                            std::memcpy(targets[k][1], ps[i], sizeof(double) * 2);
                            break;
                        }
                    }
                }
            }
            // value and derivatives at both ends of each bracket
            for (int k = 0; k < ne; ++k) {
                for (int side = 0; side < 2; ++side) set(targets[k][side], 2 * k + side);
            }
            std::vector<float> d4(4 * 2 * ne);
            eval.derivs(2 * ne, *tape, d4.data());
            bool amb[8];
            eval.ambiguous(2 * ne, *tape, amb);
            for (int i = 0; i < 2 * ne; ++i) {
                const int k = i / 2;
                const double* p = targets[k][i & 1];
                Inter& it = inter[edges[k]];
                if (!amb[i]) {
                    const double g[2] = {d4[4 * i], d4[4 * i + 1]};
                    lfb::qef2_push(it.q, p, g, static_cast<double>(d4[4 * i + 3]));
                    it.used = true;
                } else {
                    const auto fs = eval.features(static_cast<float>(p[0]),
                                                  static_cast<float>(p[1]), pf(), tape);
                    for (const auto& f : fs) {
                        const double g[2] = {f.x[0], f.x[1]};
                        lfb::qef2_push(it.q, p, g, static_cast<double>(d4[4 * i + 3]));
                        it.used = true;
                    }
                }
            }
            // mass point from the max-rank intersections, then the QEF sums
            Qef2 q;
            lfb::qef2_zero(q);
            int max_rank = 0;
            for (int k = 0; k < ne; ++k) {
                if (inter[edges[k]].used) max_rank = std::max(max_rank, lfb::qef2_rank(inter[edges[k]].q));
            }
            for (int k = 0; k < ne; ++k) {
                const Inter& it = inter[edges[k]];
                if (it.used && lfb::qef2_rank(it.q) == max_rank) {
                    for (int a = 0; a < 2; ++a) q.mass[a] += it.q.mass[a] / it.q.mass[2];
                    q.mass[2] += 1.0;
                }
            }
            for (int k = 0; k < ne; ++k) {
                if (inter[edges[k]].used) lfb::qef2_add(q, inter[edges[k]].q);
            }
            int rank = 0;
            lfb::qef2_vertex(q, L.verts[patch], &rank);
            L.rank = rank;
            L.q = q;
            L.vertex_count = patch + 1;
        }
    }

    // -- collectChildren (N = 2) -----------------------------------------------
    static bool leafs_manifold(const Cell2* c, const int corners[4])
    {
        auto cs = [&](int child, int corner) { return corner_state(c->child[child].get(), corner); };
        const bool edges_safe =
            (cs(0, AX) == corners[0] || cs(0, AX) == corners[AX]) &&
            (cs(0, AY) == corners[0] || cs(0, AY) == corners[AY]) &&
            (cs(AX, AX | AY) == corners[AX] || cs(AX, AX | AY) == corners[AX | AY]) &&
            (cs(AY, AY | AX) == corners[AY] || cs(AY, AY | AX) == corners[AY | AX]);
        const int m = cs(0, AX | AY);
        const bool faces_safe = m == corners[0] || m == corners[AY] || m == corners[AX] ||
                                m == corners[AX | AY];
        return edges_safe && faces_safe;
    }

    void collect(Cell2* c, const std::shared_ptr<Tape>& tape)
    {
        for (int i = 0; i < 4; ++i) {
            if (c->child[i]->branch()) return;
        }
        bool all_empty = true, all_full = true;
        int corners[4];
        for (int i = 0; i < 4; ++i) {
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
        for (int i = 0; i < 4; ++i) mask |= (corners[i] == FILLED) << i;
        bool manifold = tables2().manifold[mask];
        for (int i = 0; i < 4; ++i) manifold = manifold && is_manifold(c->child[i].get());
        manifold = manifold && leafs_manifold(c, corners);
        if (!manifold) return;

        std::unique_ptr<Leaf2> L(new Leaf2);
        L->manifold = true;
        L->corner_mask = mask;
        for (int i = 0; i < 4; ++i) L->rank = std::max(L->rank, rank_of(c->child[i].get()));
        Qef2 q;
        lfb::qef2_zero(q);
        for (int i = 0; i < 4; ++i) {
            const Cell2* k = c->child[i].get();
            if (k->type != AMBIGUOUS) continue;
            if (k->leaf->rank == L->rank) {
                for (int a = 0; a < 3; ++a) q.mass[a] += k->leaf->q.mass[a];
            }
            lfb::qef2_add(q, k->leaf->q);
        }
        const double err = lfb::qef2_vertex(q, L->verts[0], nullptr);
        L->q = q;
        L->vertex_count = 1;
        bool inside = true;
        for (int a = 0; a < 2; ++a) {
            inside = inside && L->verts[0][a] >= c->lo[a] - 1e-6 && L->verts[0][a] <= c->hi[a] + 1e-6;
        }
        if (err < max_err && inside) {
            const float vf[3] = {static_cast<float>(L->verts[0][0]),
                                 static_cast<float>(L->verts[0][1]), pf()};
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

    // -- recursive build (WorkerPool::run) -------------------------------------
    void build(Cell2* c, const std::shared_ptr<Tape>& tape)
    {
        if (c->level > 0) {
            auto next = eval_interval(c, tape);
            if (c->type != AMBIGUOUS) return;
            subdivide(c);
            for (int i = 0; i < 4; ++i) build(c->child[i].get(), next);
            collect(c, next);
        } else {
            eval_leaf(c, tape);
        }
    }

    static void subdivide(Cell2* c)
    {
        double mid[2];
        for (int a = 0; a < 2; ++a) mid[a] = (c->lo[a] + c->hi[a]) / 2;
        for (int i = 0; i < 4; ++i) {
            Cell2* k = new Cell2;
            for (int a = 0; a < 2; ++a) {
                const bool up = i & (1 << a);
                k->lo[a] = up ? mid[a] : c->lo[a];
                k->hi[a] = up ? c->hi[a] : mid[a];
            }
            k->level = c->level - 1;
            c->child[i].reset(k);
        }
    }
};

// -- Dual<2> walk + DCContourer ----------------------------------------------
struct Contourer {
    std::vector<std::array<float, 2>> verts{{0.0f, 0.0f}};   // index 0 unused
    std::vector<std::array<uint32_t, 2>> segs;

    void push(const Cell2* ts[2], int A, bool D)
    {
        const auto& T = tables2();
        int es[2];
        if (D ^ (A == AX)) {
            es[0] = T.e[3][3 ^ A];
            es[1] = T.e[A][0];
        } else {
            es[0] = T.e[3 ^ A][3];
            es[1] = T.e[0][A];
        }
        uint32_t vs[2];
        for (int i = 0; i < 2; ++i) {
            Leaf2& L = *const_cast<Cell2*>(ts[i])->leaf;
            const int vi = L.level > 0 ? 0 : T.p[L.corner_mask][es[i]];
            if (L.index[vi] == 0) {
                L.index[vi] = static_cast<uint32_t>(verts.size());
                verts.push_back({static_cast<float>(L.verts[vi][0]),
                                 static_cast<float>(L.verts[vi][1])});
            }
            vs[i] = L.index[vi];
        }
        segs.push_back({vs[!D], vs[D]});
    }

    void load(const Cell2* ts[2], int A)
    {
        for (int i = 0; i < 2; ++i) {
            if (ts[i]->type != AMBIGUOUS) return;
        }
        const int index = ts[1]->leaf->level < ts[0]->leaf->level ? 1 : 0;
        const int perp = (AX | AY) ^ A;
        const int corners[2] = {perp, 0};
        const int a = Builder2::corner_state(ts[index], corners[index]);
        const int b = Builder2::corner_state(ts[index], corners[index] | A);
        if (a == b) return;
        const bool fwd = (a == FILLED && A == AY) || (b == FILLED && A == AX);
        push(ts, A, !fwd);
    }

    void edge2(const Cell2* t0, const Cell2* t1, int A)
    {
        const int perp = (AX | AY) ^ A;
        if (t0->branch() || t1->branch()) {
            edge2(t0->kid(perp), t1->kid(0), A);
            edge2(t0->kid(A | perp), t1->kid(A), A);
        } else if (t0->type == AMBIGUOUS && t1->type == AMBIGUOUS) {
            const Cell2* ts[2] = {t0, t1};
            load(ts, A);
        }
    }

    void work(const Cell2* t)
    {
        edge2(t->kid(0), t->kid(AX), AY);
        edge2(t->kid(AY), t->kid(AY | AX), AY);
        edge2(t->kid(0), t->kid(AY), AX);
        edge2(t->kid(AX), t->kid(AX | AY), AX);
    }

    // children first, then the cell (the walk's completion order)
    void walk(const Cell2* t)
    {
        if (!t->branch()) return;
        for (int i = 0; i < 4; ++i) walk(t->child[i].get());
        work(t);
    }
};

}  // namespace

/// Contours::collect: segments welded into polylines, in segment order.
void weld_contours(const std::vector<std::array<uint32_t, 2>>& segs,
                   std::vector<std::vector<uint32_t>>& out)
{
    std::map<uint32_t, uint32_t> heads, tails;
    std::vector<std::list<uint32_t>> cs;
    for (const auto& s : segs) {
        auto t = tails.find(s[0]);
        if (t != tails.end()) {
            const uint32_t k = t->second;
            cs[k].push_back(s[1]);
            tails.insert({s[1], k});
            tails.erase(t);
            continue;
        }
        auto h = heads.find(s[1]);
        if (h != heads.end()) {
            const uint32_t k = h->second;
            cs[k].push_front(s[0]);
            heads.insert({s[0], k});
            heads.erase(h);
            continue;
        }
        heads[s[0]] = static_cast<uint32_t>(cs.size());
        tails[s[1]] = static_cast<uint32_t>(cs.size());
        cs.push_back({s[0], s[1]});
    }
    std::vector<bool> done(cs.size(), false);
    for (size_t i = 0; i < cs.size(); ++i) {
        if (done[i]) continue;
        out.emplace_back();
        size_t target = i;
        for (;;) {
            for (uint32_t p : cs[target]) out.back().push_back(p);
            done[target] = true;
            auto h = heads.find(cs[target].back());
            if (h != heads.end() && !done[h->second]) {
                out.back().pop_back();
                target = h->second;
            } else {
                break;
            }
        }
    }
}

/// Contours::render on the CPU: points of every contour, x and y
/// interleaved, and their counts.  Returns the quadtree depth.
int render_contours(const Tape& tape, const double lo[2], const double hi[2], double z,
                    double min_feature, double max_err, std::vector<float>& pts,
                    std::vector<uint32_t>& counts)
{
    // Region<2>::withResolution (region.hpp:226-231)
    const double md = std::min(hi[0] - lo[0], hi[1] - lo[1]);
    const int level = static_cast<int>(
        std::ceil(std::fmax(0.0f, std::log(static_cast<float>(md / min_feature))) /
                  std::log(2.0f)));
    Builder2 b(tape, max_err, z);
    Cell2 root;
    for (int a = 0; a < 2; ++a) {
        root.lo[a] = lo[a];
        root.hi[a] = hi[a];
    }
    root.level = level;
    auto t = std::make_shared<Tape>(tape);
    b.build(&root, t);
    Contourer m;
    m.walk(&root);
    std::vector<std::vector<uint32_t>> welded;
    weld_contours(m.segs, welded);
    pts.clear();
    counts.clear();
    for (const auto& c : welded) {
        counts.push_back(static_cast<uint32_t>(c.size()));
        for (uint32_t k : c) {
            pts.push_back(m.verts[k][0]);
            pts.push_back(m.verts[k][1]);
        }
    }
    return level;
}

}  // namespace ora

extern "C" {

/// ora_render_contours: see render_contours.  The arrays are released by
/// ora_free.
int ora_render_contours(void* h, double xl, double yl, double xu, double yu, double z,
                        double min_feature, double max_err, void** pts_out,
                        uint32_t* n_pts, void** counts_out, uint32_t* n_contours)
{
    const ora::Tape& t = *static_cast<ora::Tape*>(h);
    std::vector<float> p;
    std::vector<uint32_t> c;
    const double lo[2] = {xl, yl}, hi[2] = {xu, yu};
    const int L = ora::render_contours(t, lo, hi, z, min_feature, max_err, p, c);
    void* po = ::operator new[](std::max<size_t>(p.size(), 1) * sizeof(float));
    std::memcpy(po, p.data(), p.size() * sizeof(float));
    void* co = ::operator new[](std::max<size_t>(c.size(), 1) * sizeof(uint32_t));
    std::memcpy(co, c.data(), c.size() * sizeof(uint32_t));
    *pts_out = po;
    *counts_out = co;
    *n_pts = static_cast<uint32_t>(p.size() / 2);
    *n_contours = static_cast<uint32_t>(c.size());
    return L;
}

/// The quadtree tables (DcTables2) for the table tests.
void ora_dc_tables2(void* out) { lfb::build_dc_tables2(*static_cast<lfb::DcTables2*>(out)); }

/// Contours::collect on given segments (for tests of the welding rule):
/// counts[i] points of contour i in out (vertex ids).
uint32_t ora_weld(const uint32_t* segs, uint32_t n, uint32_t* out, uint32_t* counts)
{
    std::vector<std::array<uint32_t, 2>> s(n);
    for (uint32_t i = 0; i < n; ++i) s[i] = {segs[2 * i], segs[2 * i + 1]};
    std::vector<std::vector<uint32_t>> w;
    ora::weld_contours(s, w);
    uint32_t k = 0;
    for (size_t i = 0; i < w.size(); ++i) {
        counts[i] = static_cast<uint32_t>(w[i].size());
        for (uint32_t v : w[i]) out[k++] = v;
    }
    return static_cast<uint32_t>(w.size());
}

}  // extern "C"
