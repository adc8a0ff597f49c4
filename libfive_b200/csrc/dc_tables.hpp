// Constant tables of the dual-contouring mesher, generated at start-up.
//
//  * Patch table (MarchingTable<3>, libfive/src/render/brep/dc/marching.cpp):
//    for each of the 256 corner masks, the surface patches inside a cell and
//    the filled->empty corner pairs (edges) that bound each patch.  It is
//    generated exactly as the reference does: the 22 base configurations of
//    Nielson's dual marching cubes (marching.cpp:114-320) are closed under
//    the three 90-degree rigid rotations, visiting masks in the same order,
//    and directed edges are numbered in order of first appearance
//    (marching.cpp:385-405).  The table has to match the reference's because
//    patch membership decides which vertex each triangle corner uses.
//  * Corner-manifold table (DCTree<3>::cornersAreManifold, dc_tree3.cpp:
//    111-154): a mask is safe to collapse when merging same-sign corners
//    along cube edges leaves at most one edge class, the test of Gerstner et
//    al. 2000 as used by Ju et al. 2002.
//
// Corner i of a cell is at (i & 1 ? upper.x : lower.x, i & 2 ? .y, i & 4 ? .z).
#pragma once
#include <cstdint>
#include <cstring>

namespace lfb {

struct DcTables {
    // v[mask][patch][k] = {filled corner, empty corner}, -1 terminated
    int8_t v[256][4][12][2];
    // e[a][b] = directed edge id (0..23) of corner pair a->b, -1 otherwise
    int8_t e[8][8];
    // p[mask][edge] = patch containing the directed edge, -1 otherwise
    int8_t p[256][24];
    uint8_t manifold[256];
    uint8_t npatch[256];
    uint8_t nedge[256][4];
};

namespace dc_tables_detail {

inline int rotate_vertex(int v, int axis)
{
    int c[3] = {(v & 1) ? 1 : -1, (v & 2) ? 1 : -1, (v & 4) ? 1 : -1};
    int r[3];
    if (axis == 0) {        // +90 degrees about X: (x, y, z) -> (x, -z, y)
        r[0] = c[0]; r[1] = -c[2]; r[2] = c[1];
    } else if (axis == 1) { // about Y: (x, y, z) -> (z, y, -x)
        r[0] = c[2]; r[1] = c[1]; r[2] = -c[0];
    } else {                // about Z: (x, y, z) -> (-y, x, z)
        r[0] = -c[1]; r[1] = c[0]; r[2] = c[2];
    }
    return (r[0] > 0 ? 1 : 0) | (r[1] > 0 ? 2 : 0) | (r[2] > 0 ? 4 : 0);
}

inline int rotate_mask(int mask, int axis)
{
    int out = 0;
    for (int i = 0; i < 8; ++i) {
        if (mask & (1 << i)) out |= 1 << rotate_vertex(i, axis);
    }
    return out;
}

// Base configurations: corner set, then patches as lists of
// (filled, empty) corner pairs; a pair (-1, -1) starts the next patch.
struct Base {
    int corners[8];
    int ncorners;
    int pairs[16][2];
    int npairs;
};

inline const Base* bases(int* count)
{
    static const Base b[] = {
        {{0}, 1, {{0, 1}, {0, 2}, {0, 4}}, 3},
        {{0, 1}, 2, {{1, 3}, {0, 2}, {0, 4}, {1, 5}}, 4},
        {{0, 5}, 2, {{0, 1}, {0, 2}, {0, 4}, {-1, -1}, {5, 7}, {5, 4}, {5, 1}}, 7},
        {{0, 7}, 2, {{0, 1}, {0, 2}, {0, 4}, {-1, -1}, {7, 6}, {7, 3}, {7, 5}}, 7},
        {{1, 2, 3}, 3, {{1, 0}, {1, 5}, {3, 7}, {2, 6}, {2, 0}}, 5},
        {{0, 1, 7}, 3, {{1, 3}, {0, 2}, {0, 4}, {1, 5}, {-1, -1}, {7, 6}, {7, 3}, {7, 5}}, 8},
        {{1, 4, 7}, 3, {{1, 3}, {1, 0}, {1, 5}, {-1, -1}, {4, 6}, {4, 5}, {4, 0},
                        {-1, -1}, {7, 6}, {7, 3}, {7, 5}}, 11},
        {{0, 1, 2, 3}, 4, {{0, 4}, {1, 5}, {3, 7}, {2, 6}}, 4},
        {{0, 2, 3, 6}, 4, {{0, 1}, {3, 1}, {3, 7}, {6, 7}, {6, 4}, {0, 4}}, 6},
        {{0, 4, 3, 7}, 4, {{0, 1}, {0, 2}, {4, 6}, {4, 5}, {-1, -1}, {3, 2}, {3, 1},
                           {7, 5}, {7, 6}}, 9},
        {{0, 2, 3, 7}, 4, {{0, 1}, {3, 1}, {7, 5}, {7, 6}, {2, 6}, {0, 4}}, 6},
        {{1, 2, 3, 4}, 4, {{4, 6}, {4, 5}, {4, 0}, {-1, -1}, {1, 0}, {1, 5}, {3, 7},
                           {2, 6}, {2, 0}}, 9},
        {{0, 3, 6, 5}, 4, {{0, 2}, {0, 4}, {0, 1}, {-1, -1}, {3, 7}, {3, 2}, {3, 1},
                           {-1, -1}, {6, 4}, {6, 2}, {6, 7}, {-1, -1}, {5, 7}, {5, 1},
                           {5, 4}}, 15},
        {{1, 3, 2, 6}, 4, {{1, 5}, {3, 7}, {6, 7}, {6, 4}, {2, 0}, {1, 0}}, 6},
        {{0, 2, 3, 5, 6}, 5, {{0, 1}, {3, 1}, {3, 7}, {6, 7}, {6, 4}, {0, 4},
                              {-1, -1}, {5, 7}, {5, 1}, {5, 4}}, 10},
        {{2, 3, 4, 5, 6}, 5, {{3, 1}, {3, 7}, {6, 7}, {5, 7}, {5, 1}, {4, 0}, {2, 0}}, 7},
        {{0, 4, 5, 6, 7}, 5, {{0, 2}, {6, 2}, {7, 3}, {5, 1}, {0, 1}}, 5},
        {{1, 2, 3, 4, 5, 6}, 6, {{1, 0}, {4, 0}, {2, 0}, {-1, -1}, {6, 7}, {5, 7}, {3, 7}}, 7},
        {{1, 2, 3, 4, 6, 7}, 6, {{1, 0}, {1, 5}, {7, 5}, {4, 5}, {4, 0}, {2, 0}}, 6},
        {{2, 3, 4, 5, 6, 7}, 6, {{4, 0}, {5, 1}, {3, 1}, {2, 0}}, 4},
        {{1, 2, 3, 4, 5, 6, 7}, 7, {{1, 0}, {4, 0}, {2, 0}}, 3},
    };
    *count = static_cast<int>(sizeof(b) / sizeof(b[0]));
    return b;
}

inline bool corners_manifold(int index)
{
    int f[8];
    for (int i = 0; i < 8; ++i) f[i] = (index >> i) & 1;
    int edges[12][2] = {{0, 1}, {0, 2}, {2, 3}, {1, 3}, {4, 5}, {4, 6},
                        {6, 7}, {5, 7}, {0, 4}, {2, 6}, {1, 5}, {3, 7}};
    int ne = 12;
    for (;;) {
        int hit = -1;
        for (int k = 0; k < ne; ++k) {
            if (f[edges[k][0]] == f[edges[k][1]]) { hit = k; break; }
        }
        if (hit < 0) break;
        // Contract the edge: every reference to corner a becomes b, and
        // edges that collapse to a point are dropped.
        const int a = edges[hit][0], b = edges[hit][1];
        int m = 0;
        for (int k = 0; k < ne; ++k) {
            int e0 = edges[k][0] == a ? b : edges[k][0];
            int e1 = edges[k][1] == a ? b : edges[k][1];
            if (e0 != e1) {
                edges[m][0] = e0;
                edges[m][1] = e1;
                ++m;
            }
        }
        ne = m;
    }
    // Count distinct unordered edges that remain.
    int distinct = 0;
    for (int k = 0; k < ne; ++k) {
        const int lo = edges[k][0] < edges[k][1] ? edges[k][0] : edges[k][1];
        const int hi = edges[k][0] < edges[k][1] ? edges[k][1] : edges[k][0];
        bool seen = false;
        for (int q = 0; q < k; ++q) {
            const int lo2 = edges[q][0] < edges[q][1] ? edges[q][0] : edges[q][1];
            const int hi2 = edges[q][0] < edges[q][1] ? edges[q][1] : edges[q][0];
            if (lo == lo2 && hi == hi2) { seen = true; break; }
        }
        if (!seen) ++distinct;
    }
    return distinct <= 1;
}

}  // namespace dc_tables_detail

inline void build_dc_tables(DcTables& t)
{
    using namespace dc_tables_detail;
    std::memset(t.v, -1, sizeof(t.v));
    std::memset(t.e, -1, sizeof(t.e));
    std::memset(t.p, -1, sizeof(t.p));

    int nb = 0;
    const Base* b = bases(&nb);
    for (int i = 0; i < nb; ++i) {
        int mask = 0;
        for (int k = 0; k < b[i].ncorners; ++k) mask |= 1 << b[i].corners[k];
        int patch = 0, edge = 0;
        for (int k = 0; k < b[i].npairs; ++k) {
            if (b[i].pairs[k][0] < 0) {
                ++patch;
                edge = 0;
                continue;
            }
            t.v[mask][patch][edge][0] = static_cast<int8_t>(b[i].pairs[k][0]);
            t.v[mask][patch][edge][1] = static_cast<int8_t>(b[i].pairs[k][1]);
            ++edge;
        }
    }

    // Close the table under rotations (marching.cpp:340-383).
    bool changed[256];
    for (int i = 0; i < 256; ++i) changed[i] = t.v[i][0][0][0] != -1;
    bool any = true;
    while (any) {
        any = false;
        for (int i = 0; i < 256; ++i) {
            if (!changed[i]) continue;
            changed[i] = false;
            for (int axis = 0; axis < 3; ++axis) {
                const int j = rotate_mask(i, axis);
                if (t.v[j][0][0][0] != -1) continue;
                changed[j] = true;
                any = true;
                for (int p = 0; p < 4 && t.v[i][p][0][0] != -1; ++p) {
                    for (int e = 0; e < 12 && t.v[i][p][e][0] != -1; ++e) {
                        t.v[j][p][e][0] = static_cast<int8_t>(rotate_vertex(t.v[i][p][e][0], axis));
                        t.v[j][p][e][1] = static_cast<int8_t>(rotate_vertex(t.v[i][p][e][1], axis));
                    }
                }
            }
        }
    }

    // Directed edge ids in order of first appearance, edge -> patch map.
    int next = 0;
    for (int i = 0; i < 256; ++i) {
        t.npatch[i] = 0;
        for (int p = 0; p < 4; ++p) t.nedge[i][p] = 0;
        for (int p = 0; p < 4 && t.v[i][p][0][0] != -1; ++p) {
            t.npatch[i] = static_cast<uint8_t>(p + 1);
            for (int e = 0; e < 12 && t.v[i][p][e][0] != -1; ++e) {
                t.nedge[i][p] = static_cast<uint8_t>(e + 1);
                int8_t& id = t.e[t.v[i][p][e][0]][t.v[i][p][e][1]];
                if (id == -1) id = static_cast<int8_t>(next++);
                t.p[i][id] = static_cast<int8_t>(p);
            }
        }
        t.manifold[i] = corners_manifold(i) ? 1 : 0;
    }
}

////////////////////////////////////////////////////////////////////////////////
// Quadtree tables (MarchingTable<2>, DCTree<2>::cornersAreManifold), built
// the same way: the four base cases of marching squares (marching.cpp:
// 66-96) closed under the 90-degree rotation of the square, directed edges
// numbered in order of first appearance.  Corner i of a square cell is at
// (i & 1 ? upper.x : lower.x, i & 2 ? upper.y : lower.y).

struct DcTables2 {
    int8_t v[16][2][4][2];   // v[mask][patch][k] = {filled, empty}, -1 terminated
    int8_t e[4][4];          // directed edge id (0..7) of a corner pair, -1 otherwise
    int8_t p[16][8];         // patch containing a directed edge, -1 otherwise
    uint8_t manifold[16];
    uint8_t npatch[16];
    uint8_t nedge[16][2];
};

namespace dc_tables_detail {

// +90 degrees about the square's centre: (x, y) -> (-y, x)
inline int rotate_vertex2(int v)
{
    const int x = (v & 1) ? 1 : -1, y = (v & 2) ? 1 : -1;
    return (-y > 0 ? 1 : 0) | (x > 0 ? 2 : 0);
}

inline int rotate_mask2(int mask)
{
    int out = 0;
    for (int i = 0; i < 4; ++i) {
        if (mask & (1 << i)) out |= 1 << rotate_vertex2(i);
    }
    return out;
}

/// The contraction test of corners_manifold on the square's four edges.
inline bool corners_manifold2(int index)
{
    int f[4];
    for (int i = 0; i < 4; ++i) f[i] = (index >> i) & 1;
    int edges[4][2] = {{0, 1}, {0, 2}, {1, 3}, {2, 3}};
    int ne = 4;
    for (;;) {
        int hit = -1;
        for (int k = 0; k < ne; ++k) {
            if (f[edges[k][0]] == f[edges[k][1]]) { hit = k; break; }
        }
        if (hit < 0) break;
        const int a = edges[hit][0], b = edges[hit][1];
        int m = 0;
        for (int k = 0; k < ne; ++k) {
            const int e0 = edges[k][0] == a ? b : edges[k][0];
            const int e1 = edges[k][1] == a ? b : edges[k][1];
            if (e0 != e1) {
                edges[m][0] = e0;
                edges[m][1] = e1;
                ++m;
            }
        }
        ne = m;
    }
    int distinct = 0;
    for (int k = 0; k < ne; ++k) {
        const int lo = edges[k][0] < edges[k][1] ? edges[k][0] : edges[k][1];
        const int hi = edges[k][0] < edges[k][1] ? edges[k][1] : edges[k][0];
        bool seen = false;
        for (int q = 0; q < k; ++q) {
            const int lo2 = edges[q][0] < edges[q][1] ? edges[q][0] : edges[q][1];
            const int hi2 = edges[q][0] < edges[q][1] ? edges[q][1] : edges[q][0];
            if (lo == lo2 && hi == hi2) { seen = true; break; }
        }
        if (!seen) ++distinct;
    }
    return distinct <= 1;
}

}  // namespace dc_tables_detail

inline void build_dc_tables2(DcTables2& t)
{
    using namespace dc_tables_detail;
    std::memset(t.v, -1, sizeof(t.v));
    std::memset(t.e, -1, sizeof(t.e));
    std::memset(t.p, -1, sizeof(t.p));
    // {mask, patch, k, filled corner, empty corner}
    static const int base[][5] = {
        {1, 0, 0, 0, 1}, {1, 0, 1, 0, 2},
        {3, 0, 0, 1, 3}, {3, 0, 1, 0, 2},
        {9, 0, 0, 0, 1}, {9, 0, 1, 0, 2}, {9, 1, 0, 3, 2}, {9, 1, 1, 3, 1},
        {7, 0, 0, 1, 3}, {7, 0, 1, 2, 3},
    };
    for (const auto& b : base) {
        t.v[b[0]][b[1]][b[2]][0] = static_cast<int8_t>(b[3]);
        t.v[b[0]][b[1]][b[2]][1] = static_cast<int8_t>(b[4]);
    }
    bool changed[16];
    for (int i = 0; i < 16; ++i) changed[i] = t.v[i][0][0][0] != -1;
    bool any = true;
    while (any) {
        any = false;
        for (int i = 0; i < 16; ++i) {
            if (!changed[i]) continue;
            changed[i] = false;
            const int j = rotate_mask2(i);
            if (t.v[j][0][0][0] != -1) continue;
            changed[j] = true;
            any = true;
            for (int p = 0; p < 2 && t.v[i][p][0][0] != -1; ++p) {
                for (int e = 0; e < 4 && t.v[i][p][e][0] != -1; ++e) {
                    t.v[j][p][e][0] = static_cast<int8_t>(rotate_vertex2(t.v[i][p][e][0]));
                    t.v[j][p][e][1] = static_cast<int8_t>(rotate_vertex2(t.v[i][p][e][1]));
                }
            }
        }
    }
    int next = 0;
    for (int i = 0; i < 16; ++i) {
        t.npatch[i] = 0;
        t.nedge[i][0] = t.nedge[i][1] = 0;
        for (int p = 0; p < 2 && t.v[i][p][0][0] != -1; ++p) {
            t.npatch[i] = static_cast<uint8_t>(p + 1);
            for (int e = 0; e < 4 && t.v[i][p][e][0] != -1; ++e) {
                t.nedge[i][p] = static_cast<uint8_t>(e + 1);
                int8_t& id = t.e[t.v[i][p][e][0]][t.v[i][p][e][1]];
                if (id == -1) id = static_cast<int8_t>(next++);
                t.p[i][id] = static_cast<int8_t>(p);
            }
        }
        t.manifold[i] = corners_manifold2(i) ? 1 : 0;
    }
}

}  // namespace lfb
