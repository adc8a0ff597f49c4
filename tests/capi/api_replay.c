/*
 * A plain C program against the unchanged libfive.h, linked to this
 * library's lib/libfive.so: the C-API cases of libfive/test/api.cpp that the
 * evaluate-and-mesh path serves, replayed through the C ABI.
 *
 *   libfive_opcode_enum       api.cpp:21-29
 *   libfive_tree identity     api.cpp:31-42
 *   libfive_tree_eval_f       api.cpp:44-57   (exact values)
 *   libfive_tree_eval_r       api.cpp:59-73   (exact bounds)
 *   libfive_tree_eval_d       (derivatives of the same quotient)
 *   libfive_tree_render_mesh  api.cpp:107-146 (unit sphere radii)
 *   libfive_tree_save_mesh    (binary STL: 80-byte header, count, records)
 *   libfive_tree_render_pixels api.cpp:175-193 (no crash)
 *   libfive_tree_print        api.cpp:195-215
 *   nullary / unary / binary  api.cpp:217-252 (NULL for invalid opcodes)
 *
 * Prints "api_replay ok" and exits 0 when every check passes; otherwise
 * prints the failing check and exits 1.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "libfive.h"

static int failures = 0;
#define CHECK(c)                                                         \
    do {                                                                 \
        if (!(c)) {                                                      \
            fprintf(stderr, "api_replay: check failed at line %d: %s\n", \
                    __LINE__, #c);                                       \
            ++failures;                                                  \
        }                                                                \
    } while (0)

static int op(const char* name) { return libfive_opcode_enum(name); }

static libfive_tree unit_sphere(libfive_tree* keep)
{
    libfive_tree x = libfive_tree_x(), y = libfive_tree_y(), z = libfive_tree_z();
    libfive_tree x2 = libfive_tree_unary(op("square"), x);
    libfive_tree y2 = libfive_tree_unary(op("square"), y);
    libfive_tree z2 = libfive_tree_unary(op("square"), z);
    libfive_tree r_ = libfive_tree_binary(op("add"), x2, y2);
    libfive_tree r = libfive_tree_binary(op("add"), r_, z2);
    libfive_tree one = libfive_tree_const(1.0f);
    libfive_tree d = libfive_tree_binary(op("sub"), r, one);
    libfive_tree all[9] = {x, y, z, x2, y2, z2, r_, r, one};
    memcpy(keep, all, sizeof(all));
    return d;
}

int main(int argc, char** argv)
{
    const char* stl = argc > 1 ? argv[1] : "api_replay.stl";

    /* libfive_opcode_enum */
    CHECK(op("min") >= 0 && op("max") >= 0 && op("VAR-X") >= 0);
    CHECK(op("min") != op("max"));
    CHECK(op("wat") == -1);
    CHECK(op("") == -1);

    /* libfive_tree: x is one node, y another */
    {
        libfive_tree a = libfive_tree_x(), b = libfive_tree_x(), c = libfive_tree_y();
        CHECK(a == b);
        CHECK(b != c);
        libfive_tree_delete(a);
        libfive_tree_delete(b);
        libfive_tree_delete(c);
    }

    /* eval_f / eval_r / eval_d */
    {
        libfive_tree a = libfive_tree_x(), b = libfive_tree_y();
        libfive_tree c = libfive_tree_binary(op("div"), a, b);
        libfive_vec3 p1 = {1, 2, 3}, p2 = {1, 4, 3}, p3 = {1, -1, 3};
        CHECK(libfive_tree_eval_f(c, p1) == 0.5f);
        CHECK(libfive_tree_eval_f(c, p2) == 0.25f);
        CHECK(libfive_tree_eval_f(c, p3) == -1.0f);
        libfive_vec3 d = libfive_tree_eval_d(c, p1);   /* d(x/y) = (1/y, -x/y^2, 0) */
        CHECK(d.x == 0.5f && d.y == -0.25f && d.z == 0.0f);

        libfive_tree s = libfive_tree_binary(op("sub"), a, b);
        libfive_region3 R = {{1, 2}, {2, 3}, {0, 0}};
        libfive_interval r = libfive_tree_eval_r(s, R);
        CHECK(r.lower == -2.0f);
        CHECK(r.upper == 0.0f);
        libfive_tree_delete(a);
        libfive_tree_delete(b);
        libfive_tree_delete(c);
        libfive_tree_delete(s);
    }

    /* render_mesh: every vertex of every triangle on the unit sphere */
    {
        libfive_tree keep[9];
        libfive_tree d = unit_sphere(keep);
        libfive_region3 R = {{-2, 2}, {-2, 2}, {-2, 2}};
        libfive_mesh* m = libfive_tree_render_mesh(d, R, 10);
        CHECK(m != NULL);
        if (m) {
            CHECK(m->tri_count > 0);
            float rmin = 2, rmax = 0;
            for (unsigned i = 0; i < m->tri_count; ++i) {
                const uint32_t ids[3] = {m->tris[i].a, m->tris[i].b, m->tris[i].c};
                for (int k = 0; k < 3; ++k) {
                    const libfive_vec3 v = m->verts[ids[k]];
                    const float rr = v.x * v.x + v.y * v.y + v.z * v.z;
                    rmin = fminf(rmin, rr);
                    rmax = fmaxf(rmax, rr);
                }
            }
            CHECK(rmin > 0.99f);
            CHECK(rmax < 1.01f);

            /* save_mesh: binary STL with the same triangle count */
            CHECK(libfive_tree_save_mesh(d, R, 10, stl));
            FILE* f = fopen(stl, "rb");
            CHECK(f != NULL);
            if (f) {
                unsigned char head[84];
                CHECK(fread(head, 1, 84, f) == 84);
                uint32_t n = 0;
                memcpy(&n, head + 80, 4);
                CHECK(n == m->tri_count);
                fseek(f, 0, SEEK_END);
                CHECK(ftell(f) == 84 + 50 * (long)n);
                fclose(f);
            }
            libfive_mesh_delete(m);
        }

        libfive_region2 R2 = {{-2, 2}, {-2, 2}};
        libfive_pixels* px = libfive_tree_render_pixels(d, R2, 0, 10);
        CHECK(px != NULL);
        if (px) libfive_pixels_delete(px);

        char* s = libfive_tree_print(d);
        CHECK(s && strcmp(s, "(- (+ (square x) (square y) (square z)) 1)") == 0);
        free(s);
        for (int i = 0; i < 9; ++i) libfive_tree_delete(keep[i]);
        libfive_tree_delete(d);
    }

    /* libfive_tree_render_slice (api.cpp:75-105): x^2 + y^2 - 1 cut at z = 0,
     * one contour, every point at radius^2 in (0.99, 1.01) */
    {
        libfive_tree x = libfive_tree_x(), y = libfive_tree_y();
        libfive_tree x2 = libfive_tree_unary(op("square"), x);
        libfive_tree y2 = libfive_tree_unary(op("square"), y);
        libfive_tree r = libfive_tree_binary(op("add"), x2, y2);
        libfive_tree one = libfive_tree_const(1.0f);
        libfive_tree d = libfive_tree_binary(op("sub"), r, one);
        libfive_region2 R = {{-2, 2}, {-2, 2}};
        libfive_contours* cs = libfive_tree_render_slice(d, R, 0, 10);
        CHECK(cs != NULL);
        if (cs) {
            CHECK(cs->count == 1);
            if (cs->count == 1) {
                CHECK(cs->cs[0].count > 0);
                float rmin = 2, rmax = 0;
                for (uint32_t i = 0; i < cs->cs[0].count; ++i) {
                    const libfive_vec2 v = cs->cs[0].pts[i];
                    const float q = v.x * v.x + v.y * v.y;
                    rmin = q < rmin ? q : rmin;
                    rmax = q > rmax ? q : rmax;
                }
                CHECK(rmin > 0.99f && rmax < 1.01f);
            }
            libfive_contours_delete(cs);
        }
        libfive_tree ts[7] = {x, y, x2, y2, r, one, d};
        for (int i = 0; i < 7; ++i) libfive_tree_delete(ts[i]);
    }

    /* invalid opcodes and arguments give NULL */
    {
        CHECK(libfive_tree_nullary(op("min")) == NULL);
        libfive_tree vx = libfive_tree_nullary(op("var-x"));
        CHECK(vx != NULL);
        libfive_tree_delete(vx);

        libfive_tree x = libfive_tree_x(), y = libfive_tree_y();
        CHECK(libfive_tree_unary(op("add"), x) == NULL);
        CHECK(libfive_tree_unary(op("cos"), NULL) == NULL);
        CHECK(libfive_tree_unary(op("add"), NULL) == NULL);
        libfive_tree t = libfive_tree_unary(op("cos"), x);
        CHECK(t != NULL);
        libfive_tree_delete(t);
        CHECK(libfive_tree_binary(op("cos"), x, y) == NULL);
        CHECK(libfive_tree_binary(op("add"), x, NULL) == NULL);
        CHECK(libfive_tree_binary(op("add"), NULL, y) == NULL);
        t = libfive_tree_binary(op("add"), x, y);
        CHECK(t != NULL);
        libfive_tree_delete(t);
        libfive_tree_delete(x);
        libfive_tree_delete(y);
    }

    if (failures) {
        fprintf(stderr, "api_replay: %d check(s) failed\n", failures);
        return 1;
    }
    printf("api_replay ok\n");
    return 0;
}
