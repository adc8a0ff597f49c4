/*
 *  libfive C API, served by the B200 implementation in this repository.
 *
 *  The structs and function signatures are identical to the reference
 *  header (libfive/include/libfive.h), so C programs, the Python ctypes
 *  binding (libfive/bind/python/libfive/ffi.py) and the Guile FFI
 *  (libfive/bind/guile/libfive/lib.scm) link against this library without
 *  source changes.  Each declaration cites the reference declaration it
 *  replaces.  Tree handles are opaque pointers; meshes and strings returned
 *  here are freed with the matching *_delete / libfive_free_str call.
 *
 *  Functions outside the evaluate-and-mesh path (2D slices and contours,
 *  pixel rendering, tree serialization) are declared for link compatibility
 *  and report "unsupported" as described next to each of them.
 */
#pragma once

#ifdef __cplusplus
#include <cstdint>
extern "C" {
#else
#include <stdint.h>
#include <stdbool.h>
#endif

/* libfive.h:26 */
typedef struct libfive_interval  { float lower; float upper; } libfive_interval;
/* libfive.h:31 */
typedef struct libfive_region2   { libfive_interval X, Y; } libfive_region2;
/* libfive.h:36 */
typedef struct libfive_region3   { libfive_interval X, Y, Z; } libfive_region3;
/* libfive.h:41 */
typedef struct libfive_vec2      { float x, y; } libfive_vec2;
/* libfive.h:46 */
typedef struct libfive_vec3      { float x, y, z; } libfive_vec3;
/* libfive.h:51 */
typedef struct libfive_vec4      { float x, y, z, w; } libfive_vec4;
/* libfive.h:57 */
typedef struct libfive_tri       { uint32_t a, b, c; } libfive_tri;

/* libfive.h:63-66 */
typedef struct libfive_contour {
    libfive_vec2* pts;
    uint32_t count;
} libfive_contour;

/* libfive.h:72-75 */
typedef struct libfive_contours {
    libfive_contour* cs;
    uint32_t count;
} libfive_contours;

/* libfive.h:81-84 */
typedef struct libfive_contour3 {
    libfive_vec3* pts;
    uint32_t count;
} libfive_contour3;

/* libfive.h:90-93 */
typedef struct libfive_contours3 {
    libfive_contour3* cs;
    uint32_t count;
} libfive_contours3;

/* libfive.h:99-104: verts[0] is an unused (0, 0, 0) placeholder and
 * triangle indices start at 1, as in the reference. */
typedef struct libfive_mesh {
    libfive_vec3* verts;
    libfive_tri* tris;
    uint32_t tri_count;
    uint32_t vert_count;
} libfive_mesh;

/* libfive.h:113-118 */
typedef struct libfive_mesh_coords {
    libfive_vec3* verts;
    uint32_t vert_count;
    int32_t* coord_indices;
    uint32_t coord_index_count;
} libfive_mesh_coords;

/* libfive.h:124-128 */
typedef struct libfive_pixels {
    bool* pixels;
    uint32_t width;
    uint32_t height;
} libfive_pixels;

/* libfive.h:135 */
void libfive_contours_delete(libfive_contours* cs);
/* libfive.h:140 */
void libfive_contours3_delete(libfive_contours3* cs);
/* libfive.h:145 */
void libfive_mesh_delete(libfive_mesh* m);
/* libfive.h:150 */
void libfive_mesh_coords_delete(libfive_mesh_coords* m);
/* libfive.h:155 */
void libfive_pixels_delete(libfive_pixels* ps);
/* libfive.h:161: -1 when the name is unknown */
int libfive_opcode_enum(const char* op);
/* libfive.h:167: 0, 1, 2 or -1 */
int libfive_opcode_args(int op);

/* libfive.h:174-178 */
typedef struct libfive_vars {
    void* const* vars;
    float* values;
    uint32_t size;
} libfive_vars;
/* libfive.h:179 */
void libfive_vars_delete(libfive_vars* j);

typedef struct libfive_tree_ libfive_tree_;
typedef struct libfive_tree_* libfive_tree;
typedef struct libfive_evaluator_ libfive_evaluator_;
typedef struct libfive_evaluator_* libfive_evaluator;

/* libfive.h:196-206 */
libfive_tree libfive_tree_x(void);
libfive_tree libfive_tree_y(void);
libfive_tree libfive_tree_z(void);
/* libfive.h:211 */
libfive_tree libfive_tree_var(void);
/* libfive.h:216 */
bool libfive_tree_is_var(libfive_tree t);
/* libfive.h:221 */
libfive_tree libfive_tree_const(float f);
/* libfive.h:227 */
float libfive_tree_get_const(libfive_tree t, bool* success);
/* libfive.h:233 */
libfive_tree libfive_tree_nullary(int op);
/* libfive.h:239 */
libfive_tree libfive_tree_unary(int op, libfive_tree a);
/* libfive.h:245 */
libfive_tree libfive_tree_binary(int op, libfive_tree a, libfive_tree b);
/* libfive.h:255 */
const void* libfive_tree_id(libfive_tree t);

/* libfive.h:262: value at one point (free variables read as zero) */
float libfive_tree_eval_f(libfive_tree t, libfive_vec3 p);
/* libfive.h:269: interval enclosing the values over a box */
libfive_interval libfive_tree_eval_r(libfive_tree t, libfive_region3 r);
/* libfive.h:275: partial derivatives at one point */
libfive_vec3 libfive_tree_eval_d(libfive_tree t, libfive_vec3 p);

/* libfive.h:281 */
void libfive_tree_delete(libfive_tree ptr);
/* libfive.h:285: unsupported here (serialization is outside this library);
 * prints a message and returns false. */
bool libfive_tree_save(libfive_tree ptr, const char* filename);
/* libfive.h:288: unsupported here; prints a message and returns NULL. */
libfive_tree libfive_tree_load(const char* filename);
/* libfive.h:292 */
libfive_tree libfive_tree_remap(libfive_tree p,
        libfive_tree x, libfive_tree y, libfive_tree z);
/* libfive.h:298 */
libfive_tree libfive_tree_optimized(libfive_tree t);
/* libfive.h:306 */
char* libfive_tree_print(libfive_tree t);
/* libfive.h:311 */
void libfive_free_str(char* ptr);

/* libfive.h:326, 331, 340: 2D contouring is not part of this library;
 * these print a message and return NULL / do nothing. */
libfive_contours* libfive_tree_render_slice(libfive_tree tree,
                                            libfive_region2 R,
                                            float z, float res);
libfive_contours3* libfive_tree_render_slice3(libfive_tree tree,
                                              libfive_region2 R,
                                              float z, float res);
void libfive_tree_save_slice(libfive_tree tree, libfive_region2 R,
                             float z, float res, const char* f);

/* libfive.h:356: dual-contouring mesh on the GPU; NULL on failure */
libfive_mesh* libfive_tree_render_mesh(libfive_tree tree,
                                       libfive_region3 R, float res);
/* libfive.h:362: same as libfive_tree_render_mesh (the GPU path has no
 * worker threads to restrict) */
libfive_mesh* libfive_tree_render_mesh_st(libfive_tree tree,
                                          libfive_region3 R, float res);
/* libfive.h:369 */
libfive_mesh_coords* libfive_tree_render_mesh_coords(libfive_tree tree,
                                                     libfive_region3 R,
                                                     float res);
/* libfive.h:379: binary STL; false on failure */
bool libfive_tree_save_mesh(libfive_tree tree, libfive_region3 R,
                            float res, const char* f);
/* libfive.h:389 */
bool libfive_evaluator_save_mesh(libfive_evaluator evaluator,
                                 libfive_region3 R, const char* f);
/* libfive.h:404: trees[] is NULL-terminated */
bool libfive_tree_save_meshes(libfive_tree trees[], libfive_region3 R,
                              float res, float quality, const char* f);

/* libfive.h:414: not part of this library; prints a message, returns NULL */
libfive_pixels* libfive_tree_render_pixels(libfive_tree tree,
                                           libfive_region2 R,
                                           float z, float res);

/* libfive.h:420 */
libfive_evaluator libfive_tree_evaluator(libfive_tree tree, libfive_vars vars);
/* libfive.h:425 */
bool libfive_evaluator_update_vars(libfive_evaluator eval_tree,
                                   libfive_vars vars);
/* libfive.h:430 */
void libfive_evaluator_delete(libfive_evaluator ptr);

/* libfive.h:436-446 */
const char* libfive_git_version(void);
const char* libfive_git_revision(void);
const char* libfive_git_branch(void);

#ifdef __cplusplus
}
#endif
