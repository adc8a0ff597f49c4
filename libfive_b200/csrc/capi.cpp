// libfive.h and libfive_b200.h entry points.
//
// Tree construction follows libfive/src/libfive.cpp:75-190; evaluation and
// meshing run on the GPU through the device tapes in runtime.cpp and the
// kernels in eval_kernels.cu / dc_mesher.cu.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "libfive.h"
#include "libfive_b200.h"
#include "heightmap.hpp"
#include "contours.hpp"
#include "mesher.hpp"
#include "eval_api.hpp"
#include "runtime.hpp"
#include "tree.hpp"

using namespace lfb;

static const Node* N(libfive_tree t) { return reinterpret_cast<const Node*>(t); }
static libfive_tree H(const Node* n)
{
    return reinterpret_cast<libfive_tree>(const_cast<Node*>(n));
}

struct lfb_tape_ {
    std::shared_ptr<GpuTape> g;
};

struct libfive_evaluator_ {
    std::shared_ptr<GpuTape> g;
};

namespace lfb {
/// The device tape behind an lfb_tape handle (used by entry points that
/// live in other translation units).
GpuTape* tape_of(lfb_tape t) { return t ? t->g.get() : nullptr; }
}  // namespace lfb

extern "C" {

////////////////////////////////////////////////////////////////////////////////
// Deleters (libfive.cpp:31-71)

void libfive_contours_delete(libfive_contours* cs)
{
    if (!cs) return;
    for (unsigned i = 0; i < cs->count; ++i) delete[] cs->cs[i].pts;
    delete[] cs->cs;
    delete cs;
}

void libfive_contours3_delete(libfive_contours3* cs)
{
    if (!cs) return;
    for (unsigned i = 0; i < cs->count; ++i) delete[] cs->cs[i].pts;
    delete[] cs->cs;
    delete cs;
}

void libfive_mesh_delete(libfive_mesh* m)
{
    if (!m) return;
    host_free(m->verts);
    host_free(m->tris);
    delete m;
}

void libfive_mesh_coords_delete(libfive_mesh_coords* m)
{
    if (!m) return;
    host_free(m->verts);
    host_free(m->coord_indices);
    delete m;
}

void libfive_pixels_delete(libfive_pixels* m)
{
    if (!m) return;
    delete[] m->pixels;
    delete m;
}

void libfive_vars_delete(libfive_vars* vs)
{
    if (!vs) return;
    delete[] vs->vars;
    delete[] vs->values;
    delete vs;
}

int libfive_opcode_enum(const char* name)
{
    if (!name) return -1;
    const int o = op::from_scm_name(name);
    return (o == op::INVALID || o == op::LAST_OP) ? -1 : o;
}

int libfive_opcode_args(int o)
{
    return (o >= 0 && o < op::LAST_OP) ? op::arity(o) : -1;
}

////////////////////////////////////////////////////////////////////////////////
// Trees (libfive.cpp:75-190)

libfive_tree libfive_tree_x(void) { return H(Tree::X().release()); }
libfive_tree libfive_tree_y(void) { return H(Tree::Y().release()); }
libfive_tree libfive_tree_z(void) { return H(Tree::Z().release()); }
libfive_tree libfive_tree_var(void) { return H(Tree::var().release()); }
libfive_tree libfive_tree_const(float f) { return H(Tree::constant(f).release()); }

bool libfive_tree_is_var(libfive_tree t)
{
    return t && Tree(N(t)).op() == op::VAR_FREE;
}

float libfive_tree_get_const(libfive_tree t, bool* success)
{
    if (t && N(t)->kind == Kind::Constant) {
        if (success) *success = true;
        return N(t)->value;
    }
    if (success) *success = false;
    return 0;
}

static bool opcode_ok(int o, int args)
{
    return o >= 0 && o < op::LAST_OP && op::arity(o) == args;
}

libfive_tree libfive_tree_nullary(int o)
{
    return opcode_ok(o, 0) ? H(Tree::nullary(o).release()) : nullptr;
}

libfive_tree libfive_tree_unary(int o, libfive_tree a)
{
    return (opcode_ok(o, 1) && a) ? H(Tree::unary(o, Tree(N(a))).release())
                                  : nullptr;
}

libfive_tree libfive_tree_binary(int o, libfive_tree a, libfive_tree b)
{
    return (opcode_ok(o, 2) && a && b)
        ? H(Tree::binary(o, Tree(N(a)), Tree(N(b))).release())
        : nullptr;
}

const void* libfive_tree_id(libfive_tree t)
{
    return static_cast<const void*>(t);
}

void libfive_tree_delete(libfive_tree ptr)
{
    if (!ptr) return;
    invalidate_cached(N(ptr));
    Tree::reclaim(N(ptr));
}

bool libfive_tree_save(libfive_tree, const char*)
{
    std::fprintf(stderr, "libfive_tree_save: tree serialization is not "
                         "provided by libfive_b200\n");
    return false;
}

libfive_tree libfive_tree_load(const char*)
{
    std::fprintf(stderr, "libfive_tree_load: tree serialization is not "
                         "provided by libfive_b200\n");
    return nullptr;
}

libfive_tree libfive_tree_remap(libfive_tree p, libfive_tree x,
                                libfive_tree y, libfive_tree z)
{
    if (!p || !x || !y || !z) return nullptr;
    return H(Tree(N(p)).remap(Tree(N(x)), Tree(N(y)), Tree(N(z))).release());
}

libfive_tree libfive_tree_optimized(libfive_tree t)
{
    if (!t) return nullptr;
    return H(Tree(N(t)).optimized().release());
}

char* libfive_tree_print(libfive_tree t)
{
    std::stringstream ss;
    if (t) Tree(N(t)).print(ss);
    const std::string s = ss.str();
    char* out = static_cast<char*>(std::malloc(s.size() + 1));
    std::memcpy(out, s.c_str(), s.size() + 1);
    return out;
}

void libfive_free_str(char* ptr) { std::free(ptr); }

////////////////////////////////////////////////////////////////////////////////
// Single-point evaluation (libfive.cpp:195-214), served by cached device tapes

float libfive_tree_eval_f(libfive_tree t, libfive_vec3 p)
{
    if (!t) return NAN;
    auto g = cached_tape(N(t));
    float out = NAN;
    if (!g || eval_values_host(*g, 1, &p.x, &p.y, &p.z, &out) != 0) {
        std::string msg;
        last_error(&msg);
        std::fprintf(stderr, "libfive_tree_eval_f: %s\n", msg.c_str());
        return NAN;
    }
    return out;
}

libfive_interval libfive_tree_eval_r(libfive_tree t, libfive_region3 r)
{
    libfive_interval out{NAN, NAN};
    if (!t) return out;
    auto g = cached_tape(N(t));
    uint8_t nan_flag = 0;
    if (!g || eval_intervals_host(*g, 1, &r.X.lower, &r.X.upper, &r.Y.lower,
                                  &r.Y.upper, &r.Z.lower, &r.Z.upper,
                                  &out.lower, &out.upper, &nan_flag) != 0) {
        std::string msg;
        last_error(&msg);
        std::fprintf(stderr, "libfive_tree_eval_r: %s\n", msg.c_str());
        return {NAN, NAN};
    }
    return out;
}

libfive_vec3 libfive_tree_eval_d(libfive_tree t, libfive_vec3 p)
{
    libfive_vec3 out{NAN, NAN, NAN};
    if (!t) return out;
    auto g = cached_tape(N(t));
    float v = 0;
    if (!g || eval_derivs_host(*g, 1, &p.x, &p.y, &p.z, &v, &out.x, &out.y,
                               &out.z) != 0) {
        std::string msg;
        last_error(&msg);
        std::fprintf(stderr, "libfive_tree_eval_d: %s\n", msg.c_str());
        return {NAN, NAN, NAN};
    }
    return out;
}

////////////////////////////////////////////////////////////////////////////////
// Outside the evaluate-and-mesh path

static double min_feature_of(float res);

/// Contours::render for the slice calls (libfive.cpp:233-304): the GPU
/// contourer with BRepSettings' max_err (1e-8) and min_feature = 1 / res;
/// false, with the message printed, on failure.
static bool render_slice(const std::shared_ptr<GpuTape>& g, libfive_region2 R, float z,
                         double min_feature, double max_err, ContoursOut& cs, const char* who)
{
    const double lo[2] = {R.X.lower, R.Y.lower}, hi[2] = {R.X.upper, R.Y.upper};
    if (!g || render_contours(*g, lo, hi, z, min_feature, max_err, cs) != 0) {
        std::string msg;
        last_error(&msg);
        std::fprintf(stderr, "%s: %s\n", who, msg.c_str());
        return false;
    }
    return true;
}

/// The contours as the reference's C structs (arrays from new[], freed by
/// libfive_contours_delete / libfive_contours3_delete).
static libfive_contours* contours_struct(const ContoursOut& cs)
{
    auto out = new libfive_contours;
    out->count = static_cast<uint32_t>(cs.counts.size());
    out->cs = new libfive_contour[out->count];
    size_t k = 0;
    for (uint32_t i = 0; i < out->count; ++i) {
        out->cs[i].count = cs.counts[i];
        out->cs[i].pts = new libfive_vec2[cs.counts[i]];
        for (uint32_t j = 0; j < cs.counts[i]; ++j, ++k) {
            out->cs[i].pts[j] = {cs.pts[2 * k], cs.pts[2 * k + 1]};
        }
    }
    return out;
}

static libfive_contours3* contours3_struct(const ContoursOut& cs, float z)
{
    auto out = new libfive_contours3;
    out->count = static_cast<uint32_t>(cs.counts.size());
    out->cs = new libfive_contour3[out->count];
    size_t k = 0;
    for (uint32_t i = 0; i < out->count; ++i) {
        out->cs[i].count = cs.counts[i];
        out->cs[i].pts = new libfive_vec3[cs.counts[i]];
        for (uint32_t j = 0; j < cs.counts[i]; ++j, ++k) {
            out->cs[i].pts[j] = {cs.pts[2 * k], cs.pts[2 * k + 1], z};
        }
    }
    return out;
}

libfive_contours* libfive_tree_render_slice(libfive_tree tree, libfive_region2 R,
                                            float z, float res)
{
    if (!tree) return nullptr;
    ContoursOut cs;
    if (!render_slice(cached_tape(N(tree)), R, z, min_feature_of(res), 1e-8, cs,
                      "libfive_tree_render_slice")) {
        return nullptr;
    }
    return contours_struct(cs);
}

libfive_contours3* libfive_tree_render_slice3(libfive_tree tree, libfive_region2 R,
                                              float z, float res)
{
    if (!tree) return nullptr;
    ContoursOut cs;
    if (!render_slice(cached_tape(N(tree)), R, z, min_feature_of(res), 1e-8, cs,
                      "libfive_tree_render_slice3")) {
        return nullptr;
    }
    // each 2D point gets z as its third coordinate (libfive.cpp:289-293)
    return contours3_struct(cs, z);
}

void libfive_tree_save_slice(libfive_tree tree, libfive_region2 R, float z, float res,
                             const char* f)
{
    if (!tree || !f) return;
    ContoursOut cs;
    if (!render_slice(cached_tape(N(tree)), R, z, min_feature_of(res), 1e-8, cs,
                      "libfive_tree_save_slice")) {
        return;
    }
    const double lo[2] = {R.X.lower, R.Y.lower}, hi[2] = {R.X.upper, R.Y.upper};
    save_svg(f, cs, lo, hi);
}

libfive_contours* lfb_render_slice(lfb_tape t, libfive_region2 R, float z,
                                   double min_feature, double max_err)
{
    auto g = tape_of(t);
    ContoursOut cs;
    if (!g) {
        set_error(LFB_E_INVALID, "null tape");
        return nullptr;
    }
    const double lo[2] = {R.X.lower, R.Y.lower}, hi[2] = {R.X.upper, R.Y.upper};
    if (render_contours(*g, lo, hi, z, min_feature, max_err, cs) != 0) return nullptr;
    return contours_struct(cs);
}

libfive_pixels* libfive_tree_render_pixels(libfive_tree tree, libfive_region2 R,
                                           float z, float res)
{
    // libfive.cpp:442-465: a one-sample-deep Voxels region at height z, the
    // height map rendered, and a pixel set wherever the depth is finite.
    clear_error();
    if (!tree) return nullptr;
    const float lo[3] = {R.X.lower, R.Y.lower, z};
    const float hi[3] = {R.X.upper, R.Y.upper, z};
    const float r3[3] = {res, res, res};
    const VoxelGrid V = make_voxel_grid(lo, hi, r3);
    auto g = cached_tape(N(tree));
    const size_t w = V.pts[0].size(), h = V.pts[1].size();
    std::vector<float> depth(w * h);
    if (!g || render_heightmap(*g, V, depth.data(), nullptr) != 0) {
        std::string msg;
        last_error(&msg);
        std::fprintf(stderr, "libfive_tree_render_pixels: %s\n", msg.c_str());
        return nullptr;
    }
    auto out = new libfive_pixels;
    out->width = static_cast<uint32_t>(w);
    out->height = static_cast<uint32_t>(h);
    out->pixels = new bool[w * h];
    for (size_t i = 0; i < w * h; ++i) out->pixels[i] = !std::isinf(depth[i]);
    return out;
}

////////////////////////////////////////////////////////////////////////////////
// Meshing (libfive.cpp:306-440)

/// BRepSettings::min_feature as the reference's C API sets it: `1/res`
/// divides in float (libfive.cpp:301), and that float is what is widened.
static double min_feature_of(float res)
{
    return static_cast<double>(1 / res);
}

/// Renders into `mesh` (whose format says what comes back); false with the
/// message printed on failure, as the reference's callers see a null mesh.
static bool render_into(const std::shared_ptr<GpuTape>& g, libfive_region3 R,
                        double min_feature, double max_err, const char* who,
                        MeshOut& mesh)
{
    if (!g || render_dc_mesh(*g, R, min_feature, max_err, mesh, nullptr) != 0) {
        std::string msg;
        last_error(&msg);
        std::fprintf(stderr, "%s: %s\n", who, msg.c_str());
        return false;
    }
    return true;
}

static libfive_mesh* render_with(const std::shared_ptr<GpuTape>& g,
                                 libfive_region3 R, double min_feature,
                                 double max_err, const char* who)
{
    MeshOut mesh;
    if (!render_into(g, R, min_feature, max_err, who, mesh)) return nullptr;
    return mesh.release();
}

/// Mesh::saveSTL of a freshly rendered mesh, the records packed on the
/// device and streamed to the file (no file is created when the render
/// fails, as in the reference, which renders before it opens the file).
static bool save_with(const std::shared_ptr<GpuTape>& g, libfive_region3 R,
                      double min_feature, double max_err, const char* path,
                      const char* who)
{
    if (!path) return false;
    MeshOut mesh;
    mesh.format = MeshFormat::Stl;
    mesh.stl_path = path;
    return render_into(g, R, min_feature, max_err, who, mesh);
}

libfive_mesh* libfive_tree_render_mesh(libfive_tree tree, libfive_region3 R,
                                       float res)
{
    if (!tree) return nullptr;
    return render_with(cached_tape(N(tree)), R, min_feature_of(res), 1e-8,
                       "libfive_tree_render_mesh");
}

libfive_mesh* libfive_tree_render_mesh_st(libfive_tree tree,
                                          libfive_region3 R, float res)
{
    if (!tree) return nullptr;
    return render_with(cached_tape(N(tree)), R, min_feature_of(res), 1e-8,
                       "libfive_tree_render_mesh_st");
}

libfive_mesh_coords* libfive_tree_render_mesh_coords(libfive_tree tree,
                                                     libfive_region3 R,
                                                     float res)
{
    if (!tree) return nullptr;
    // the index list (a, b, c, -1 per triangle) is packed on the device
    MeshOut mesh;
    mesh.format = MeshFormat::Coords;
    if (!render_into(cached_tape(N(tree)), R, min_feature_of(res), 1e-8,
                     "libfive_tree_render_mesh_coords", mesh)) {
        return nullptr;
    }
    auto out = new libfive_mesh_coords;
    out->vert_count = mesh.vert_count;
    out->verts = mesh.verts;
    out->coord_index_count = 4 * mesh.tri_count;
    out->coord_indices = mesh.coords;
    mesh.verts = nullptr;
    mesh.coords = nullptr;
    return out;
}

bool libfive_tree_save_mesh(libfive_tree tree, libfive_region3 R, float res,
                            const char* f)
{
    if (!tree) return false;
    return save_with(cached_tape(N(tree)), R, min_feature_of(res), 1e-8, f,
                     "libfive_tree_save_mesh");
}

bool libfive_tree_save_meshes(libfive_tree trees[], libfive_region3 R,
                              float res, float quality, const char* f)
{
    // The reference renders the trees one after another (libfive.cpp:419-440);
    // here they render concurrently, each on its own stream.
    std::vector<std::shared_ptr<GpuTape>> tapes;
    for (unsigned i = 0; trees && trees[i] != nullptr; ++i) {
        auto g = cached_tape(N(trees[i]));
        if (!g) {
            std::string msg;
            last_error(&msg);
            std::fprintf(stderr, "libfive_tree_save_meshes: %s\n", msg.c_str());
            return false;
        }
        tapes.push_back(std::move(g));
    }
    std::vector<MeshJob> jobs(tapes.size());
    for (size_t i = 0; i < tapes.size(); ++i) {
        jobs[i].g = tapes[i].get();
        jobs[i].R = R;
        jobs[i].min_feature = min_feature_of(res);
        jobs[i].max_err = std::pow(10.0, -quality);
    }
    if (render_dc_meshes(jobs.data(), jobs.size(), 4) != 0) {
        std::string msg;
        last_error(&msg);
        std::fprintf(stderr, "libfive_tree_save_meshes: %s\n", msg.c_str());
        return false;
    }
    std::vector<libfive_mesh*> ms;
    for (auto& j : jobs) ms.push_back(j.out.release());
    const bool ok = save_stl(f, ms);
    for (auto m : ms) libfive_mesh_delete(m);
    return ok;
}

bool libfive_evaluator_save_mesh(libfive_evaluator ev, libfive_region3 R,
                                 const char* f)
{
    if (!ev) return false;
    // BRepSettings defaults (settings.hpp:34-43): min_feature 0.1, max_err 1e-8
    return save_with(ev->g, R, 0.1, 1e-8, f, "libfive_evaluator_save_mesh");
}

////////////////////////////////////////////////////////////////////////////////
// Evaluators (libfive.cpp:467-502)

libfive_evaluator libfive_tree_evaluator(libfive_tree tree, libfive_vars vars)
{
    if (!tree) return nullptr;
    auto g = make_tape(Tree(N(tree)));
    if (!g) return nullptr;
    g->set_vars(vars.vars, vars.values, vars.size);
    if (!g->upload_cpool()) return nullptr;
    auto e = new libfive_evaluator_;
    e->g = g;
    return e;
}

bool libfive_evaluator_update_vars(libfive_evaluator ev, libfive_vars vars)
{
    if (!ev) return false;
    const bool changed = ev->g->set_vars(vars.vars, vars.values, vars.size);
    ev->g->upload_cpool();
    return changed;
}

void libfive_evaluator_delete(libfive_evaluator ptr)
{
    delete ptr;
}

const char* libfive_git_version(void) { return "libfive_b200"; }
const char* libfive_git_revision(void) { return "b200"; }
const char* libfive_git_branch(void) { return "main"; }

////////////////////////////////////////////////////////////////////////////////
// libfive_b200.h

int lfb_last_error(char* buf, uint32_t len)
{
    std::string msg;
    const int code = last_error(&msg);
    if (buf && len) {
        std::snprintf(buf, len, "%s", msg.c_str());
    }
    return code;
}

lfb_tape lfb_tape_new(libfive_tree t, libfive_vars vars)
{
    clear_error();
    if (!t) {
        set_error(LFB_E_INVALID, "null tree");
        return nullptr;
    }
    auto g = make_tape(Tree(N(t)));
    if (!g) return nullptr;
    if (vars.size) {
        g->set_vars(vars.vars, vars.values, vars.size);
        if (!g->upload_cpool()) return nullptr;
    }
    auto out = new lfb_tape_;
    out->g = g;
    return out;
}

void lfb_tape_delete(lfb_tape t) { delete t; }

int lfb_tape_set_vars(lfb_tape t, libfive_vars vars)
{
    if (!t) return set_error(LFB_E_INVALID, "null tape");
    if (!t->g->on_current_device()) return LFB_E_INVALID;
    std::lock_guard<std::mutex> lock(t->g->mu);
    // variables that fit steps changed on the device keep their new values
    if (!t->g->pull_vars()) return LFB_E_CUDA;
    const bool changed = t->g->set_vars(vars.vars, vars.values, vars.size);
    if (!t->g->upload_cpool()) return LFB_E_CUDA;
    return changed ? 1 : 0;
}

int lfb_debug_set(const char* key, int64_t value)
{
    clear_error();
    if (!key) return set_error(LFB_E_INVALID, "null key");
    const std::string k(key);
    if (k == "fail_alloc_after") {
        debug_hooks().fail_alloc_after = value > 0 ? value : 0;
    } else if (k == "small_capacity") {
        debug_hooks().small_capacity = value ? 1 : 0;
    } else {
        return set_error(LFB_E_INVALID, "unknown debug key: " + k);
    }
    return 0;
}

int lfb_tape_set_vars_device(lfb_tape t, const float* values, uint32_t n, void* stream)
{
    clear_error();
    if (!t || !values) return set_error(LFB_E_INVALID, "null argument");
    if (!t->g->on_current_device()) return LFB_E_INVALID;
    GpuTape& g = *t->g;
    std::lock_guard<std::mutex> lock(g.mu);
    if (n != g.reg.n_vars) {
        return set_error(LFB_E_INVALID, "expected " + std::to_string(g.reg.n_vars) +
                                            " variable values, got " + std::to_string(n));
    }
    if (n == 0) return 0;
    if (!cuda_ok(cudaMemcpyAsync(g.d_cpool + g.reg.n_const, values, n * sizeof(float),
                                 cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)),
                 "variable copy")) {
        return LFB_E_CUDA;
    }
    g.vars_on_device = true;
    return 0;
}

int lfb_tape_get_vars(lfb_tape t, float* values, uint32_t len)
{
    clear_error();
    if (!t || (!values && len)) return set_error(LFB_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lock(t->g->mu);
    if (!t->g->pull_vars()) return LFB_E_CUDA;
    const auto& r = t->g->reg;
    for (uint32_t i = 0; i < r.n_vars && i < len; ++i) {
        values[i] = r.cpool[r.n_const + i];
    }
    return 0;
}

int lfb_fit_adam_step(const lfb_tape* tapes, uint32_t n_shapes,
                      const uint64_t* point_offsets, const float* x,
                      const float* y, const float* z,
                      const uint64_t* var_offsets, float* m, float* v,
                      lfb_adam_settings adam, uint32_t step, float* losses,
                      void* stream)
{
    clear_error();
    if (!tapes) return set_error(LFB_E_INVALID, "null tape list");
    try {
        std::vector<GpuTape*> gs(n_shapes);
        for (uint32_t j = 0; j < n_shapes; ++j) {
            if (!tapes[j]) return set_error(LFB_E_INVALID, "null tape");
            if (!tapes[j]->g->on_current_device()) return LFB_E_INVALID;
            gs[j] = tapes[j]->g.get();
        }
        return fit_adam_step(gs.data(), n_shapes, point_offsets, x, y, z, var_offsets, m, v,
                             adam, step, losses, static_cast<cudaStream_t>(stream));
    } catch (const std::exception& e) {
        // nothing may unwind through the C ABI
        return set_error(LFB_E_INVALID, std::string("lfb_fit_adam_step: ") + e.what());
    }
}

int lfb_tape_compiled(lfb_tape t)
{
    if (!t) return 0;
    std::lock_guard<std::mutex> lock(t->g->mu);
    return t->g->jit[0].state == 1 ? 1 : 0;
}

int lfb_tape_info(lfb_tape t, uint32_t counts[6])
{
    if (!t || !counts) return set_error(LFB_E_INVALID, "null argument");
    const auto& r = t->g->reg;
    counts[0] = static_cast<uint32_t>(r.clauses.size());
    counts[1] = r.n_regs;
    counts[2] = r.n_const;
    counts[3] = r.n_vars;
    counts[4] = r.n_choices;
    counts[5] = t->g->slot.num_clauses;
    return 0;
}

int lfb_tape_var_ids(lfb_tape t, const void** ids, uint32_t len)
{
    if (!t) return set_error(LFB_E_INVALID, "null tape");
    const auto& r = t->g->reg;
    for (uint32_t i = 0; i < r.n_vars && i < len; ++i) {
        ids[i] = r.var_nodes[i];
    }
    return 0;
}

int lfb_eval_values(lfb_tape t, uint64_t n, const float* x, const float* y,
                    const float* z, float* out, void* stream, uint32_t flags)
{
    clear_error();
    if (!t) return set_error(LFB_E_INVALID, "null tape");
    if (!t->g->on_current_device()) return LFB_E_INVALID;
    if (flags & LFB_DEVICE_PTRS) {
        return eval_values_device(*t->g, n, x, y, z, out,
                                  static_cast<cudaStream_t>(stream));
    }
    return eval_values_host(*t->g, n, x, y, z, out);
}

int lfb_eval_derivs(lfb_tape t, uint64_t n, const float* x, const float* y,
                    const float* z, float* v, float* dx, float* dy, float* dz,
                    void* stream, uint32_t flags)
{
    clear_error();
    if (!t) return set_error(LFB_E_INVALID, "null tape");
    if (!t->g->on_current_device()) return LFB_E_INVALID;
    if (flags & LFB_DEVICE_PTRS) {
        return eval_derivs_device(*t->g, n, x, y, z, v, dx, dy, dz,
                                  static_cast<cudaStream_t>(stream));
    }
    return eval_derivs_host(*t->g, n, x, y, z, v, dx, dy, dz);
}

int lfb_eval_features(lfb_tape t, uint64_t n, const float* x, const float* y,
                      const float* z, uint8_t* inside, float* feats, uint32_t max_feats,
                      uint32_t* n_feats)
{
    clear_error();
    if (!t) return set_error(LFB_E_INVALID, "null tape");
    if (!t->g->on_current_device()) return LFB_E_INVALID;
    return eval_features_host(*t->g, n, x, y, z, inside, feats, max_feats, n_feats);
}

int lfb_eval_intervals(lfb_tape t, uint64_t n, const float* xlo,
                       const float* xhi, const float* ylo, const float* yhi,
                       const float* zlo, const float* zhi, float* out_lo,
                       float* out_hi, uint8_t* out_nan, void* stream,
                       uint32_t flags)
{
    clear_error();
    if (!t) return set_error(LFB_E_INVALID, "null tape");
    if (!t->g->on_current_device()) return LFB_E_INVALID;
    if (flags & LFB_DEVICE_PTRS) {
        return eval_intervals_device(*t->g, n, xlo, xhi, ylo, yhi, zlo, zhi,
                                     out_lo, out_hi, out_nan,
                                     static_cast<cudaStream_t>(stream));
    }
    return eval_intervals_host(*t->g, n, xlo, xhi, ylo, yhi, zlo, zhi,
                               out_lo, out_hi, out_nan);
}

int lfb_eval_jacobian(lfb_tape t, uint64_t n, const float* x, const float* y,
                      const float* z, float* out, void* stream, uint32_t flags)
{
    clear_error();
    if (!t) return set_error(LFB_E_INVALID, "null tape");
    if (!t->g->on_current_device()) return LFB_E_INVALID;
    return eval_jacobian(*t->g, n, x, y, z, out,
                         static_cast<cudaStream_t>(stream),
                         (flags & LFB_DEVICE_PTRS) != 0);
}

int lfb_eval_grad(lfb_tape t, uint64_t n, const float* x, const float* y,
                  const float* z, const float* seed, float* f, float* gx,
                  float* gy, float* gz, float* gvars, void* stream,
                  uint32_t flags)
{
    clear_error();
    if (!t) return set_error(LFB_E_INVALID, "null tape");
    if (!t->g->on_current_device()) return LFB_E_INVALID;
    return eval_grad(*t->g, n, x, y, z, seed, f, gx, gy, gz, gvars,
                     static_cast<cudaStream_t>(stream),
                     (flags & LFB_DEVICE_PTRS) != 0);
}

int lfb_eval_loss_grad(lfb_tape t, uint64_t n, const float* x, const float* y,
                       const float* z, float* f, float* gx, float* gy, float* gz,
                       float* gvars, float* loss, void* stream, uint32_t flags)
{
    clear_error();
    if (!t) return set_error(LFB_E_INVALID, "null tape");
    if (!(flags & LFB_DEVICE_PTRS)) {
        return set_error(LFB_E_INVALID, "lfb_eval_loss_grad takes device arrays (LFB_DEVICE_PTRS)");
    }
    if (!t->g->on_current_device()) return LFB_E_INVALID;
    return eval_loss_grad(*t->g, n, x, y, z, f, gx, gy, gz, gvars, loss,
                          static_cast<cudaStream_t>(stream));
}

libfive_mesh* lfb_render_mesh(lfb_tape t, libfive_region3 R,
                              lfb_mesh_settings s, lfb_mesh_stats* stats)
{
    clear_error();
    if (!t) {
        set_error(LFB_E_INVALID, "null tape");
        return nullptr;
    }
    if (!t->g->on_current_device()) return nullptr;
    MeshOut mesh;
    if (render_dc_mesh(*t->g, R, s.min_feature, s.max_err, mesh, stats, s.cancel) != 0) {
        return nullptr;
    }
    return mesh.release();
}

int lfb_render_heightmap(lfb_tape t, const float lower[3], const float upper[3],
                         const float res[3], uint32_t dims[3], float* depth, uint32_t* norm)
{
    clear_error();
    if (!t || !lower || !upper || !res || !dims) {
        return set_error(LFB_E_INVALID, "null argument");
    }
    const VoxelGrid V = make_voxel_grid(lower, upper, res);
    for (int a = 0; a < 3; ++a) dims[a] = static_cast<uint32_t>(V.pts[a].size());
    if (!depth) return 0;
    if (!t->g->on_current_device()) return LFB_E_INVALID;
    return render_heightmap(*t->g, V, depth, norm);
}

int lfb_render_meshes(const lfb_tape* tapes, uint32_t n, const libfive_region3* regions,
                      const lfb_mesh_settings* settings, uint32_t workers,
                      libfive_mesh** meshes, lfb_mesh_stats* stats)
{
    clear_error();
    if (n && (!tapes || !regions || !settings || !meshes)) {
        return set_error(LFB_E_INVALID, "null argument");
    }
    for (uint32_t i = 0; i < n; ++i) {
        meshes[i] = nullptr;
        if (!tapes[i]) return set_error(LFB_E_INVALID, "null tape");
        if (!tapes[i]->g->on_current_device()) return LFB_E_INVALID;
    }
    std::vector<MeshJob> jobs(n);
    for (uint32_t i = 0; i < n; ++i) {
        jobs[i].g = tapes[i]->g.get();
        jobs[i].R = regions[i];
        jobs[i].min_feature = settings[i].min_feature;
        jobs[i].max_err = settings[i].max_err;
        jobs[i].cancel = settings[i].cancel;
        jobs[i].want_stats = stats != nullptr;
    }
    const int rc = render_dc_meshes(jobs.data(), n, workers ? workers : 4);
    for (uint32_t i = 0; i < n; ++i) {
        if (jobs[i].rc == 0) meshes[i] = jobs[i].out.release();
        if (stats) stats[i] = jobs[i].stats;
    }
    return rc;
}

uint64_t lfb_kernel_launches(void) { return launches(); }

int lfb_tree_slot_tape(libfive_tree t, uint32_t counts[8], int32_t* clauses,
                       uint32_t* const_slots, float* const_values,
                       uint32_t* var_slots, const void** var_ids)
{
    clear_error();
    if (!t || !counts) return set_error(LFB_E_INVALID, "null argument");
    SlotTape st;
    std::string err;
    if (!build_slot_tape(Tree(N(t)), st, &err)) {
        return set_error(LFB_E_UNSUPPORTED, err);
    }
    counts[0] = st.num_clauses;
    counts[1] = static_cast<uint32_t>(st.clauses.size());
    counts[2] = static_cast<uint32_t>(st.constants.size());
    counts[3] = static_cast<uint32_t>(st.vars.size());
    counts[4] = st.X;
    counts[5] = st.Y;
    counts[6] = st.Z;
    counts[7] = st.root;
    if (clauses) {
        for (size_t i = 0; i < st.clauses.size(); ++i) {
            clauses[4 * i + 0] = st.clauses[i].op;
            clauses[4 * i + 1] = static_cast<int32_t>(st.clauses[i].id);
            clauses[4 * i + 2] = static_cast<int32_t>(st.clauses[i].a);
            clauses[4 * i + 3] = static_cast<int32_t>(st.clauses[i].b);
        }
    }
    for (size_t i = 0; i < st.constants.size(); ++i) {
        if (const_slots) const_slots[i] = st.constants[i].first;
        if (const_values) const_values[i] = st.constants[i].second;
    }
    for (size_t i = 0; i < st.vars.size(); ++i) {
        if (var_slots) var_slots[i] = st.vars[i].first;
        if (var_ids) var_ids[i] = st.vars[i].second;
    }
    return 0;
}

}  // extern "C"
