/*
 *  Additional entry points of the B200 implementation (additive: nothing in
 *  libfive.h changes).  They expose what the reference keeps behind C++
 *  classes — reusable evaluators, batched evaluation of many points, the
 *  gradient with respect to free variables — as plain C calls over flat
 *  float arrays, so that the GPU can be fed large batches.
 *
 *  Pointer arguments are host pointers unless LFB_DEVICE_PTRS is set in
 *  `flags`, in which case they are CUDA device pointers and `stream` (a
 *  cudaStream_t, or NULL for the legacy default stream) orders the work.
 *  Every call returns 0 on success or a negative LFB_E* code; the message of
 *  the last failure on the calling thread is read with lfb_last_error.
 */
#pragma once
#include "libfive.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
    LFB_OK = 0,
    LFB_E_INVALID = -1,      /* bad argument / invalid tree */
    LFB_E_UNSUPPORTED = -2,  /* opcode or feature the device path lacks */
    LFB_E_CUDA = -3,         /* CUDA error or no CUDA device */
    LFB_E_CAPACITY = -4,     /* a device buffer was too small (retried
                                internally; reported only if retries fail) */
    LFB_E_CANCELLED = -5,
};

#define LFB_DEVICE_PTRS 1u

/* Message and code of the last failure on this thread. */
int lfb_last_error(char* buf, uint32_t len);

/*  A device tape: the tree flattened once (Deck, deck.cpp:19-94) and kept
 *  resident on the GPU, with values for its free variables (unlisted
 *  variables read as zero).  Replaces constructing a libfive::Evaluator
 *  (libfive/include/libfive/eval/evaluator.hpp:16-50). */
typedef struct lfb_tape_* lfb_tape;
lfb_tape lfb_tape_new(libfive_tree t, libfive_vars vars);
void lfb_tape_delete(lfb_tape t);
/* Evaluator::updateVars (evaluator.hpp:35-44); returns 1 if any changed. */
int lfb_tape_set_vars(lfb_tape t, libfive_vars vars);
/* counts[0..5] = clauses, registers, constants, free variables, min/max
 * clauses, reference slot count (Deck::num_clauses). */
int lfb_tape_info(lfb_tape t, uint32_t counts[6]);
/* 1 when the tape's values (lfb_eval_values and the callers built on it)
 * run through the kernel compiled for this tape at its first evaluation
 * (straight-line code for tapes of at most 4096 clauses, segments of a few
 * hundred clauses up to 65536; NVRTC present, LFB_JIT not set to 0); 0 when
 * they run through the interpreter or nothing was evaluated yet.  Both give
 * identical values. */
int lfb_tape_compiled(lfb_tape t);
/* Variable order used by the gradient calls: var_ids[i] receives the
 * libfive_tree_id of variable i (ascending reference slot order, as
 * JacobianEvaluator::gradient, eval_jacobian.cpp:77-90). */
int lfb_tape_var_ids(lfb_tape t, const void** var_ids, uint32_t len);

/*  No counterpart in the reference.  Value and d/dx, d/dy, d/dz of at most
 *  262144 host points per call (larger n is rejected with LFB_E_INVALID),
 *  staged through a fixed 7 MiB device array that is part of the library,
 *  so the call allocates no device memory: for callers that cannot call
 *  cudaMalloc while they run.  All arguments are host pointers (dx, dy, dz
 *  may be NULL).  The first call on each device looks the array up and
 *  should come before any stream capture; calls must not overlap on the
 *  GPU, since they share the array. */
int lfb_eval_derivs_static(lfb_tape t, uint64_t n, const float* x,
                           const float* y, const float* z, float* v,
                           float* dx, float* dy, float* dz);

/* ArrayEvaluator::values (eval_array.cpp:106-118) over n points. */
int lfb_eval_values(lfb_tape t, uint64_t n, const float* x, const float* y,
                    const float* z, float* out, void* stream, uint32_t flags);

/* DerivArrayEvaluator::derivs (eval_deriv_array.cpp:101-117): value and
 * d/dx, d/dy, d/dz (any of dx/dy/dz may be NULL). */
int lfb_eval_derivs(lfb_tape t, uint64_t n, const float* x, const float* y,
                    const float* z, float* v, float* dx, float* dy, float* dz,
                    void* stream, uint32_t flags);

/* FeatureEvaluator at n host points (the path the mesher takes at samples
 * whose value is exactly zero): inside[i] = isInside (eval_feature.cpp:
 * 56-116); when n_feats is not NULL, n_feats[i] = the number of distinct
 * feature gradients at point i (features, eval_feature.cpp:125-169) and, when
 * feats is not NULL, feats[(i * max_feats + k) * 3 + 0..2] the first
 * max_feats of them.  LFB_E_CAPACITY when a feature list outgrows the
 * device evaluator's fixed capacity (15 features of 4 epsilons per clause). */
int lfb_eval_features(lfb_tape t, uint64_t n, const float* x, const float* y,
                      const float* z, uint8_t* inside, float* feats,
                      uint32_t max_feats, uint32_t* n_feats);

/* IntervalEvaluator::eval (eval_interval.cpp:68-93) over n boxes; out_nan
 * receives the "may be NaN" flag (0/1). */
int lfb_eval_intervals(lfb_tape t, uint64_t n,
                       const float* xlo, const float* xhi,
                       const float* ylo, const float* yhi,
                       const float* zlo, const float* zhi,
                       float* out_lo, float* out_hi, uint8_t* out_nan,
                       void* stream, uint32_t flags);

/* JacobianEvaluator::gradient (eval_jacobian.cpp:49-115) for n points:
 * out[i * n_vars + k] = df(p_i)/dvar_k (CONST_VAR blocks the gradient). */
int lfb_eval_jacobian(lfb_tape t, uint64_t n, const float* x,
                      const float* y, const float* z, float* out,
                      void* stream, uint32_t flags);

/*  Reverse-mode gradient (new; the reference has forward mode only).
 *  For each point i: f[i] = f(p_i); with seed s_i (1 when seed is NULL):
 *    gx/gy/gz[i] = s_i * df/dp_i            (any of them may be NULL)
 *    gvars[k]   += sum_i s_i * df(p_i)/dvar_k   (if gvars is not NULL;
 *                  accumulated, so zero it first)
 *  Subgradient choices at min / max / abs match the forward rules of
 *  DerivArrayEvaluator (eval_deriv_array.cpp:139-146, 219-222). */
int lfb_eval_grad(lfb_tape t, uint64_t n, const float* x, const float* y,
                  const float* z, const float* seed, float* f, float* gx,
                  float* gy, float* gz, float* gvars, void* stream,
                  uint32_t flags);

/*  Sets all of the tape's free variables (lfb_tape_var_ids order) from n
 *  floats in DEVICE memory, ordered on `stream` (NULL: legacy default
 *  stream); no host synchronisation.  n must equal the variable count.
 *  Later evaluations on that stream, meshes and lfb_tape_get_vars see the
 *  new values.  Device-side counterpart of lfb_tape_set_vars
 *  (Evaluator::updateVars, evaluator.hpp:35-44). */
int lfb_tape_set_vars_device(lfb_tape t, const float* values, uint32_t n,
                             void* stream);

/*  Loss and gradient in one call (new; the reference has no optimiser):
 *  loss = mean_i f(p_i)^2 over n points, f[i] = f(p_i), and its gradients
 *    gx/gy/gz[i] = 2 f(p_i) / n * df/dp_i     (any may be NULL)
 *    gvars[k]   += sum_i 2 f(p_i) / n * df(p_i)/dvar_k   (NULL to skip)
 *  *loss (NULL to skip) receives the loss as a float.  One forward pass
 *  serves both f and the gradient (lfb_eval_grad with seed 2 f / n, without
 *  a separate evaluation of f).  All arrays are device arrays: flags must
 *  hold LFB_DEVICE_PTRS; work is ordered on `stream`. */
int lfb_eval_loss_grad(lfb_tape t, uint64_t n, const float* x, const float* y,
                       const float* z, float* f, float* gx, float* gy, float* gz,
                       float* gvars, float* loss, void* stream, uint32_t flags);

/*  Current values of the tape's free variables (lfb_tape_var_ids order) in
 *  a host array of len floats; after lfb_fit_adam_step this waits for the
 *  device and reads the values it wrote.  Counterpart of reading
 *  Evaluator's variable map (evaluator.hpp:35-44). */
int lfb_tape_get_vars(lfb_tape t, float* values, uint32_t len);

/*  Adam hyper-parameters (Kingma & Ba, 2015). */
typedef struct lfb_adam_settings {
    float lr;     /* step size */
    float beta1;  /* first-moment decay, e.g. 0.9 */
    float beta2;  /* second-moment decay, e.g. 0.999 */
    float eps;    /* added to the root of the second moment, e.g. 1e-8 */
} lfb_adam_settings;

/*  Batched least-squares fitting (new; the reference has no optimiser).
 *  One Adam step on every shape j of loss_j = mean_i f_j(p_i)^2 over its
 *  points p_i = (x, y, z)[point_offsets[j] .. point_offsets[j + 1]), with
 *  respect to the free variables of tapes[j]:
 *    g   = (2 / n_j) * sum_i f_j(p_i) df_j(p_i)/dvar   (reverse mode, as
 *          lfb_eval_grad with seed f)
 *    m   = m + (1 - beta1) (g - m);   v = beta2 v + (1 - beta2) g g
 *    var = var - lr / (1 - beta1^step) * m / (sqrt(v) / sqrt(1 - beta2^step) + eps)
 *  The new values are written into the tapes' variables on the device
 *  (later evaluations and meshes use them; lfb_tape_get_vars reads them).
 *  x, y, z, m, v and losses are device arrays; point_offsets and
 *  var_offsets are host arrays of n_shapes + 1 entries, and
 *  var_offsets[j + 1] - var_offsets[j] must equal tapes[j]'s variable
 *  count (m and v hold each shape's moments there; zero them before
 *  step 1).  losses[j] receives loss_j at the values before the step.
 *  step counts from 1.  Work is ordered on `stream`; calls on different
 *  streams must not overlap, since they share scratch buffers. */
int lfb_fit_adam_step(const lfb_tape* tapes, uint32_t n_shapes,
                      const uint64_t* point_offsets, const float* x,
                      const float* y, const float* z,
                      const uint64_t* var_offsets, float* m, float* v,
                      lfb_adam_settings adam, uint32_t step, float* losses,
                      void* stream);

/*  Mesh settings (BRepSettings, settings.hpp:27-74, minus the CPU-thread
 *  fields).  min_feature: subdivide until cells are smaller; max_err: QEF
 *  error below which cells collapse (negative disables collapsing).
 *  cancel (NULL: none): BRepSettings::cancel (settings.hpp:73); the mesher
 *  reads it between octree levels, before the leaf and collapse stages and
 *  between dual-walk rounds, and when it is non-zero stops, releases what
 *  the call holds and fails with LFB_E_CANCELLED (the reference returns a
 *  null mesh, worker_pool.inl:82-85, mesh.cpp:61-66). */
typedef struct lfb_mesh_settings {
    double min_feature;
    double max_err;
    const volatile int32_t* cancel;
} lfb_mesh_settings;

typedef struct lfb_mesh_stats {
    uint32_t levels;            /* octree depth (Region::withResolution) */
    uint64_t cells_evaluated;   /* interval-evaluated cells, all levels */
    uint64_t leaf_groups;       /* sibling groups evaluated at the finest level */
    uint64_t leaves_ambiguous;  /* leaf records (ambiguous leaves + collapses) */
    uint64_t clause_evals;      /* value-mode clause x point evaluations in
                                   the leaf kernel (active lanes only) */
    uint64_t clause_evals_grad; /* value+gradient clause x point evaluations */
    uint64_t triangles;
    uint64_t vertices;          /* excluding the placeholder vertex 0 */
    uint64_t kernel_launches;   /* kernels of this library launched */
    double ms_total;            /* host wall time of the whole call */
    double ms_interval;         /* device time per stage (CUDA events) */
    double ms_leaf;
    double ms_collapse;
    double ms_dual;
} lfb_mesh_stats;

/* Number of kernels this library has launched since it was loaded. */
uint64_t lfb_kernel_launches(void);

/* Mesh::render with DUAL_CONTOURING (mesh.cpp:35-125) on the GPU.  The
 * result is freed with libfive_mesh_delete; NULL on failure. */
libfive_mesh* lfb_render_mesh(lfb_tape t, libfive_region3 R,
                              lfb_mesh_settings settings,
                              lfb_mesh_stats* stats);

/* Contours::render (contours.cpp:25-49) on the GPU: the contours of the
 * slice z of the tape over the region R, with BRepSettings' min_feature and
 * max_err (libfive_tree_render_slice uses 1 / res and 1e-8).  Freed with
 * libfive_contours_delete; NULL on failure (lfb_last_error says why).  A
 * closed contour repeats its first point at its end. */
libfive_contours* lfb_render_slice(lfb_tape t, libfive_region2 R, float z,
                                   double min_feature, double max_err);

/* Heightmap::render (heightmap.cpp:247-296) on the GPU over the Voxels
 * region (voxels.cpp:16-44) of lower / upper / res (per-axis voxels per
 * unit; 0 gives one sample).  dims receives {cols, rows, z samples}; when
 * depth is not NULL it receives rows x cols floats (row-major, row = y):
 * the highest z sample at which the shape is filled, -inf where none is;
 * norm (NULL to skip) receives the packed normals (0xAABBGGRR of the
 * normalised gradient mapped to 0..255, 0xffff7f7f at the top sample, 0
 * where empty).  Call with depth NULL to size the arrays. */
int lfb_render_heightmap(lfb_tape t, const float lower[3], const float upper[3],
                         const float res[3], uint32_t dims[3], float* depth,
                         uint32_t* norm);

/* n meshes in one call, each tape over its own region with its own
 * settings.  The reference has no such call (libfive_tree_save_meshes,
 * libfive.cpp:419-440, renders its trees one after another through
 * Mesh::render, mesh.cpp:35-125); here up to `workers` meshes are in flight
 * at once, each on its own CUDA stream with its own scratch buffers (0
 * workers: 4); large meshes run one at a time beside the small ones.  meshes[i] receives tape i's mesh (free it with
 * libfive_mesh_delete), or NULL if that mesh failed; stats is NULL or an
 * array of n.  Returns 0 when every mesh succeeded, else the first failure's
 * LFB_E* code (message from lfb_last_error). */
int lfb_render_meshes(const lfb_tape* tapes, uint32_t n,
                      const libfive_region3* regions,
                      const lfb_mesh_settings* settings, uint32_t workers,
                      libfive_mesh** meshes, lfb_mesh_stats* stats);

/*  Test hooks of the mesher's recovery paths (no counterpart in the
 *  reference), process-wide until set back to 0:
 *    "fail_alloc_after" n > 0: the n-th device allocation from now on fails
 *        as if cudaMalloc had run out of memory (the call in progress fails
 *        with LFB_E_CUDA; nothing else is affected);
 *    "small_capacity" 1: every mesh starts from empty scratch buffers and
 *        minimal tape-arena, list and dual-walk capacities, so each growth
 *        and retry path runs.
 *  Returns 0, or LFB_E_INVALID for an unknown key. */
int lfb_debug_set(const char* key, int64_t value);

/* The reference-layout tape of a tree (Deck, deck.cpp:19-94), for
 * checking slot numbering and for CPU cross-checks.  counts[0..7] =
 * num_clauses, tape length, constants, variables, X, Y, Z, root slot.
 * clauses holds 4 int32 per clause (op, id, a, b) root first; any array may
 * be NULL (call once with NULLs to size them). */
int lfb_tree_slot_tape(libfive_tree t, uint32_t counts[8], int32_t* clauses,
                       uint32_t* const_slots, float* const_values,
                       uint32_t* var_slots, const void** var_ids);

#ifdef __cplusplus
}
#endif
