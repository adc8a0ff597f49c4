"""ctypes bindings to libfive_b200/lib/libfive.so.

The structs mirror include/libfive.h, which matches the reference's
libfive/include/libfive.h field for field, so these are the same bindings the
reference's Python package declares (libfive/bind/python/libfive/ffi.py),
plus the batched entry points of include/libfive_b200.h.

Loading fails loudly when the shared library has not been built: there is
no CPU fallback for any entry point.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libfive.so")


class Interval(ctypes.Structure):
    _fields_ = [("lower", ctypes.c_float), ("upper", ctypes.c_float)]


class Region2(ctypes.Structure):
    _fields_ = [("X", Interval), ("Y", Interval)]


class Pixels(ctypes.Structure):
    _fields_ = [("pixels", ctypes.POINTER(ctypes.c_bool)), ("width", ctypes.c_uint32),
                ("height", ctypes.c_uint32)]


class Region3(ctypes.Structure):
    _fields_ = [("X", Interval), ("Y", Interval), ("Z", Interval)]


class Vec3(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float),
                ("z", ctypes.c_float)]


class MeshCoords(ctypes.Structure):
    _fields_ = [("verts", ctypes.POINTER(Vec3)), ("vert_count", ctypes.c_uint32),
                ("coord_indices", ctypes.POINTER(ctypes.c_int32)),
                ("coord_index_count", ctypes.c_uint32)]


class Tri(ctypes.Structure):
    _fields_ = [("a", ctypes.c_uint32), ("b", ctypes.c_uint32),
                ("c", ctypes.c_uint32)]


class Contour(ctypes.Structure):
    _fields_ = [("pts", ctypes.c_void_p), ("count", ctypes.c_uint32)]


class Contours(ctypes.Structure):
    _fields_ = [("cs", ctypes.POINTER(Contour)), ("count", ctypes.c_uint32)]


class Mesh(ctypes.Structure):
    _fields_ = [("verts", ctypes.POINTER(Vec3)), ("tris", ctypes.POINTER(Tri)),
                ("tri_count", ctypes.c_uint32), ("vert_count", ctypes.c_uint32)]


class Vars(ctypes.Structure):
    _fields_ = [("vars", ctypes.POINTER(ctypes.c_void_p)),
                ("values", ctypes.POINTER(ctypes.c_float)),
                ("size", ctypes.c_uint32)]


class AdamSettings(ctypes.Structure):
    _fields_ = [("lr", ctypes.c_float), ("beta1", ctypes.c_float),
                ("beta2", ctypes.c_float), ("eps", ctypes.c_float)]


class MeshSettings(ctypes.Structure):
    _fields_ = [("min_feature", ctypes.c_double), ("max_err", ctypes.c_double),
                ("cancel", ctypes.POINTER(ctypes.c_int32))]


class MeshStats(ctypes.Structure):
    _fields_ = [("levels", ctypes.c_uint32),
                ("cells_evaluated", ctypes.c_uint64),
                ("leaf_groups", ctypes.c_uint64),
                ("leaves_ambiguous", ctypes.c_uint64),
                ("clause_evals", ctypes.c_uint64),
                ("clause_evals_grad", ctypes.c_uint64),
                ("triangles", ctypes.c_uint64),
                ("vertices", ctypes.c_uint64),
                ("kernel_launches", ctypes.c_uint64),
                ("ms_total", ctypes.c_double),
                ("ms_interval", ctypes.c_double),
                ("ms_leaf", ctypes.c_double),
                ("ms_collapse", ctypes.c_double),
                ("ms_dual", ctypes.c_double)]


tree_t = ctypes.c_void_p
tape_t = ctypes.c_void_p
fp = ctypes.POINTER(ctypes.c_float)
u8p = ctypes.POINTER(ctypes.c_uint8)
u32p = ctypes.POINTER(ctypes.c_uint32)
i32p = ctypes.POINTER(ctypes.c_int32)
vp = ctypes.c_void_p

# (name, restype, argtypes); every symbol declared in include/*.h
SIGNATURES = [
    ("libfive_contours_delete", None, [vp]),
    ("libfive_contours3_delete", None, [vp]),
    ("libfive_mesh_delete", None, [ctypes.POINTER(Mesh)]),
    ("libfive_mesh_coords_delete", None, [vp]),
    ("libfive_pixels_delete", None, [ctypes.POINTER(Pixels)]),
    ("libfive_opcode_enum", ctypes.c_int, [ctypes.c_char_p]),
    ("libfive_opcode_args", ctypes.c_int, [ctypes.c_int]),
    ("libfive_vars_delete", None, [vp]),
    ("libfive_tree_x", tree_t, []),
    ("libfive_tree_y", tree_t, []),
    ("libfive_tree_z", tree_t, []),
    ("libfive_tree_var", tree_t, []),
    ("libfive_tree_is_var", ctypes.c_bool, [tree_t]),
    ("libfive_tree_const", tree_t, [ctypes.c_float]),
    ("libfive_tree_get_const", ctypes.c_float, [tree_t, ctypes.POINTER(ctypes.c_bool)]),
    ("libfive_tree_nullary", tree_t, [ctypes.c_int]),
    ("libfive_tree_unary", tree_t, [ctypes.c_int, tree_t]),
    ("libfive_tree_binary", tree_t, [ctypes.c_int, tree_t, tree_t]),
    ("libfive_tree_id", vp, [tree_t]),
    ("libfive_tree_eval_f", ctypes.c_float, [tree_t, Vec3]),
    ("libfive_tree_eval_r", Interval, [tree_t, Region3]),
    ("libfive_tree_eval_d", Vec3, [tree_t, Vec3]),
    ("libfive_tree_delete", None, [tree_t]),
    ("libfive_tree_save", ctypes.c_bool, [tree_t, ctypes.c_char_p]),
    ("libfive_tree_load", tree_t, [ctypes.c_char_p]),
    ("libfive_tree_remap", tree_t, [tree_t, tree_t, tree_t, tree_t]),
    ("libfive_tree_optimized", tree_t, [tree_t]),
    ("libfive_tree_print", ctypes.c_void_p, [tree_t]),
    ("libfive_free_str", None, [ctypes.c_void_p]),
    ("libfive_tree_render_slice", ctypes.POINTER(Contours), [tree_t, Region2, ctypes.c_float, ctypes.c_float]),
    ("libfive_tree_render_slice3", ctypes.POINTER(Contours), [tree_t, Region2, ctypes.c_float, ctypes.c_float]),
    ("libfive_tree_save_slice", None, [tree_t, Region2, ctypes.c_float, ctypes.c_float, ctypes.c_char_p]),
    ("libfive_tree_render_mesh", ctypes.POINTER(Mesh), [tree_t, Region3, ctypes.c_float]),
    ("libfive_tree_render_mesh_st", ctypes.POINTER(Mesh), [tree_t, Region3, ctypes.c_float]),
    ("libfive_tree_render_mesh_coords", ctypes.POINTER(MeshCoords), [tree_t, Region3, ctypes.c_float]),
    ("libfive_tree_save_mesh", ctypes.c_bool, [tree_t, Region3, ctypes.c_float, ctypes.c_char_p]),
    ("libfive_evaluator_save_mesh", ctypes.c_bool, [vp, Region3, ctypes.c_char_p]),
    ("libfive_tree_save_meshes", ctypes.c_bool, [ctypes.POINTER(tree_t), Region3, ctypes.c_float, ctypes.c_float, ctypes.c_char_p]),
    ("libfive_tree_render_pixels", ctypes.POINTER(Pixels), [tree_t, Region2, ctypes.c_float, ctypes.c_float]),
    ("libfive_tree_evaluator", vp, [tree_t, Vars]),
    ("libfive_evaluator_update_vars", ctypes.c_bool, [vp, Vars]),
    ("libfive_evaluator_delete", None, [vp]),
    ("libfive_git_version", ctypes.c_char_p, []),
    ("libfive_git_revision", ctypes.c_char_p, []),
    ("libfive_git_branch", ctypes.c_char_p, []),
    # libfive_b200.h
    ("lfb_last_error", ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint32]),
    ("lfb_tape_new", tape_t, [tree_t, Vars]),
    ("lfb_tape_delete", None, [tape_t]),
    ("lfb_tape_set_vars", ctypes.c_int, [tape_t, Vars]),
    ("lfb_tape_info", ctypes.c_int, [tape_t, u32p]),
    ("lfb_tape_compiled", ctypes.c_int, [tape_t]),
    ("lfb_tape_var_ids", ctypes.c_int, [tape_t, ctypes.POINTER(vp), ctypes.c_uint32]),
    ("lfb_eval_derivs_static", ctypes.c_int, [tape_t, ctypes.c_uint64, vp, vp, vp, vp, vp, vp, vp]),
    ("lfb_eval_values", ctypes.c_int, [tape_t, ctypes.c_uint64, vp, vp, vp, vp, vp, ctypes.c_uint32]),
    ("lfb_eval_derivs", ctypes.c_int, [tape_t, ctypes.c_uint64, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_uint32]),
    ("lfb_eval_intervals", ctypes.c_int, [tape_t, ctypes.c_uint64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_uint32]),
    ("lfb_eval_features", ctypes.c_int, [tape_t, ctypes.c_uint64, vp, vp, vp, vp, vp, ctypes.c_uint32, vp]),
    ("lfb_eval_loss_grad", ctypes.c_int, [tape_t, ctypes.c_uint64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_uint32]),
    ("lfb_eval_jacobian", ctypes.c_int, [tape_t, ctypes.c_uint64, vp, vp, vp, vp, vp, ctypes.c_uint32]),
    ("lfb_eval_grad", ctypes.c_int, [tape_t, ctypes.c_uint64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_uint32]),
    ("lfb_tape_get_vars", ctypes.c_int, [tape_t, fp, ctypes.c_uint32]),
    ("lfb_tape_set_vars_device", ctypes.c_int, [tape_t, vp, ctypes.c_uint32, vp]),
    ("lfb_debug_set", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int64]),
    ("lfb_fit_adam_step", ctypes.c_int, [ctypes.POINTER(tape_t), ctypes.c_uint32,
                                         ctypes.POINTER(ctypes.c_uint64), vp, vp, vp,
                                         ctypes.POINTER(ctypes.c_uint64), vp, vp, AdamSettings,
                                         ctypes.c_uint32, vp, vp]),
    ("lfb_render_mesh", ctypes.POINTER(Mesh), [tape_t, Region3, MeshSettings, ctypes.POINTER(MeshStats)]),
    ("lfb_render_slice", ctypes.POINTER(Contours), [tape_t, Region2, ctypes.c_float, ctypes.c_double,
                                                    ctypes.c_double]),
    ("lfb_render_heightmap", ctypes.c_int, [tape_t, fp, fp, fp, u32p, fp, u32p]),
    ("lfb_render_meshes", ctypes.c_int, [ctypes.POINTER(tape_t), ctypes.c_uint32,
                                         ctypes.POINTER(Region3), ctypes.POINTER(MeshSettings),
                                         ctypes.c_uint32, ctypes.POINTER(ctypes.POINTER(Mesh)),
                                         ctypes.POINTER(MeshStats)]),
    ("lfb_kernel_launches", ctypes.c_uint64, []),
    ("lfb_tree_slot_tape", ctypes.c_int, [tree_t, u32p, i32p, u32p, fp, u32p, ctypes.POINTER(vp)]),
]

LFB_DEVICE_PTRS = 1

_lib = None


def load(path=LIB_PATH):
    """Loads the shared library (once) and declares every signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -m libfive_b200.build`")
    lib = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def last_error():
    lib = load()
    buf = ctypes.create_string_buffer(512)
    code = lib.lfb_last_error(buf, 512)
    return code, buf.value.decode()


def check(rc, what="libfive_b200"):
    if rc < 0:
        code, msg = last_error()
        raise RuntimeError(f"{what} failed ({code}): {msg}")
    return rc
