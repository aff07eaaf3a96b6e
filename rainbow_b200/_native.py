"""ctypes binding of the C ABI in ``include/rainbow_b200.h`` (``rainbow_b200/lib/librainbow_b200.so``).

There is no fallback: if the CUDA library is missing, unloadable, or no CUDA device is present, every entry
point that needs it raises.  The structures below mirror the header field by field.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "librainbow_b200.so")

RB_OK = 0
RB_ERR_ARG, RB_ERR_CUDA, RB_ERR_WORKSPACE, RB_ERR_UNSUPPORTED = 1, 2, 3, 4

STATUS_PAIR_OVERFLOW = 1
STATUS_ITEM_OVERFLOW = 2
STATUS_CONTACT_OVERFLOW = 4
STATUS_NONFINITE = 8
STATUS_NONUNIT_NORMAL = 16
STATUS_MESH_TOO_LARGE = 32

SCHEME_RIGID_GS, SCHEME_GS, SCHEME_JACOBI, SCHEME_JACOBI_HYBRID, SCHEME_COLOURED_GS = 0, 1, 2, 3, 4
TERMINATE_MERIT, TERMINATE_RESIDUAL, TERMINATE_RESIDUAL_FIXED_R = 0, 1, 2
PRECISION_FP64, PRECISION_FP32_REFINE, PRECISION_FP32 = 0, 1, 2
ORDER_SERIAL, ORDER_COLOURED = 0, 1
RB_TOPOLOGY_SCRATCH_BYTES = 4096

_vp = ctypes.c_void_p
_sz = ctypes.c_size_t
_i32 = ctypes.c_int32


class RbShapes(ctypes.Structure):
    _fields_ = [("n_shapes", _i32), ("V", _vp), ("v_off", _vp), ("T", _vp), ("t_off", _vp), ("grid", _vp),
                ("g_off", _vp), ("grid_meta", _vp), ("max_shape_triangles", _i32), ("grid32", _vp)]


class RbBodies(ctypes.Structure):
    _fields_ = [
        ("n_bodies", _i32), ("n_scenes", _i32), ("scene_start", _vp), ("shape", _vp), ("mass", _vp),
        ("inertia", _vp), ("fixed", _vp), ("material", _vp), ("force_ptr", _vp), ("force_list", _vp),
        ("n_forces", _i32), ("scene_force_start", _vp), ("force_kind", _vp), ("force_params", _vp),
        ("scene_material_offset", _vp), ("scene_material_count", _vp), ("material_mu", _vp),
        ("material_eps", _vp),
        ("n_body_vertices", _i32), ("n_body_triangles", _i32), ("n_clusters", _i32), ("max_scene_bodies", _i32),
        ("body_v0", _vp), ("body_t0", _vp), ("body_c0", _vp), ("vert_body", _vp), ("tri_body", _vp),
        ("clu_body", _vp), ("x", _vp), ("u", _vp),
        ("n_hinges", _i32), ("scene_hinge_start", _vp), ("hinge_bodies", _vp), ("hinge_frames", _vp),
    ]


class RbCaps(ctypes.Structure):
    _fields_ = [("pair_capacity", _i32), ("item_capacity", _i32), ("contact_capacity", _i32),
                ("max_iterations", _i32)]


class RbParams(ctypes.Structure):
    _fields_ = [
        ("dt", ctypes.c_double), ("max_iterations", _i32), ("use_bounce", _i32), ("use_pre_stabilization", _i32),
        ("use_post_stabilization", _i32), ("gap_reduction", ctypes.c_double), ("min_gap_value", ctypes.c_double),
        ("max_gap_value", ctypes.c_double), ("absolute_tolerance", ctypes.c_double),
        ("relative_tolerance", ctypes.c_double), ("nu_reduce", ctypes.c_double), ("nu_increase", ctypes.c_double),
        ("too_small_merit_change", ctypes.c_double), ("contact_optimization_max_iterations", _i32),
        ("contact_optimization_tolerance", ctypes.c_double), ("envelope", ctypes.c_double), ("scheme", _i32),
        ("termination", _i32), ("residual_tolerance", ctypes.c_double), ("profiling", _i32),
        ("relaxation", ctypes.c_double), ("residual_interval", _i32), ("precision", _i32),
        ("refine_iterations", _i32), ("warm_start", _i32), ("ordering", _i32),
        ("fp32_small_slab", _i32), ("fp32_mid_slab", _i32), ("mid_blocks", _i32), ("narrow_blocks", _i32),
        ("narrow_threads", _i32),
    ]


class RbSceneStats(ctypes.Structure):
    _fields_ = [
        ("n_contacts", _i32), ("contact_start", _i32), ("iterations", _i32), ("exitcode", _i32),
        ("post_iterations", _i32), ("post_exitcode", _i32), ("n_pairs", _i32), ("n_candidates", _i32),
        ("n_leaf_overlaps", _i32), ("n_grid_lookups", _i32),
        ("n_levels", _i32), ("fp32_sweeps", _i32), ("merit", ctypes.c_double), ("residual", ctypes.c_double), ("kinetic_energy", ctypes.c_double),
        ("potential_energy", ctypes.c_double), ("max_penetration", ctypes.c_double),
        ("solve_start_us", ctypes.c_double), ("solve_us", ctypes.c_double),
        ("n_search_flips", _i32), ("n_accept_flips", _i32), ("n_grid_lookups32", _i32),
    ]


class RbOutputs(ctypes.Structure):
    _fields_ = [("contact_ids", _vp), ("contact_p", _vp), ("contact_n", _vp), ("contact_g", _vp),
                ("contact_sol", _vp), ("stats", _vp), ("residuals", _vp), ("status", _vp),
                ("n_contacts_total", _vp), ("needed", _vp), ("cache_key", _vp), ("cache_sol", _vp),
                ("cache_count", _vp), ("hinge_sol", _vp)]


# exported symbols and their ctypes signatures: every function declared in include/rainbow_b200.h
SIGNATURES = {
    "rb_abi_version": (ctypes.c_int, []),
    "rb_last_error": (ctypes.c_char_p, []),
    "rb_topology_sizes": (ctypes.c_int, [_i32, _vp, _i32, _vp, _vp, _vp]),
    "rb_workspace_bytes": (ctypes.c_int, [ctypes.POINTER(RbBodies), ctypes.POINTER(RbCaps),
                                          ctypes.POINTER(ctypes.c_size_t)]),
    "rb_step": (ctypes.c_int, [ctypes.POINTER(RbShapes), ctypes.POINTER(RbBodies), ctypes.POINTER(RbCaps),
                               ctypes.POINTER(RbParams), ctypes.POINTER(RbOutputs), _vp, ctypes.c_size_t, _vp]),
    "rb_signed_distance_grid": (ctypes.c_int, [_vp, _i32, _vp, _i32, _vp, _vp, _vp]),
    "rb_signed_distance_grids": (ctypes.c_int, [_i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int64, _vp, _vp]),
    "rb_profile_times": (ctypes.c_int, [ctypes.POINTER(ctypes.c_float), _i32]),
    "rb_launch_count": (ctypes.c_int64, []),
    "rb_build_topology": (ctypes.c_int, [ctypes.POINTER(RbShapes), ctypes.POINTER(RbBodies), _vp, _sz, _vp]),
    "rb_repack_workspace_bytes": (ctypes.c_int, [_i32, ctypes.POINTER(_sz)]),
    "rb_repack": (ctypes.c_int, [_vp, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _vp, _vp, _vp, _i32, _vp, _sz,
                                 _vp]),
    "rb_step_noalloc": (ctypes.c_int, [ctypes.POINTER(RbShapes), ctypes.POINTER(RbBodies), ctypes.POINTER(RbCaps),
                                       ctypes.POINTER(RbParams), ctypes.POINTER(RbOutputs), _vp]),
}

_lib = None


class NativeError(RuntimeError):
    """Raised when the CUDA library reports an error or cannot be used."""


def load():
    """Load the CUDA library (raises if it is missing: there is no CPU path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise NativeError("rainbow_b200 CUDA library not built: %s (run __graft_entry__.build())" % LIB_PATH)
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if lib.rb_abi_version() != 2:
            raise NativeError("rainbow_b200 ABI version mismatch")
        _lib = lib
    return _lib


def check(rc, what):
    if rc != RB_OK:
        msg = load().rb_last_error().decode(errors="replace")
        if rc == RB_ERR_ARG:
            raise ValueError("%s: %s" % (what, msg))
        raise NativeError("%s failed (code %d): %s" % (what, rc, msg))
