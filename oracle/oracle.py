"""ctypes wrapper around the C restatement of the reference time step (``oracle/rb_oracle.c``).

TEST INFRASTRUCTURE ONLY: used by the tests, by ``__graft_entry__.smoke()`` as the checker, and by the CPU
baseline leg of ``bench.py``.  The product path (``rainbow_b200``) never imports this module.

The library is built by :func:`build` (``gcc -O2 -ffp-contract=off``) into ``oracle/_build/librb_oracle.so``.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "rb_oracle.c")
LIB = os.path.join(HERE, "_build", "librb_oracle.so")

PARAM_FIELDS = [
    "time_step", "max_iterations", "use_bounce", "use_pre_stabilization", "use_post_stabilization",
    "gap_reduction", "min_gap_value", "max_gap_value", "absolute_tolerance", "relative_tolerance",
    "nu_reduce", "nu_increase", "too_small_merit_change", "contact_optimization_max_iterations",
    "contact_optimization_tolerance", "bvh_chunk_size", "K", "envelope", "resolution",
]

SCHEMES = {"rigid_gauss_seidel": 0, "gauss_seidel": 1, "parallel_jacobi": 2, "parallel_jacobi_hybrid": 3,
           "parallel_jacboi_hybrid": 3, "parallel_gauss_seidel": 4}


def build(force=False):
    """Compile the oracle.  Returns the library path."""
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        cmd = ["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-o", LIB, SRC, "-lm"]
        subprocess.check_call(cmd)
    return LIB


_P = ctypes.POINTER
_d = _P(ctypes.c_double)
_i32 = _P(ctypes.c_int32)
_i64 = _P(ctypes.c_int64)
_u8 = _P(ctypes.c_uint8)


class OScene(ctypes.Structure):
    _fields_ = [
        ("n_shapes", ctypes.c_int32), ("V", _d), ("v_off", _i64), ("T", _i32), ("t_off", _i64),
        ("grid", _d), ("g_off", _i64), ("grid_meta", _d),
        ("n_bodies", ctypes.c_int32), ("body_shape", _i32), ("mass", _d), ("inertia", _d), ("fixed", _u8),
        ("material", _i32), ("n_forces", ctypes.c_int32), ("force_kind", _i32), ("force_params", _d),
        ("body_force_order", _i32), ("n_materials", ctypes.c_int32), ("material_mu", _d), ("material_eps", _d),
        ("n_hinges", ctypes.c_int32), ("hinge_bodies", _i32), ("hinge_frames", _d),
    ]


class OStepOut(ctypes.Structure):
    _fields_ = [
        ("scheme", ctypes.c_int32), ("capacity", ctypes.c_int32),
        ("n_contacts", ctypes.c_int32), ("iterations", ctypes.c_int32), ("exitcode", ctypes.c_int32),
        ("post_iterations", ctypes.c_int32), ("post_exitcode", ctypes.c_int32), ("overflow", ctypes.c_int32),
        ("n_overlap_pairs", ctypes.c_int32), ("n_leaf_overlaps", ctypes.c_int64), ("n_candidates", ctypes.c_int64),
        ("n_colours", ctypes.c_int32),
        ("ids", _i32), ("p", _d), ("n", _d), ("g", _d), ("b", _d), ("diag", _d), ("sol", _d),
        ("residuals", _d), ("delta_u_ext", _d),
        ("kinetic", ctypes.c_double), ("potential", ctypes.c_double), ("max_penetration", ctypes.c_double),
        ("hinge_b", _d), ("hinge_diag", _d), ("hinge_sol", _d),
        ("warm_count", ctypes.c_int32), ("warm_key", _i64), ("warm_sol", _d), ("keys", _i64),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = LIB if os.path.exists(LIB) else build()
        L = ctypes.CDLL(path)
        L.rbo_step.restype = ctypes.c_int
        L.rbo_step.argtypes = [_P(OScene), _d, ctypes.c_double, _d, _d, _d, _d, _P(OStepOut), ctypes.c_int,
                               ctypes.c_double]
        L.rbo_set_residual_interval.argtypes = [ctypes.c_int]
        L.rbo_set_relaxation.argtypes = [ctypes.c_double]
        L.rbo_set_ordering.argtypes = [ctypes.c_int]
        L.rbo_colour_contacts.restype = ctypes.c_int
        L.rbo_colour_contacts.argtypes = [ctypes.c_int, ctypes.c_int, _i32, _u8, _i32]
        L.rbo_grid_value.restype = ctypes.c_double
        L.rbo_grid_value.argtypes = [_d, _d, _d]
        L.rbo_grid_gradient.argtypes = [_d, _d, _d, _d]
        L.rbo_grid_is_inside.restype = ctypes.c_int
        L.rbo_grid_is_inside.argtypes = [_d, _d, ctypes.c_double]
        L.rbo_grid_cell.argtypes = [_d, _d, _i64]
        for name in ("rbo_quat_prod", "rbo_quat_rotate"):
            getattr(L, name).argtypes = [_d, _d, _d]
        L.rbo_quat_rotate_array.argtypes = [_d, _d, ctypes.c_int, _d]
        L.rbo_quat_to_matrix.argtypes = [_d, _d]
        L.rbo_quat_unit.argtypes = [_d, _d]
        L.rbo_make_orthonormal_vectors.argtypes = [_d, _d, _d, _d]
        L.rbo_prox_sphere.argtypes = [ctypes.c_double] * 5 + [_d]
        L.rbo_update_inertia_tensor.argtypes = [_d, _d, _d]
        _lib = L
    return _lib


def _ptr(a, t):
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# --------------------------------------------------------------------------------------------------------------
# primitives (reference unit-test pins)
# --------------------------------------------------------------------------------------------------------------
def quat_prod(a, b):
    a, b, o = _f64(a), _f64(b), np.zeros(4)
    lib().rbo_quat_prod(_ptr(a, _d), _ptr(b, _d), _ptr(o, _d))
    return o


def quat_rotate(q, r):
    q, r, o = _f64(q), _f64(r), np.zeros(3)
    lib().rbo_quat_rotate(_ptr(q, _d), _ptr(r, _d), _ptr(o, _d))
    return o


def quat_rotate_array(q, V):
    q, V = _f64(q), _f64(V).reshape(-1, 3)
    o = np.zeros_like(V)
    lib().rbo_quat_rotate_array(_ptr(q, _d), _ptr(V, _d), len(V), _ptr(o, _d))
    return o


def quat_to_matrix(q):
    q, R = _f64(q), np.zeros(9)
    lib().rbo_quat_to_matrix(_ptr(q, _d), _ptr(R, _d))
    return R.reshape(3, 3)


def quat_unit(q):
    q, o = _f64(q), np.zeros(4)
    lib().rbo_quat_unit(_ptr(q, _d), _ptr(o, _d))
    return o


def make_orthonormal_vectors(n):
    n = _f64(n)
    t, b, nn = np.zeros(3), np.zeros(3), np.zeros(3)
    lib().rbo_make_orthonormal_vectors(_ptr(n, _d), _ptr(t, _d), _ptr(b, _d), _ptr(nn, _d))
    return t, b, nn


def prox_sphere(zs, zt, ztau, mu, xn):
    o = np.zeros(3)
    lib().rbo_prox_sphere(zs, zt, ztau, mu, xn, _ptr(o, _d))
    return tuple(o)


def update_inertia_tensor(R, Bv):
    R, Bv, W = _f64(R).ravel(), _f64(Bv), np.zeros(9)
    lib().rbo_update_inertia_tensor(_ptr(R, _d), _ptr(Bv, _d), _ptr(W, _d))
    return W.reshape(3, 3)


def grid_meta(min_coord, max_coord, I, J, K):
    mn, mx = _f64(min_coord), _f64(max_coord)
    spacing = np.divide(mx - mn, np.array([I - 1, J - 1, K - 1], dtype=np.float64))
    return np.concatenate([mn, mx, spacing, [I, J, K]]).astype(np.float64)


def grid_value(values, meta, p):
    values, meta, p = _f64(values).ravel(), _f64(meta), _f64(p)
    return lib().rbo_grid_value(_ptr(values, _d), _ptr(meta, _d), _ptr(p, _d))


def grid_gradient(values, meta, p):
    values, meta, p = _f64(values).ravel(), _f64(meta), _f64(p)
    g = np.zeros(3)
    lib().rbo_grid_gradient(_ptr(values, _d), _ptr(meta, _d), _ptr(p, _d), _ptr(g, _d))
    return g


def grid_is_inside(meta, p, boundary=0.5):
    meta, p = _f64(meta), _f64(p)
    return bool(lib().rbo_grid_is_inside(_ptr(meta, _d), _ptr(p, _d), boundary))


def grid_cell(meta, p):
    meta, p = _f64(meta), _f64(p)
    o = np.zeros(3, dtype=np.int64)
    lib().rbo_grid_cell(_ptr(meta, _d), _ptr(p, _d), _ptr(o, _i64))
    return tuple(int(v) for v in o)


def colour_contacts(ids, fixed, n_bodies):
    ids = np.ascontiguousarray(ids, dtype=np.int32).reshape(-1, 2)
    fixed = np.ascontiguousarray(fixed, dtype=np.uint8)
    colour = np.zeros(len(ids), dtype=np.int32)
    nc = lib().rbo_colour_contacts(len(ids), n_bodies, _ptr(ids, _i32), _ptr(fixed, _u8), _ptr(colour, _i32))
    return colour, nc


# --------------------------------------------------------------------------------------------------------------
# whole step
# --------------------------------------------------------------------------------------------------------------
class OracleScene:
    """Holds the flat scene arrays (same layout as the golden fixtures) and steps them on the CPU."""

    def __init__(self, arrays):
        a = {k: arrays[k] for k in arrays.keys()}
        self._keep = []

        def keep(x, dt):
            x = np.ascontiguousarray(x, dtype=dt)
            self._keep.append(x)
            return x

        self.n_bodies = int(len(a["body_mass"]))
        self.fixed = keep(a["body_fixed"], np.uint8)
        self.scene = OScene()
        s = self.scene
        s.n_shapes = len(a["shape_v_off"]) - 1
        s.V = _ptr(keep(a["shape_V"], np.float64), _d)
        s.v_off = _ptr(keep(a["shape_v_off"], np.int64), _i64)
        s.T = _ptr(keep(a["shape_T"], np.int32), _i32)
        s.t_off = _ptr(keep(a["shape_t_off"], np.int64), _i64)
        s.grid = _ptr(keep(a["shape_grid"], np.float64), _d)
        s.g_off = _ptr(keep(a["shape_g_off"], np.int64), _i64)
        s.grid_meta = _ptr(keep(a["shape_grid_meta"], np.float64), _d)
        s.n_bodies = self.n_bodies
        s.body_shape = _ptr(keep(a["body_shape"], np.int32), _i32)
        s.mass = _ptr(keep(a["body_mass"], np.float64), _d)
        s.inertia = _ptr(keep(a["body_inertia"], np.float64), _d)
        s.fixed = _ptr(self.fixed, _u8)
        s.material = _ptr(keep(a["body_material"], np.int32), _i32)
        s.n_forces = int(len(a["force_kind"]))
        s.force_kind = _ptr(keep(a["force_kind"], np.int32), _i32)
        s.force_params = _ptr(keep(np.asarray(a["force_params"]).reshape(-1, 4) if s.n_forces else np.zeros((1, 4)),
                                   np.float64), _d)
        s.body_force_order = _ptr(keep(a["body_force_order"] if s.n_forces else np.full((self.n_bodies, 1), -1),
                                       np.int32), _i32)
        s.n_materials = int(len(a["material_epsilon"]))
        s.material_mu = _ptr(keep(a["material_mu"], np.float64), _d)
        s.material_eps = _ptr(keep(a["material_epsilon"], np.float64), _d)
        hb = np.asarray(a["hinge_bodies"], np.int32).reshape(-1, 2) if "hinge_bodies" in a else np.zeros((0, 2))
        self.n_hinges = int(len(hb))
        s.n_hinges = self.n_hinges
        s.hinge_bodies = _ptr(keep(hb if len(hb) else np.zeros((1, 2)), np.int32), _i32)
        hf = np.asarray(a["hinge_frames"], np.float64).reshape(-1, 12) if self.n_hinges else np.zeros((1, 12))
        s.hinge_frames = _ptr(keep(hf, np.float64), _d)
        self.params = np.ascontiguousarray(a["params"], dtype=np.float64).copy()
        self.r = np.ascontiguousarray(a["body_r"], dtype=np.float64).copy()
        self.q = np.ascontiguousarray(a["body_q"], dtype=np.float64).copy()
        self.v = np.ascontiguousarray(a["body_v"], dtype=np.float64).copy()
        self.w = np.ascontiguousarray(a["body_w"], dtype=np.float64).copy()
        # warm-start cache of the last step: contact keys (2 int64 each, ascending) and impulses (4 each)
        self.cache_key = np.zeros((0, 2), np.int64)
        self.cache_sol = np.zeros((0, 4), np.float64)

    def set_state(self, x, u):
        """Body state from (N, 7) x = (r, q) and (N, 6) u = (v, w) arrays."""
        x, u = np.asarray(x, np.float64).reshape(-1, 7), np.asarray(u, np.float64).reshape(-1, 6)
        self.r[:] = x[:, :3]; self.q[:] = x[:, 3:]
        self.v[:] = u[:, :3]; self.w[:] = u[:, 3:]

    def reset_warm_start(self):
        self.cache_key = np.zeros((0, 2), np.int64)
        self.cache_sol = np.zeros((0, 4), np.float64)

    def set_param(self, name, value):
        self.params[PARAM_FIELDS.index(name)] = float(value)

    def step(self, dt=None, scheme="rigid_gauss_seidel", capacity=None, tol_mode=0, tol=0.0, residual_interval=1,
             relaxation=1.0, ordering="serial", warm_start=False):
        """Advance one step; returns a dict with the contact set, solver result and statistics.

        ordering="coloured" makes the Gauss-Seidel schemes visit contacts colour by colour (the colouring of
        rbo_colour_contacts); scheme "parallel_gauss_seidel" always does.  warm_start=True starts each contact
        from the impulses the previous step found for the same key (body pair, side, triangle), as the GPU
        step's cache does; the cache is always refreshed."""
        dt = float(self.params[0] if dt is None else dt)
        cap = int(capacity or max(1024, 64 * self.n_bodies))
        max_it = int(self.params[PARAM_FIELDS.index("max_iterations")])
        out = OStepOut()
        out.scheme = SCHEMES[scheme]
        out.capacity = cap
        bufs = dict(ids=np.zeros((cap, 2), np.int32), p=np.zeros((cap, 3)), n=np.zeros((cap, 3)), g=np.zeros(cap),
                    b=np.zeros(4 * cap), diag=np.zeros(4 * cap), sol=np.zeros(4 * cap),
                    residuals=np.full(max(1, max_it), np.inf), delta_u_ext=np.zeros(6 * self.n_bodies))
        H = max(1, self.n_hinges)
        bufs.update(hinge_b=np.zeros(5 * H), hinge_diag=np.zeros(5 * H), hinge_sol=np.zeros(5 * H))
        for k in ("hinge_b", "hinge_diag", "hinge_sol"):
            setattr(out, k, _ptr(bufs[k], _d))
        keys = np.zeros((cap, 2), np.int64)
        out.keys = _ptr(keys, _i64)
        wk = np.ascontiguousarray(self.cache_key, np.int64)
        ws = np.ascontiguousarray(self.cache_sol, np.float64)
        out.warm_count = len(wk) if warm_start else 0
        out.warm_key = _ptr(wk if len(wk) else np.zeros((1, 2), np.int64), _i64)
        out.warm_sol = _ptr(ws if len(ws) else np.zeros((1, 4)), _d)
        self._warm_keep = (wk, ws)
        out.ids = _ptr(bufs["ids"], _i32)
        for k in ("p", "n", "g", "b", "diag", "sol", "residuals", "delta_u_ext"):
            setattr(out, k, _ptr(bufs[k], _d))
        lib().rbo_set_residual_interval(int(residual_interval))
        lib().rbo_set_relaxation(float(relaxation))
        lib().rbo_set_ordering({"serial": 0, "coloured": 1}[ordering])
        rc = lib().rbo_step(ctypes.byref(self.scene), _ptr(self.params, _d), dt, _ptr(self.r, _d), _ptr(self.q, _d),
                            _ptr(self.v, _d), _ptr(self.w, _d), ctypes.byref(out), int(tol_mode), float(tol))
        if rc == 2:
            raise ValueError("a non-fixed body has no mass")
        if rc == 3:
            raise RuntimeError("ContactPoint.init() was called with non-unit size normal")
        if rc == 1:
            raise RuntimeError("oracle contact capacity %d exceeded (%d contacts)" % (cap, out.n_contacts))
        if rc == 4:
            raise NotImplementedError("hinge joints are solved with the reference stepper's rule only "
                                      "(rigid Gauss-Seidel, merit termination, serial order)")
        K = out.n_contacts
        self.cache_key = keys[:K].copy()
        self.cache_sol = bufs["sol"][:4 * K].reshape(-1, 4).copy()
        return dict(keys=self.cache_key.copy(),
            n_contacts=K, ids=bufs["ids"][:K].copy(), p=bufs["p"][:K].copy(), n=bufs["n"][:K].copy(),
            g=bufs["g"][:K].copy(), b=bufs["b"][:4 * K].copy(), diag=bufs["diag"][:4 * K].copy(),
            sol=bufs["sol"][:4 * K].copy(), iterations=out.iterations, exitcode=out.exitcode,
            residuals=bufs["residuals"].copy(), post_iterations=out.post_iterations,
            post_exitcode=out.post_exitcode, delta_u_ext=bufs["delta_u_ext"].copy(),
            n_overlap_pairs=out.n_overlap_pairs, n_leaf_overlaps=out.n_leaf_overlaps,
            n_candidates=out.n_candidates, n_colours=out.n_colours, kinetic=out.kinetic, potential=out.potential,
            max_penetration=out.max_penetration,
            hinge_b=bufs["hinge_b"][:5 * self.n_hinges].copy(), hinge_diag=bufs["hinge_diag"][:5 * self.n_hinges].copy(),
            hinge_sol=bufs["hinge_sol"][:5 * self.n_hinges].copy(),
            x=np.concatenate([self.r, self.q], axis=1).ravel(), u=np.concatenate([self.v, self.w], axis=1).ravel(),
        )
