"""Device-resident batch of scenes and the host driver of ``rb_step``.

A *scene* is described by flat arrays in the reference's body order (``scene_arrays`` below builds them from an
engine; the golden fixtures store the same layout).  :class:`DeviceWorld` packs one or more scenes into device
tensors, keeps them resident, and advances all of them with one ``rb_step`` call per time step.  Work-list
capacities grow automatically when a step reports an overflow (the step is then repeated from the unchanged
state).
"""
import ctypes

import numpy as np
import torch

from . import _native as N

PARAM_FIELDS = [
    "time_step", "max_iterations", "use_bounce", "use_pre_stabilization", "use_post_stabilization",
    "gap_reduction", "min_gap_value", "max_gap_value", "absolute_tolerance", "relative_tolerance",
    "nu_reduce", "nu_increase", "too_small_merit_change", "contact_optimization_max_iterations",
    "contact_optimization_tolerance", "bvh_chunk_size", "K", "envelope", "resolution",
]

SCHEME_NAMES = {
    "rigid_gauss_seidel": N.SCHEME_RIGID_GS, "gauss_seidel": N.SCHEME_GS, "parallel_jacobi": N.SCHEME_JACOBI,
    "parallel_jacboi_hybrid": N.SCHEME_JACOBI_HYBRID, "parallel_jacobi_hybrid": N.SCHEME_JACOBI_HYBRID,
    "parallel_gauss_seidel": N.SCHEME_COLOURED_GS,
}

MAX_TRIANGLES_PER_SHAPE = 16384


def params_from_vector(vec):
    return {name: float(v) for name, v in zip(PARAM_FIELDS, np.asarray(vec, dtype=np.float64))}


def make_rb_params(p, dt=None, scheme="rigid_gauss_seidel", termination="merit", residual_tolerance=1e-6,
                   profiling=False, warm_start=False, residual_interval=1, relaxation=1.0, precision="fp64",
                   refine_iterations=0, ordering="serial"):
    """rb_params from a Parameters-like mapping (types.py:356 field names).

    ordering="coloured" sweeps the Gauss-Seidel schemes colour by colour (the scheme
    "parallel_gauss_seidel" always does); "serial" is the reference's ascending order."""
    g = p.__getitem__ if isinstance(p, dict) else (lambda k: getattr(p, k))
    rp = N.RbParams()
    rp.dt = float(g("time_step") if dt is None else dt)
    rp.max_iterations = int(g("max_iterations"))
    rp.use_bounce = int(bool(g("use_bounce")))
    rp.use_pre_stabilization = int(bool(g("use_pre_stabilization")))
    rp.use_post_stabilization = int(bool(g("use_post_stabilization")))
    for f in ("gap_reduction", "min_gap_value", "max_gap_value", "absolute_tolerance", "relative_tolerance",
              "nu_reduce", "nu_increase", "too_small_merit_change", "contact_optimization_tolerance", "envelope"):
        setattr(rp, f, float(g(f)))
    rp.contact_optimization_max_iterations = int(g("contact_optimization_max_iterations"))
    if scheme not in SCHEME_NAMES:
        raise NotImplementedError("Unknown solver scheme: %s" % scheme)
    rp.scheme = SCHEME_NAMES[scheme]
    rp.termination = {"merit": N.TERMINATE_MERIT, "residual": N.TERMINATE_RESIDUAL,
                      "residual_fixed_r": N.TERMINATE_RESIDUAL_FIXED_R}[termination]
    rp.residual_tolerance = float(residual_tolerance)
    rp.profiling = int(profiling)   # bit 2 (value 2): also check the FP32 contact search against the FP64 one
    rp.warm_start = int(bool(warm_start))
    rp.residual_interval = int(residual_interval)
    rp.relaxation = float(relaxation)
    rp.precision = {"fp64": N.PRECISION_FP64, "fp32_refine": N.PRECISION_FP32_REFINE,
                    "fp32": N.PRECISION_FP32}[precision]
    rp.refine_iterations = int(refine_iterations)
    rp.ordering = {"serial": N.ORDER_SERIAL, "coloured": N.ORDER_COLOURED}[ordering]
    return rp


def _t(a, dtype, device):
    if isinstance(a, torch.Tensor):   # already a tensor (grids built on the device): no host round trip
        return a.to(device=device, dtype=dtype)
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype)


def _cat_pieces(pieces):
    """Concatenation of (array, start, end) pieces; device tensors stay on the device (adjacent ranges of one
    tensor are joined first, so a scene's grids are copied in one piece)."""
    if not any(isinstance(a, torch.Tensor) for a, _, _ in pieces):
        return np.concatenate([np.asarray(a).ravel()[i:j] for a, i, j in pieces])
    dev = next(a.device for a, _, _ in pieces if isinstance(a, torch.Tensor))
    merged = []
    for a, i, j in pieces:
        if merged and merged[-1][0] is a and merged[-1][2] == i:
            merged[-1][2] = j
        else:
            merged.append([a, i, j])
    return torch.cat([(a.reshape(-1)[i:j] if isinstance(a, torch.Tensor)
                       else torch.from_numpy(np.ascontiguousarray(np.asarray(a).ravel()[i:j])).to(dev))
                      for a, i, j in merged])


PACKED_DTYPES = {
    "shape_V": torch.float64, "shape_v_off": torch.int32, "shape_T": torch.int32, "shape_t_off": torch.int32,
    "shape_grid": torch.float64, "shape_g_off": torch.int64, "shape_grid_meta": torch.float64,
    "scene_start": torch.int32, "body_shape": torch.int32, "body_mass": torch.float64,
    "body_inertia": torch.float64, "body_fixed": torch.uint8, "body_material": torch.int32,
    "force_ptr": torch.int32, "force_list": torch.int32, "scene_force_start": torch.int32,
    "force_kind": torch.int32, "force_params": torch.float64, "scene_material_offset": torch.int32,
    "scene_material_count": torch.int32, "material_mu": torch.float64, "material_eps": torch.float64,
    "body_v0": torch.int32, "body_t0": torch.int32, "body_c0": torch.int32, "vert_body": torch.int32,
    "tri_body": torch.int32, "clu_body": torch.int32, "x": torch.float64, "u": torch.float64,
    "scene_hinge_start": torch.int32, "hinge_bodies": torch.int32, "hinge_frames": torch.float64,
}

# rb_bodies field -> packed array
BODY_FIELDS = {
    "scene_start": "scene_start", "shape": "body_shape", "mass": "body_mass", "inertia": "body_inertia",
    "fixed": "body_fixed", "material": "body_material", "force_ptr": "force_ptr", "force_list": "force_list",
    "scene_force_start": "scene_force_start", "force_kind": "force_kind", "force_params": "force_params",
    "scene_material_offset": "scene_material_offset", "scene_material_count": "scene_material_count",
    "material_mu": "material_mu", "material_eps": "material_eps", "body_v0": "body_v0", "body_t0": "body_t0",
    "body_c0": "body_c0", "vert_body": "vert_body", "tri_body": "tri_body", "clu_body": "clu_body",
    "x": "x", "u": "u", "scene_hinge_start": "scene_hinge_start", "hinge_bodies": "hinge_bodies",
    "hinge_frames": "hinge_frames",
}


def pack_scenes(scenes):
    """Concatenate the flat arrays of several scenes into the rb_shapes / rb_bodies layout (host numpy).

    Shapes carrying the same ``shape_key`` entry are stored once and shared.  Force and material indices are
    rebased per scene; body material indices stay local to their
    scene and index that scene's interaction table.  The topology prefix arrays (vertices, triangles and
    32-triangle clusters per body) are derived from the body-to-shape assignment."""
    V, T, G, meta = [], [], [], []
    v_off, t_off, g_off = [0], [0], [0]
    shape_maps = []
    by_key = {}
    nshape = 0
    for s in scenes:
        sv, st, sg = np.asarray(s["shape_v_off"]), np.asarray(s["shape_t_off"]), np.asarray(s["shape_g_off"])
        ns = len(sv) - 1
        keys = s.get("shape_key")
        local = np.empty(ns, np.int64)
        for k in range(ns):
            if keys is not None and keys[k] in by_key:   # a shape shared by several scenes is stored once
                local[k] = by_key[keys[k]]
                continue
            local[k] = nshape
            if keys is not None:
                by_key[keys[k]] = nshape
            nshape += 1
            nt = int(st[k + 1] - st[k])
            if nt > MAX_TRIANGLES_PER_SHAPE:
                raise ValueError("shape with %d triangles exceeds %d" % (nt, MAX_TRIANGLES_PER_SHAPE))
            V.append(np.asarray(s["shape_V"])[sv[k]:sv[k + 1]])
            T.append(np.asarray(s["shape_T"])[st[k]:st[k + 1]])
            G.append((s["shape_grid"], int(sg[k]), int(sg[k + 1])))
            v_off.append(v_off[-1] + int(sv[k + 1] - sv[k]))
            t_off.append(t_off[-1] + nt)
            g_off.append(g_off[-1] + int(sg[k + 1] - sg[k]))
            meta.append(np.asarray(s["shape_grid_meta"]).reshape(-1, 12)[k])
        shape_maps.append(local)
    P = {"n_shapes": nshape}
    P["shape_V"] = np.concatenate(V).reshape(-1)
    P["shape_T"] = np.concatenate(T).astype(np.int32).reshape(-1)
    P["shape_grid"] = _cat_pieces(G)
    P["shape_v_off"] = np.array(v_off, np.int32)
    P["shape_t_off"] = np.array(t_off, np.int32)
    P["shape_g_off"] = np.array(g_off, np.int64)
    P["shape_grid_meta"] = np.array(meta, np.float64).reshape(-1)
    v_cnt = np.diff(np.array(v_off))
    t_cnt = np.diff(np.array(t_off))

    scene_start, shape_idx, x, u, mass, inertia, fixed, mat = [0], [], [], [], [], [], [], []
    force_ptr, force_list = [0], []
    fkind, fparams, scene_force_start = [], [], [0]
    mat_off, mat_cnt, mu, eps = [], [], [], []
    for si, s in enumerate(scenes):
        nb = len(s["body_mass"])
        scene_start.append(scene_start[-1] + nb)
        shape_idx.append(shape_maps[si][np.asarray(s["body_shape"], np.int64)])
        x.append(np.concatenate([np.asarray(s["body_r"]).reshape(nb, 3), np.asarray(s["body_q"]).reshape(nb, 4)], axis=1))
        u.append(np.concatenate([np.asarray(s["body_v"]).reshape(nb, 3), np.asarray(s["body_w"]).reshape(nb, 3)], axis=1))
        mass.append(np.asarray(s["body_mass"], np.float64))
        inertia.append(np.asarray(s["body_inertia"], np.float64).reshape(nb, 3))
        fixed.append(np.asarray(s["body_fixed"], np.uint8))
        mat.append(np.asarray(s["body_material"], np.int32))
        fbase = scene_force_start[-1]
        nf = len(s["force_kind"])
        order = np.asarray(s["body_force_order"]).reshape(nb, -1) if nf else np.zeros((nb, 0), np.int32)
        for b in range(nb):
            conn = [int(f) + fbase for f in order[b] if f >= 0]
            force_list.extend(conn)
            force_ptr.append(force_ptr[-1] + len(conn))
        fkind.extend(np.asarray(s["force_kind"], np.int32).tolist())
        fparams.extend(np.asarray(s["force_params"], np.float64).reshape(-1, 4).tolist())
        scene_force_start.append(fbase + nf)
        M = len(s["material_epsilon"])
        mat_off.append(len(eps))
        mat_cnt.append(M)
        mu.extend(np.asarray(s["material_mu"], np.float64).reshape(M * M, 3).tolist())
        eps.extend(np.asarray(s["material_epsilon"], np.float64).reshape(M * M).tolist())
    shape_idx = np.concatenate(shape_idx).astype(np.int32)
    n_bodies = int(scene_start[-1])
    P["n_bodies"] = n_bodies
    P["scene_start"] = np.array(scene_start, np.int32)
    P["body_shape"] = shape_idx
    nv = v_cnt[shape_idx]
    nt = t_cnt[shape_idx]
    nc = (nt + 31) // 32
    P["body_v0"] = np.concatenate([[0], np.cumsum(nv)]).astype(np.int64)
    P["body_t0"] = np.concatenate([[0], np.cumsum(nt)]).astype(np.int64)
    P["body_c0"] = np.concatenate([[0], np.cumsum(nc)]).astype(np.int64)
    if max(P["body_v0"][-1], P["body_t0"][-1], 48 * P["body_c0"][-1]) >= 2 ** 31:
        raise ValueError("scene batch too large for 32-bit topology indices")
    for k in ("body_v0", "body_t0", "body_c0"):
        P[k] = P[k].astype(np.int32)
    ar = np.arange(n_bodies, dtype=np.int32)
    P["vert_body"] = np.repeat(ar, nv)
    P["tri_body"] = np.repeat(ar, nt)
    P["clu_body"] = np.repeat(ar, nc)
    P["x"] = np.concatenate(x).reshape(-1)
    P["u"] = np.concatenate(u).reshape(-1)
    P["body_mass"] = np.concatenate(mass)
    P["body_inertia"] = np.concatenate(inertia).reshape(-1)
    P["body_fixed"] = np.concatenate(fixed)
    P["body_material"] = np.concatenate(mat)
    P["force_ptr"] = np.array(force_ptr, np.int32)
    P["force_list"] = np.array(force_list or [0], np.int32)
    P["force_kind"] = np.array(fkind or [0], np.int32)[:max(1, len(fkind))]
    P["force_params"] = np.array(fparams or [[0, 0, 0, 0]], np.float64).reshape(-1)
    P["scene_force_start"] = np.array(scene_force_start, np.int32)
    P["scene_material_offset"] = np.array(mat_off, np.int32)
    P["scene_material_count"] = np.array(mat_cnt, np.int32)
    P["material_mu"] = np.array(mu, np.float64).reshape(-1)
    P["material_eps"] = np.array(eps, np.float64)
    P["n_forces"] = len(fkind)
    hinge_arrays(P, [np.asarray(s_["hinge_bodies"], np.int64).reshape(-1, 2) if "hinge_bodies" in s_
                     else np.zeros((0, 2), np.int64) for s_ in scenes],
                 [np.asarray(s_["hinge_frames"], np.float64).reshape(-1, 12) if "hinge_frames" in s_
                  else np.zeros((0, 12)) for s_ in scenes])
    return P


def hinge_arrays(P, bodies, frames):
    """Hinges of the packed scenes (per scene: parent/child body indices local to the scene, 12 frame values)
    into P: scene_hinge_start, hinge_bodies (global body indices), hinge_frames, n_hinges."""
    start = np.asarray(P["scene_start"], np.int64)
    counts = np.array([len(hb) for hb in bodies], np.int64)
    P["n_hinges"] = int(counts.sum())
    P["scene_hinge_start"] = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    if P["n_hinges"]:
        P["hinge_bodies"] = np.concatenate([hb + start[i] for i, hb in enumerate(bodies)]).astype(np.int32).reshape(-1)
        P["hinge_frames"] = np.concatenate(frames).astype(np.float64).reshape(-1)
    else:
        P["hinge_bodies"] = np.zeros(2, np.int32)
        P["hinge_frames"] = np.zeros(12)


class DeviceWorld:
    """Scenes packed into device tensors; ``step`` advances all of them by one time step."""

    def __init__(self, scenes, device="cuda", caps=None, max_iterations=None):
        if not torch.cuda.is_available():
            raise N.NativeError("rainbow_b200 needs a CUDA device; no CPU path exists")
        self.lib = N.load()
        self.device = torch.device(device)
        if isinstance(scenes, dict):
            scenes = [scenes]
        self.n_scenes = len(scenes)
        self._pack(scenes)
        it = int(max_iterations or max(int(s["params"][1]) for s in scenes))
        self.caps = N.RbCaps()
        self.caps.max_iterations = max(1, it)
        nb = self.n_bodies
        c = caps or {}
        self.caps.pair_capacity = int(c.get("pairs", max(1024, 8 * nb)))
        self.caps.item_capacity = int(c.get("items", max(4096, 64 * nb)))
        self.caps.contact_capacity = int(c.get("contacts", max(1024, 16 * nb)))
        self._alloc()

    # ------------------------------------------------------------------------------------------------------
    def _pack(self, scenes):
        dev = self.device
        P = pack_scenes(scenes)
        self.packed = P
        self.n_shapes = int(P["n_shapes"])
        self.n_bodies = int(P["n_bodies"])
        self.scene_start = P["scene_start"]
        self.body_shape = P["body_shape"]
        self.fixed = P["body_fixed"]
        self.n_forces = int(P["n_forces"])
        self.n_body_vertices = int(P["body_v0"][-1])
        self.n_body_triangles = int(P["body_t0"][-1])
        self.n_clusters = int(P["body_c0"][-1])
        T = {}
        for key, dt in PACKED_DTYPES.items():
            T[key] = _t(P[key], dt, dev)
        self.tensors = T
        self.t_x, self.t_u = T["x"], T["u"]
        sh = N.RbShapes()
        sh.n_shapes = self.n_shapes
        for f in ("V", "v_off", "T", "t_off", "grid", "g_off"):
            setattr(sh, f, T["shape_" + f].data_ptr())
        sh.grid_meta = T["shape_grid_meta"].data_ptr()
        sh.max_shape_triangles = int(np.diff(P["shape_t_off"]).max())
        # FP32 copy of the grids for the contact search of the FP32 precision modes (FP64 steps ignore it)
        T["shape_grid32"] = T["shape_grid"].float()
        sh.grid32 = T["shape_grid32"].data_ptr()
        self.rb_shapes = sh
        bd = N.RbBodies()
        bd.n_bodies, bd.n_scenes = self.n_bodies, self.n_scenes
        bd.n_forces = self.n_forces
        self.n_hinges = int(P["n_hinges"])
        bd.n_hinges = self.n_hinges
        bd.n_body_vertices, bd.n_body_triangles, bd.n_clusters = self.n_body_vertices, self.n_body_triangles, self.n_clusters
        bd.max_scene_bodies = int(np.diff(self.scene_start).max())
        for f, key in BODY_FIELDS.items():
            setattr(bd, f, T[key].data_ptr())
        self.rb_bodies = bd

    def _alloc(self):
        dev = self.device
        K = self.caps.contact_capacity
        self.t_cids = torch.zeros(2 * K, dtype=torch.int32, device=dev)
        self.t_cp = torch.zeros(3 * K, dtype=torch.float64, device=dev)
        self.t_cn = torch.zeros(3 * K, dtype=torch.float64, device=dev)
        self.t_cg = torch.zeros(K, dtype=torch.float64, device=dev)
        self.t_csol = torch.zeros(4 * K, dtype=torch.float64, device=dev)
        self.t_stats = torch.zeros(self.n_scenes * ctypes.sizeof(N.RbSceneStats), dtype=torch.uint8, device=dev)
        self.t_resid = torch.zeros(self.n_scenes * self.caps.max_iterations, dtype=torch.float64, device=dev)
        self.t_status = torch.zeros(8, dtype=torch.int32, device=dev)   # status, n_contacts, needed[3]
        out = N.RbOutputs()
        out.contact_ids, out.contact_p, out.contact_n = self.t_cids.data_ptr(), self.t_cp.data_ptr(), self.t_cn.data_ptr()
        out.contact_g, out.contact_sol = self.t_cg.data_ptr(), self.t_csol.data_ptr()
        out.stats, out.residuals = self.t_stats.data_ptr(), self.t_resid.data_ptr()
        out.status, out.n_contacts_total = self.t_status.data_ptr(), self.t_status.data_ptr() + 4
        out.needed = self.t_status.data_ptr() + 8
        # warm-start cache: keep the previous contents across capacity growth
        old_key = getattr(self, "t_cache_key", None)
        old_sol = getattr(self, "t_cache_sol", None)
        self.t_cache_key = torch.zeros(2 * K, dtype=torch.int64, device=dev)
        self.t_cache_sol = torch.zeros(4 * K, dtype=torch.float64, device=dev)
        if old_key is not None:
            n = min(old_key.numel(), self.t_cache_key.numel()) // 2
            self.t_cache_key[:2 * n].copy_(old_key[:2 * n])
            self.t_cache_sol[:4 * n].copy_(old_sol[:4 * n])
        else:
            self.t_cache_count = torch.zeros(1, dtype=torch.int32, device=dev)
        out.cache_key, out.cache_sol = self.t_cache_key.data_ptr(), self.t_cache_sol.data_ptr()
        out.cache_count = self.t_cache_count.data_ptr()
        self.t_hsol = torch.zeros(max(1, 5 * self.n_hinges), dtype=torch.float64, device=dev)
        out.hinge_sol = self.t_hsol.data_ptr()
        self.rb_outputs = out
        nbytes = ctypes.c_size_t(0)
        N.check(self.lib.rb_workspace_bytes(ctypes.byref(self.rb_bodies), ctypes.byref(self.caps), ctypes.byref(nbytes)),
                "rb_workspace_bytes")
        self.workspace_bytes = int(nbytes.value)
        self.t_ws = torch.empty(self.workspace_bytes, dtype=torch.uint8, device=dev)

    def _grow(self, status):
        need = self.t_status[2:5].cpu().numpy()
        grow = lambda cap, n: int(max(2 * cap, 1.25 * int(n) + 64))  # noqa: E731
        if status & N.STATUS_PAIR_OVERFLOW:
            self.caps.pair_capacity = grow(self.caps.pair_capacity, need[0])
        if status & N.STATUS_ITEM_OVERFLOW:
            self.caps.item_capacity = grow(self.caps.item_capacity, need[1])
        if status & N.STATUS_CONTACT_OVERFLOW:
            self.caps.contact_capacity = grow(self.caps.contact_capacity, need[2])
        self._alloc()

    # ------------------------------------------------------------------------------------------------------
    def launch(self, rb_params, stream=None):
        """Enqueue one step of every scene (asynchronous; the caller checks ``status()`` when it syncs)."""
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        rc = self.lib.rb_step(ctypes.byref(self.rb_shapes), ctypes.byref(self.rb_bodies), ctypes.byref(self.caps),
                              ctypes.byref(rb_params), ctypes.byref(self.rb_outputs), self.t_ws.data_ptr(),
                              self.workspace_bytes, ctypes.c_void_p(st.cuda_stream))
        N.check(rc, "rb_step")

    def capture(self, rb_params):
        """Record one step of every scene into a CUDA graph and return it.

        Replaying the graph (``graph.replay()``) advances the batch exactly like :meth:`launch` with the
        parameters given here, on the stream that replays it.  The graph holds the device addresses of this
        world's tensors, so capacity growth (which reallocates them) invalidates it: check ``t_status`` after
        replays and capture again after a growing :meth:`step`.  The device must have run one uncaptured step
        first (it grants the solver kernels their shared memory outside any capture)."""
        if rb_params.profiling:
            raise ValueError("profiling steps record host-side events and cannot be captured")
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self.launch(rb_params)
        return graph

    def step(self, rb_params, max_retries=8):
        """One synchronous step with automatic capacity growth.  Returns the status word."""
        for _ in range(max_retries):
            self.t_status.zero_()
            self.launch(rb_params)
            status = int(self.t_status[0].item())
            grow = status & (N.STATUS_PAIR_OVERFLOW | N.STATUS_ITEM_OVERFLOW | N.STATUS_CONTACT_OVERFLOW)
            if not grow:
                if status & N.STATUS_MESH_TOO_LARGE:
                    raise ValueError("a shape has more than %d triangles" % MAX_TRIANGLES_PER_SHAPE)
                return status
            self._grow(status)
        raise N.NativeError("rb_step: work-list capacities kept overflowing")

    # ------------------------------------------------------------------------------------------------------
    def stats(self):
        raw = self.t_stats.cpu().numpy().tobytes()
        size = ctypes.sizeof(N.RbSceneStats)
        return [N.RbSceneStats.from_buffer_copy(raw[i * size:(i + 1) * size]) for i in range(self.n_scenes)]

    def hinge_solution(self):
        """The hinge problem's solution of the last step (5 values per hinge, Hinge.idx order per scene)."""
        return self.t_hsol[:5 * self.n_hinges].cpu().numpy()

    def n_contacts_total(self):
        return int(self.t_status[1].item())

    def contacts(self):
        """Host copies of the contact outputs of the last step (global body indices)."""
        K = min(self.n_contacts_total(), self.caps.contact_capacity)
        return dict(ids=self.t_cids[:2 * K].view(K, 2).cpu().numpy(), p=self.t_cp[:3 * K].view(K, 3).cpu().numpy(),
                    n=self.t_cn[:3 * K].view(K, 3).cpu().numpy(), g=self.t_cg[:K].cpu().numpy(),
                    sol=self.t_csol[:4 * K].cpu().numpy())

    def _pinned(self):
        if not hasattr(self, "h_x"):
            self.h_x = torch.empty(7 * self.n_bodies, dtype=torch.float64, pin_memory=True)
            self.h_u = torch.empty(6 * self.n_bodies, dtype=torch.float64, pin_memory=True)
        return self.h_x, self.h_u

    def state(self, copy=True):
        """(x, u) read back through pinned staging buffers: (N, 7) and (N, 6) arrays.

        With ``copy=False`` the arrays are views of the pinned buffers themselves (no host copy): they hold this
        state until the next ``state`` or ``set_state`` call, and passing them back to ``set_state`` uploads
        them without a host copy either."""
        hx, hu = self._pinned()
        hx.copy_(self.t_x, non_blocking=True)
        hu.copy_(self.t_u, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        x, u = hx.numpy().reshape(-1, 7), hu.numpy().reshape(-1, 6)
        return (x.copy(), u.copy()) if copy else (x, u)


    def reset_warm_start(self):
        """Forget the contact impulses carried between steps."""
        self.t_cache_count.zero_()

    def set_state(self, x, u):
        """Upload (x, u) through pinned staging buffers (asynchronous on the current stream).  Arrays that are
        the staging buffers themselves (``state(copy=False)``) are uploaded without a host copy."""
        hx, hu = self._pinned()
        torch.cuda.current_stream(self.device).synchronize()   # staging buffers may still feed a copy
        for src, dst in ((x, hx), (u, hu)):
            d = dst.numpy()
            if not (isinstance(src, np.ndarray) and src.dtype == np.float64 and src.size == d.size
                    and src.__array_interface__["data"][0] == d.__array_interface__["data"][0]):
                d[:] = np.asarray(src, np.float64).reshape(-1)
        self.t_x.copy_(hx, non_blocking=True)
        self.t_u.copy_(hu, non_blocking=True)

    def state_bytes(self):
        return 13 * 8 * self.n_bodies

    def residual_history(self, scene=0):
        m = self.caps.max_iterations
        return self.t_resid[scene * m:(scene + 1) * m].cpu().numpy()

    def profile_times(self):
        """Phase times in seconds of the last profiled step (see rb_profile_times)."""
        buf = (ctypes.c_float * 7)()
        N.check(self.lib.rb_profile_times(buf, 7), "rb_profile_times")
        return [float(v) / 1000.0 for v in buf]
