"""Serving loop: continuous batching of scene simulations on one GPU.

A request is one scene (the flat arrays of :func:`rainbow_b200.engine_io.scene_arrays` or
:func:`rainbow_b200.scenes.batch_arrays`) and a horizon in time steps.  The :class:`Server` keeps every admitted
scene resident on the device -- bodies, their shapes' signed distance grids (in a :class:`ShapeLibrary` shared
by all scenes) and the warm-start contact impulses -- and advances all of them with one ``rb_step`` per tick.
Between ticks finished scenes leave and queued ones are admitted while the device-memory budget (a fraction
of the GPU's memory, 80 % by default) and the optional cap on resident bodies (a step-latency target) allow.
The batch is then re-laid out on the device: ``rb_build_topology`` derives the per-vertex topology and
``rb_repack`` moves the state and the warm-start cache of the staying scenes, so a scene's trajectory does not
depend on which other scenes share its ticks (FP64: bit-identical to running it alone).

Each tick reports its wall time (host bookkeeping and the device step) and the device time of the step; a
scene's step latency is the wall time of the ticks it was stepped in.
"""
import ctypes
import hashlib
import time
from collections import deque

import numpy as np
import torch

from . import _native as N
from . import world as W


def _shape_key(scene, k):
    keys = scene.get("shape_key")
    if keys is not None:
        return str(keys[k])
    sv, st, sg = scene["shape_v_off"], scene["shape_t_off"], scene["shape_g_off"]
    h = hashlib.sha1()
    h.update(np.ascontiguousarray(np.asarray(scene["shape_V"])[sv[k]:sv[k + 1]]).tobytes())
    h.update(np.ascontiguousarray(np.asarray(scene["shape_T"])[st[k]:st[k + 1]]).tobytes())
    h.update(np.ascontiguousarray(np.asarray(scene["shape_grid"]).ravel()[sg[k]:sg[k + 1]]).tobytes())
    h.update(np.asarray(scene["shape_grid_meta"]).reshape(-1, 12)[k].tobytes())
    return "sha1:" + h.hexdigest()


class ShapeLibrary:
    """Shapes resident on the device for every batch of a server, stored once per distinct shape."""

    def __init__(self, device):
        self.device = torch.device(device)
        self.index = {}
        self.V, self.T, self.G, self.meta = [], [], [], []
        self.nv, self.nt = [], []
        self.nv_arr = np.zeros(0, np.int64)
        self.nt_arr = np.zeros(0, np.int64)
        self.rb_shapes = None
        self._dirty = True

    def add(self, scene):
        """Library index of every shape of `scene`, adding the ones not seen before."""
        sv, st, sg = (np.asarray(scene[k]) for k in ("shape_v_off", "shape_t_off", "shape_g_off"))
        out = np.empty(len(sv) - 1, np.int32)
        for k in range(len(sv) - 1):
            key = _shape_key(scene, k)
            if key not in self.index:
                nt = int(st[k + 1] - st[k])
                if nt > W.MAX_TRIANGLES_PER_SHAPE:
                    raise ValueError("shape with %d triangles exceeds %d" % (nt, W.MAX_TRIANGLES_PER_SHAPE))
                self.index[key] = len(self.V)
                self.V.append(np.asarray(scene["shape_V"], np.float64)[sv[k]:sv[k + 1]].reshape(-1))
                self.T.append(np.asarray(scene["shape_T"], np.int32)[st[k]:st[k + 1]].reshape(-1))
                self.G.append(np.asarray(scene["shape_grid"], np.float64).ravel()[sg[k]:sg[k + 1]])
                self.meta.append(np.asarray(scene["shape_grid_meta"], np.float64).reshape(-1, 12)[k])
                self.nv.append(int(sv[k + 1] - sv[k]))
                self.nt.append(nt)
                self._dirty = True
            out[k] = self.index[key]
        if len(self.nv_arr) != len(self.nv):
            self.nv_arr = np.array(self.nv, np.int64)
            self.nt_arr = np.array(self.nt, np.int64)
        return out

    def sync(self):
        """Upload the table if shapes were added since the last upload."""
        if not self._dirty:
            return
        dev = self.device
        cat = lambda a, dt: torch.from_numpy(np.ascontiguousarray(np.concatenate(a))).to(dev, dt)  # noqa: E731
        off = lambda n, dt: torch.from_numpy(np.concatenate([[0], np.cumsum(n)]).astype(dt))  # noqa: E731
        self.t = {
            "V": cat(self.V, torch.float64), "T": cat(self.T, torch.int32), "grid": cat(self.G, torch.float64),
            "v_off": off(self.nv, np.int32).to(dev), "t_off": off(self.nt, np.int32).to(dev),
            "g_off": off([len(g) for g in self.G], np.int64).to(dev),
            "grid_meta": torch.from_numpy(np.concatenate(self.meta)).to(dev, torch.float64),
        }
        self.t["grid32"] = self.t["grid"].float()   # the FP32 modes' contact search reads this copy
        sh = N.RbShapes()
        sh.n_shapes = len(self.V)
        for f in ("V", "v_off", "T", "t_off", "grid", "g_off", "grid_meta"):
            setattr(sh, f, self.t[f].data_ptr())
        sh.max_shape_triangles = max(self.nt)
        sh.grid32 = self.t["grid32"].data_ptr()
        self.rb_shapes = sh
        self._dirty = False

    def nbytes(self):
        return sum(t.numel() * t.element_size() for t in self.t.values()) if not self._dirty else 0


class SceneBlock:
    """Host arrays of one admitted scene, with its shapes mapped into the library."""

    def __init__(self, scene, library):
        sm = library.add(scene)
        nb = len(scene["body_mass"])
        self.n_bodies = nb
        self.shape = sm[np.asarray(scene["body_shape"], np.int64)].astype(np.int32)
        self.mass = np.asarray(scene["body_mass"], np.float64)
        self.inertia = np.asarray(scene["body_inertia"], np.float64).reshape(nb, 3)
        self.fixed = np.asarray(scene["body_fixed"], np.uint8)
        self.material = np.asarray(scene["body_material"], np.int32)
        nf = len(scene["force_kind"])
        order = np.asarray(scene["body_force_order"]).reshape(nb, -1) if nf else np.zeros((nb, 0), np.int32)
        connected = order >= 0                          # row-major: each body's forces in connection order
        self.force_count = connected.sum(axis=1).astype(np.int32)
        self.force_list = order[connected].astype(np.int32)
        self.force_kind = np.asarray(scene["force_kind"], np.int32).reshape(-1)
        self.force_params = np.asarray(scene["force_params"], np.float64).reshape(-1, 4)
        M = len(scene["material_epsilon"])
        self.n_materials = M
        self.material_mu = np.asarray(scene["material_mu"], np.float64).reshape(M * M, 3)
        self.material_eps = np.asarray(scene["material_epsilon"], np.float64).reshape(M * M)
        self.hinge_bodies = np.asarray(scene.get("hinge_bodies", np.zeros((0, 2))), np.int64).reshape(-1, 2)
        self.hinge_frames = np.asarray(scene.get("hinge_frames", np.zeros((0, 12))), np.float64).reshape(-1, 12)
        self.x0 = np.concatenate([np.asarray(scene["body_r"]).reshape(nb, 3),
                                  np.asarray(scene["body_q"]).reshape(nb, 4)], axis=1)
        self.u0 = np.concatenate([np.asarray(scene["body_v"]).reshape(nb, 3),
                                  np.asarray(scene["body_w"]).reshape(nb, 3)], axis=1)


def pack_blocks(blocks, library):
    """Body arrays of a batch of scene blocks (rb_bodies layout; the topology arrays are left to the device)."""
    nb = np.array([b.n_bodies for b in blocks], np.int64)
    P = {"scene_start": np.concatenate([[0], np.cumsum(nb)]).astype(np.int32)}
    cat = lambda name, dt: np.concatenate([getattr(b, name) for b in blocks]).astype(dt)  # noqa: E731
    P["body_shape"] = cat("shape", np.int32)
    P["body_mass"] = cat("mass", np.float64)
    P["body_inertia"] = cat("inertia", np.float64).reshape(-1)
    P["body_fixed"] = cat("fixed", np.uint8)
    P["body_material"] = cat("material", np.int32)
    nf = np.array([len(b.force_kind) for b in blocks], np.int64)
    fbase = np.concatenate([[0], np.cumsum(nf)])
    P["scene_force_start"] = fbase.astype(np.int32)
    P["force_ptr"] = np.concatenate([[0], np.cumsum(cat("force_count", np.int64))]).astype(np.int32)
    fl = [b.force_list + fbase[i] for i, b in enumerate(blocks)]
    P["force_list"] = np.concatenate(fl).astype(np.int32) if sum(len(f) for f in fl) else np.zeros(1, np.int32)
    P["force_kind"] = cat("force_kind", np.int32) if fbase[-1] else np.zeros(1, np.int32)
    P["force_params"] = cat("force_params", np.float64).reshape(-1) if fbase[-1] else np.zeros(4)
    P["n_forces"] = int(fbase[-1])
    mcount = np.array([b.n_materials for b in blocks], np.int64)
    P["scene_material_count"] = mcount.astype(np.int32)
    P["scene_material_offset"] = np.concatenate([[0], np.cumsum(mcount * mcount)[:-1]]).astype(np.int32)
    P["material_mu"] = cat("material_mu", np.float64).reshape(-1)
    P["material_eps"] = cat("material_eps", np.float64)
    nv = library.nv_arr[P["body_shape"]]
    nt = library.nt_arr[P["body_shape"]]
    P["n_body_vertices"] = int(nv.sum())
    P["n_body_triangles"] = int(nt.sum())
    P["n_clusters"] = int(((nt + 31) // 32).sum())
    if max(P["n_body_vertices"], P["n_body_triangles"], 48 * P["n_clusters"]) >= 2 ** 31:
        raise ValueError("scene batch too large for 32-bit topology indices")
    P["n_bodies"] = int(nb.sum())
    W.hinge_arrays(P, [b.hinge_bodies for b in blocks], [b.hinge_frames for b in blocks])
    return P


_BODY_TENSORS = {
    "scene_hinge_start": torch.int32, "hinge_bodies": torch.int32, "hinge_frames": torch.float64,
    "scene_start": torch.int32, "body_shape": torch.int32, "body_mass": torch.float64,
    "body_inertia": torch.float64, "body_fixed": torch.uint8, "body_material": torch.int32,
    "force_ptr": torch.int32, "force_list": torch.int32, "scene_force_start": torch.int32,
    "force_kind": torch.int32, "force_params": torch.float64, "scene_material_offset": torch.int32,
    "scene_material_count": torch.int32, "material_mu": torch.float64, "material_eps": torch.float64,
}


class ServingBatch(W.DeviceWorld):
    """A :class:`DeviceWorld` over library shapes whose layout is rebuilt on the device when scenes come and go.

    ``prev`` (the batch this one replaces) and ``body_map`` (old body -> new body or -1) carry the staying
    scenes' state and warm-start cache; bodies beyond the carried ones start from their block's initial state."""

    def __init__(self, library, blocks, device, caps, max_iterations, prev=None, body_map=None, n_kept=0,
                 pool=None, packed=None):
        t0 = time.perf_counter()
        # device buffers reused from batch to batch (grow-only), so a re-layout allocates nothing in the
        # steady state; the warm-start cache alternates between two slots (the old one feeds rb_repack)
        self.pool = pool if pool is not None else {}
        self.cache_slot = 1 - prev.cache_slot if prev is not None else 0
        self.lib = N.load()
        self.device = torch.device(device)
        self.n_scenes = len(blocks)
        library.sync()
        P = packed if packed is not None else pack_blocks(blocks, library)
        t1 = time.perf_counter()
        dev = self.device
        T = {k: torch.from_numpy(np.ascontiguousarray(P[k])).to(dev, dt) for k, dt in _BODY_TENSORS.items()}
        nbod = P["n_bodies"]
        for k, n in (("body_v0", nbod + 1), ("body_t0", nbod + 1), ("body_c0", nbod + 1),
                     ("vert_body", P["n_body_vertices"]), ("tri_body", P["n_body_triangles"]),
                     ("clu_body", P["n_clusters"])):
            T[k] = self._pooled(k, max(1, n), torch.int32)
        T["x"] = self._pooled("x%d" % self.cache_slot, 7 * nbod, torch.float64)   # the old state feeds rb_repack
        T["u"] = self._pooled("u%d" % self.cache_slot, 6 * nbod, torch.float64)
        self.tensors = T
        self.t_x, self.t_u = T["x"], T["u"]
        self.packed = P
        self.n_shapes = len(library.V)
        self.n_bodies = nbod
        self.scene_start = P["scene_start"]
        self.body_shape = P["body_shape"]
        self.fixed = P["body_fixed"]
        self.n_forces = P["n_forces"]
        self.n_body_vertices, self.n_body_triangles = P["n_body_vertices"], P["n_body_triangles"]
        self.n_clusters = P["n_clusters"]
        self.library = library
        self.rb_shapes = library.rb_shapes
        bd = N.RbBodies()
        bd.n_bodies, bd.n_scenes, bd.n_forces = nbod, self.n_scenes, self.n_forces
        self.n_hinges = int(P["n_hinges"])
        bd.n_hinges = self.n_hinges
        bd.n_body_vertices, bd.n_body_triangles, bd.n_clusters = self.n_body_vertices, self.n_body_triangles, self.n_clusters
        bd.max_scene_bodies = int(np.diff(self.scene_start).max())
        for f, key in W.BODY_FIELDS.items():
            setattr(bd, f, T[key].data_ptr())
        self.rb_bodies = bd
        stream = torch.cuda.current_stream(dev)
        scratch = torch.empty(N.RB_TOPOLOGY_SCRATCH_BYTES, dtype=torch.uint8, device=dev)
        N.check(self.lib.rb_build_topology(ctypes.byref(self.rb_shapes), ctypes.byref(bd), scratch.data_ptr(),
                                           scratch.numel(), stream.cuda_stream), "rb_build_topology")
        self.caps = N.RbCaps()
        self.caps.max_iterations = max(1, int(max_iterations))
        self.caps.pair_capacity, self.caps.item_capacity, self.caps.contact_capacity = caps
        t2 = time.perf_counter()
        self._alloc()
        t3 = time.perf_counter()
        # state: carried rows of the staying bodies, initial rows of the new ones
        if prev is not None and n_kept > 0:
            tmap = torch.from_numpy(np.ascontiguousarray(body_map, np.int32)).to(dev)
            need = ctypes.c_size_t(0)
            N.check(self.lib.rb_repack_workspace_bytes(prev.caps.contact_capacity, ctypes.byref(need)),
                    "rb_repack_workspace_bytes")
            ws = torch.empty(max(1, need.value), dtype=torch.uint8, device=dev)
            N.check(self.lib.rb_repack(tmap.data_ptr(), prev.n_bodies, prev.t_x.data_ptr(), prev.t_u.data_ptr(),
                                       self.t_x.data_ptr(), self.t_u.data_ptr(), prev.t_cache_key.data_ptr(),
                                       prev.t_cache_sol.data_ptr(), prev.t_cache_count.data_ptr(),
                                       prev.caps.contact_capacity, self.t_cache_key.data_ptr(),
                                       self.t_cache_sol.data_ptr(), self.t_cache_count.data_ptr(),
                                       self.caps.contact_capacity, ws.data_ptr(), ws.numel(), stream.cuda_stream),
                    "rb_repack")
        kept_bodies = int(self.scene_start[n_kept])
        if kept_bodies < nbod:
            new = blocks[n_kept:]
            hx = torch.from_numpy(np.ascontiguousarray(np.concatenate([b.x0 for b in new]).reshape(-1)))
            hu = torch.from_numpy(np.ascontiguousarray(np.concatenate([b.u0 for b in new]).reshape(-1)))
            self.t_x[7 * kept_bodies:].copy_(hx.pin_memory(), non_blocking=True)
            self.t_u[6 * kept_bodies:].copy_(hu.pin_memory(), non_blocking=True)
        # host seconds of the re-layout: packing, uploads and topology, work-list allocation, state carry
        self.relayout_times = (t1 - t0, t2 - t1, t3 - t2, time.perf_counter() - t3)

    def _pooled(self, name, n, dtype):
        t = self.pool.get(name)
        if t is None or t.numel() < n:
            t = torch.empty(int(1.25 * n) + 1024, dtype=dtype, device=self.device)
            self.pool[name] = t
        return t[:n]

    def _alloc(self):
        """DeviceWorld._alloc with the server's pooled buffers (outputs are written by every step, so the
        reused buffers need no clearing)."""
        K = self.caps.contact_capacity
        self.t_cids = self._pooled("cids", 2 * K, torch.int32)
        self.t_cp = self._pooled("cp", 3 * K, torch.float64)
        self.t_cn = self._pooled("cn", 3 * K, torch.float64)
        self.t_cg = self._pooled("cg", K, torch.float64)
        self.t_csol = self._pooled("csol", 4 * K, torch.float64)
        self.t_stats = torch.zeros(self.n_scenes * ctypes.sizeof(N.RbSceneStats), dtype=torch.uint8,
                                   device=self.device)
        self.t_resid = self._pooled("resid", self.n_scenes * self.caps.max_iterations, torch.float64)
        self.t_status = torch.zeros(8, dtype=torch.int32, device=self.device)
        old_key, old_sol = getattr(self, "t_cache_key", None), getattr(self, "t_cache_sol", None)
        key = self._pooled("cache_key%d" % self.cache_slot, 2 * K, torch.int64)
        sol = self._pooled("cache_sol%d" % self.cache_slot, 4 * K, torch.float64)
        if old_key is not None and old_key.data_ptr() != key.data_ptr():   # grown within this batch
            n = min(old_key.numel(), key.numel()) // 2
            key[:2 * n].copy_(old_key[:2 * n])
            sol[:4 * n].copy_(old_sol[:4 * n])
        self.t_cache_key, self.t_cache_sol = key, sol
        if not hasattr(self, "t_cache_count"):
            self.t_cache_count = torch.zeros(1, dtype=torch.int32, device=self.device)
        out = N.RbOutputs()
        out.contact_ids, out.contact_p, out.contact_n = self.t_cids.data_ptr(), self.t_cp.data_ptr(), self.t_cn.data_ptr()
        out.contact_g, out.contact_sol = self.t_cg.data_ptr(), self.t_csol.data_ptr()
        out.stats, out.residuals = self.t_stats.data_ptr(), self.t_resid.data_ptr()
        out.status, out.n_contacts_total = self.t_status.data_ptr(), self.t_status.data_ptr() + 4
        out.needed = self.t_status.data_ptr() + 8
        out.cache_key, out.cache_sol = self.t_cache_key.data_ptr(), self.t_cache_sol.data_ptr()
        out.cache_count = self.t_cache_count.data_ptr()
        self.t_hsol = self._pooled("hsol", max(1, 5 * self.n_hinges), torch.float64)
        out.hinge_sol = self.t_hsol.data_ptr()
        self.rb_outputs = out
        nbytes = ctypes.c_size_t(0)
        N.check(self.lib.rb_workspace_bytes(ctypes.byref(self.rb_bodies), ctypes.byref(self.caps), ctypes.byref(nbytes)),
                "rb_workspace_bytes")
        self.workspace_bytes = int(nbytes.value)
        self.t_ws = self._pooled("ws", self.workspace_bytes, torch.uint8)

    def scene_state(self, s):
        """(x, u) rows of scene s on the host."""
        b0, b1 = int(self.scene_start[s]), int(self.scene_start[s + 1])
        x = self.t_x[7 * b0:7 * b1].view(-1, 7).cpu().numpy()
        u = self.t_u[6 * b0:6 * b1].view(-1, 6).cpu().numpy()
        return x, u


class Request:
    __slots__ = ("uid", "scene", "horizon", "arrival", "block", "admitted", "done", "tick_walls", "tick_device",
                 "result", "slot", "error")

    def __init__(self, uid, scene, horizon, arrival):
        self.uid, self.scene, self.horizon, self.arrival = uid, scene, int(horizon), arrival
        self.block = None
        self.admitted = None
        self.done = 0
        self.tick_walls = []
        self.tick_device = []
        self.result = None
        self.error = None   # why the request was rejected (it then never runs)


class Server:
    """Continuous-batching server of scene simulations (see module docstring).

    ``rb_params`` is shared by every scene.  ``max_active_bodies`` caps the resident bodies (None: only the
    memory budget, ``hbm_fraction`` of the device memory, limits admission)."""

    def __init__(self, rb_params, device="cuda", max_iterations=100, hbm_fraction=0.8, max_active_bodies=None,
                 caps_per_body=(8, 64, 16)):
        if not torch.cuda.is_available():
            raise N.NativeError("rainbow_b200 needs a CUDA device; no CPU path exists")
        self.rp = rb_params
        self.device = torch.device(device)
        self.lib = N.load()
        self.max_iterations = max(int(max_iterations), int(rb_params.max_iterations))
        free, total = torch.cuda.mem_get_info(self.device)
        self.budget = int(hbm_fraction * total)
        self.max_active_bodies = max_active_bodies
        self.caps_per_body = list(caps_per_body)
        self.library = ShapeLibrary(device)
        self.pool = {}
        self._next = None          # the next tick's plan, made while the current step runs
        self.queue = deque()
        self.active = []
        self.batch = None
        self.finished = []
        self.rejected = []         # requests whose scene cannot run here, with Request.error set
        self.ticks = []
        self._uid = 0
        self._dirty = False

    # ---------------------------------------------------------------------------------------------------------
    def submit(self, scene, horizon, arrival=None):
        """Queue one scene simulation of `horizon` steps; returns its id."""
        uid = self._uid
        self._uid += 1
        self.queue.append(Request(uid, scene, horizon, time.perf_counter() if arrival is None else arrival))
        return uid

    def idle(self):
        """True when nothing is queued or planned and every resident scene has finished its horizon."""
        planned = self._next is not None and bool(self._next[1])
        return not self.queue and not planned and all(r.done >= r.horizon for r in self.active)

    def _bytes_for(self, n_bodies, n_scenes, nv, nt, nc):
        """Device bytes of a batch of this size: workspace, outputs, cache and body arrays."""
        bd = N.RbBodies()
        bd.n_bodies, bd.n_scenes = n_bodies, n_scenes
        bd.n_body_vertices, bd.n_body_triangles, bd.n_clusters = nv, nt, nc
        caps = N.RbCaps()
        caps.pair_capacity, caps.item_capacity, caps.contact_capacity = self._caps(n_bodies)
        caps.max_iterations = self.max_iterations
        ws = ctypes.c_size_t(0)
        N.check(self.lib.rb_workspace_bytes(ctypes.byref(bd), ctypes.byref(caps), ctypes.byref(ws)),
                "rb_workspace_bytes")
        K = caps.contact_capacity
        outputs = K * (8 + 24 + 24 + 8 + 32 + 16 + 32) + n_scenes * (128 + 8 * self.max_iterations)
        bodies = n_bodies * (13 * 8 + 7 * 8 + 40) + 4 * (nv + nt + nc)
        return int(ws.value) + outputs + bodies

    def _caps(self, n_bodies):
        p, i, c = self.caps_per_body
        return (max(1024, int(p * n_bodies)), max(4096, int(i * n_bodies)), max(1024, int(c * n_bodies)))

    def _admit(self, staying):
        admitted = []
        nb = sum(r.block.n_bodies for r in staying)
        lib = self.library
        counts = [0, 0, 0]
        for r in staying:
            counts[0] += int(lib.nv_arr[r.block.shape].sum())
            counts[1] += int(lib.nt_arr[r.block.shape].sum())
            counts[2] += int(((lib.nt_arr[r.block.shape] + 31) // 32).sum())
        while self.queue:
            r = self.queue[0]
            if r.block is None:
                try:
                    r.block = SceneBlock(r.scene, lib)
                except ValueError as e:   # e.g. a shape beyond the triangle limit: reject it, serve the rest
                    self.queue.popleft()
                    r.error = str(e)
                    self.rejected.append(r)
                    continue
                lib.sync()
            b = r.block
            cnt = (int(lib.nv_arr[b.shape].sum()), int(lib.nt_arr[b.shape].sum()),
                   int(((lib.nt_arr[b.shape] + 31) // 32).sum()))
            # the first scene of an empty server is always admitted, whatever its size
            if self.max_active_bodies is not None and (staying or admitted) and \
                    nb + b.n_bodies > self.max_active_bodies:
                break
            need = self._bytes_for(nb + b.n_bodies, len(staying) + len(admitted) + 1,
                                   counts[0] + cnt[0], counts[1] + cnt[1], counts[2] + cnt[2])
            if need + lib.nbytes() > self.budget and (staying or admitted):
                break
            self.queue.popleft()
            admitted.append(r)
            nb += b.n_bodies
            for k in range(3):
                counts[k] += cnt[k]
        return admitted

    def _relayout(self, staying, admitted, packed=None):
        """New batch of staying + admitted scenes, carrying the staying scenes' state and cache."""
        prev = self.batch
        body_map = None
        if prev is not None:
            body_map = np.full(prev.n_bodies, -1, np.int32)
            new_start = 0
            for r in staying:
                b0, b1 = int(prev.scene_start[r.slot]), int(prev.scene_start[r.slot + 1])
                body_map[b0:b1] = np.arange(new_start, new_start + b1 - b0, dtype=np.int32)
                new_start += b1 - b0
        scenes = staying + admitted
        nb = sum(r.block.n_bodies for r in scenes)
        caps = self._caps(nb)
        if prev is not None:   # keep the grown capacities per body
            ratio = nb / max(1, prev.n_bodies)
            caps = tuple(max(c, int(pc * ratio)) for c, pc in zip(caps, (prev.caps.pair_capacity,
                                                                         prev.caps.item_capacity,
                                                                         prev.caps.contact_capacity)))
        batch = ServingBatch(self.library, [r.block for r in scenes], self.device, caps, self.max_iterations,
                             prev=prev, body_map=body_map, n_kept=len(staying) if prev is not None else 0,
                             pool=self.pool, packed=packed)
        for i, r in enumerate(scenes):
            r.slot = i
        self.batch = batch
        self.active = scenes

    # ---------------------------------------------------------------------------------------------------------
    def _plan(self, staying):
        """Membership of the next tick: the staying scenes plus the queued ones admitted now, and, when it
        differs from the current one, the host arrays of its layout."""
        admitted = self._admit(staying)
        now = time.perf_counter()
        for r in admitted:
            r.admitted = now
        changed = bool(admitted) or len(staying) != len(self.active)
        packed = None
        if changed and (staying or admitted):
            self.library.sync()
            packed = pack_blocks([r.block for r in staying + admitted], self.library)
        return staying, admitted, changed, packed

    def tick(self):
        """Re-lay out if the membership changed, step every resident scene once, retire the finished.

        The next tick's admissions and host-side packing are done while this tick's step runs on the GPU, so
        the host work of continuous batching overlaps the device work.  Returns the requests finished in
        this tick."""
        t0 = time.perf_counter()
        plan = self._next if self._next is not None else self._plan([r for r in self.active if r.done < r.horizon])
        self._next = None
        staying, admitted, changed, packed = plan
        relayout_s = 0.0
        if changed:
            t1 = time.perf_counter()
            if staying or admitted:
                self._relayout(staying, admitted, packed)
            else:
                self.batch, self.active = None, []
            relayout_s = time.perf_counter() - t1
        if not self.active:
            return []
        stream = torch.cuda.current_stream(self.device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        caps0 = (self.batch.caps.pair_capacity, self.batch.caps.item_capacity, self.batch.caps.contact_capacity)
        self.batch.t_status.zero_()
        e0.record(stream)
        self.batch.launch(self.rp)
        e1.record(stream)
        # meanwhile on the host: who stays after this step, who joins, and the next layout's arrays
        self._next = self._plan([r for r in self.active if r.done + 1 < r.horizon])
        status = int(self.batch.t_status[0].item())   # waits for the step
        if status & (N.STATUS_PAIR_OVERFLOW | N.STATUS_ITEM_OVERFLOW | N.STATUS_CONTACT_OVERFLOW):
            self.batch._grow(status)                  # the step left the state alone: grow and repeat it
            status = self.batch.step(self.rp)
            e1.record(stream)
        grown = caps0 != (self.batch.caps.pair_capacity, self.batch.caps.item_capacity,
                          self.batch.caps.contact_capacity)
        if status & N.STATUS_NONFINITE:
            raise N.NativeError("the step produced a non-finite body state")
        done = []
        for r in self.active:
            r.done += 1
            if r.done == r.horizon:
                r.result = self.batch.scene_state(r.slot)
                done.append(r)
        torch.cuda.synchronize(self.device)
        dev_ms = e0.elapsed_time(e1)
        wall = time.perf_counter() - t0
        for r in self.active:
            r.tick_walls.append(wall)
            r.tick_device.append(dev_ms)
        self.ticks.append({"wall_s": wall, "device_ms": dev_ms, "scenes": len(self.active),
                           "bodies": self.batch.n_bodies, "admitted": len(admitted), "finished": len(done),
                           "queued": len(self.queue), "grown": grown,
                           "relayout_s": relayout_s,
                           "relayout_parts_s": self.batch.relayout_times if relayout_s else None})
        self.finished.extend(done)
        return done

    def run(self, max_ticks=None):
        """Tick until every submitted request is finished (or max_ticks)."""
        n = 0
        while not self.idle() and (max_ticks is None or n < max_ticks):
            self.tick()
            n += 1
        return self.finished

    # ---------------------------------------------------------------------------------------------------------
    def report(self):
        """Throughput and latency of the ticks so far."""
        if not self.ticks:
            return {}
        walls = np.array([t["wall_s"] for t in self.ticks])
        scenes = np.array([t["scenes"] for t in self.ticks])
        per_step_wall = np.repeat(walls * 1000.0, scenes)   # one entry per scene-step
        per_step_dev = np.repeat(np.array([t["device_ms"] for t in self.ticks]), scenes)
        out = {
            "ticks": len(self.ticks), "scene_steps": int(scenes.sum()),
            "scene_steps_per_s": float(scenes.sum() / walls.sum()),
            "step_latency_ms_p50_p99": [float(np.percentile(per_step_wall, 50)), float(np.percentile(per_step_wall, 99))],
            "device_step_ms_p50_p99": [float(np.percentile(per_step_dev, 50)), float(np.percentile(per_step_dev, 99))],
            "resident_scenes_mean_max": [float(scenes.mean()), int(scenes.max())],
            "resident_bodies_max": int(max(t["bodies"] for t in self.ticks)),
            "finished": len(self.finished),
        }
        admitted = [r for r in self.finished + self.active if r.admitted is not None]
        if admitted:   # every request that got in so far, finished or still running
            wait = np.array([r.admitted - r.arrival for r in admitted])
            out["queue_wait_s_p50_p99"] = [float(np.percentile(wait, 50)), float(np.percentile(wait, 99))]
        out["rejected"] = len(self.rejected)
        return out
