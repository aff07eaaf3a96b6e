"""Drop-in GPU replacement of ``SemiImplicitStepper`` (rainbow/simulators/prox_rigid_bodies/steppers.py:39).

Install on any engine (the reference's or :mod:`rainbow_b200.types`)::

    engine.stepper = GpuStepper()
    API.simulate(engine, T)            # api.py:676 calls engine.stepper.step(dt, engine, profiling_on)

Each ``step`` uploads the body state (and, when the scene's structure changed, the whole scene), runs one
``rb_step`` on the GPU, and writes the new ``r, q, v, w`` back into the engine's bodies.  ``engine.contact_points``
becomes a sequence of ``ContactPoint`` objects created on first access.  With ``profiling_on`` a dict with the
reference's log keys (steppers.py:95-106, collision_detection.py, gauss_seidel_solver.py) is appended to ``log``.
"""
import time
from collections.abc import Sequence

import numpy as np

from . import engine_io
from . import world as W
from ._native import NativeError

PHASES = ("update_bvh", "narrow_phase", "contact_determination", "contact_point_reduction", "solver_time",
          "integration_time", "gpu_step_time")


class ContactPoints(Sequence):
    """``engine.contact_points`` of one step; ContactPoint objects are built lazily from host copies."""

    def __init__(self, bodies, ids, p, n, g, factory, offset=0):
        self._bodies = bodies
        self._ids, self._p, self._n, self._g = ids, p, n, g
        self._offset = offset   # ids are batch-global: the scene's first body index
        self._factory = factory
        self._items = None

    def __len__(self):
        return len(self._g)

    def _build(self):
        if self._items is None:
            b, o = self._bodies, self._offset
            self._items = [self._factory(b[int(i) - o], b[int(j) - o], self._p[k].copy(), self._n[k].copy(),
                                         float(self._g[k])) for k, (i, j) in enumerate(self._ids)]
        return self._items

    def __getitem__(self, i):
        return self._build()[i]

    def __iter__(self):
        return iter(self._build())

    def __bool__(self):
        return len(self) > 0

    def arrays(self):
        """The contact set as arrays: body indices (SDF owner, mesh owner), positions, normals, gaps."""
        return self._ids - self._offset if self._offset else self._ids, self._p, self._n, self._g


def _contact_factory(engine):
    """ContactPoint constructor of the engine's own type module when available."""
    mod = type(engine).__module__
    try:
        import importlib
        cls = getattr(importlib.import_module(mod), "ContactPoint")
    except (ImportError, AttributeError):
        from .types import ContactPoint as cls

    def make(a, b, p, n, g):
        return cls(a, b, p, n, g)
    return make


def _step_params(params, dt, termination, residual_tolerance, profiling_on, residual_interval=1):
    """rb_params of one step from an engine's Parameters (the reference's fields, plus the optional
    ``proximal_solver``, ``warm_start``, ``contact_ordering`` and ``solver_precision`` attributes)."""
    scheme = getattr(params, "proximal_solver", None) or "rigid_gauss_seidel"
    return W.make_rb_params(params, dt=dt, scheme=scheme, termination=termination,
                            residual_tolerance=residual_tolerance, profiling=profiling_on,
                            warm_start=bool(getattr(params, "warm_start", False)),
                            residual_interval=residual_interval,
                            ordering=getattr(params, "contact_ordering", None) or "serial",
                            precision=getattr(params, "solver_precision", None) or "fp64")


def _check_status(status):
    if status & 16:
        raise RuntimeError("ContactPoint.init() was called with non-unit size normal")
    if status & 8:
        raise NativeError("the step produced a non-finite body state")
    return status


class GpuStepper:
    """Semi-implicit stepper whose whole step runs on the GPU (see module docstring)."""

    def __init__(self, device="cuda", termination="merit", residual_tolerance=1e-6):
        self.log = []
        self.device = device
        self.termination = termination
        self.residual_tolerance = residual_tolerance
        self._world = None
        self._sig = None

    def _world_for(self, engine):
        sig = engine_io.static_signature(engine)
        if self._world is None or sig != self._sig:
            arrays = engine_io.scene_arrays(engine)
            self._world = W.DeviceWorld(arrays, device=self.device, max_iterations=max(1, int(engine.params.max_iterations)))
            self._sig = sig
        else:
            x, u = engine_io.body_state(engine)
            self._world.set_state(x, u)
        if int(engine.params.max_iterations) > self._world.caps.max_iterations:
            arrays = engine_io.scene_arrays(engine)
            self._world = W.DeviceWorld(arrays, device=self.device, max_iterations=int(engine.params.max_iterations))
        return self._world

    def step(self, dt, engine, profiling_on):
        """steppers.py:47 SemiImplicitStepper.step on the GPU."""
        t0 = time.perf_counter()
        if not engine.bodies:
            engine.contact_points = []
            return
        world = self._world_for(engine)
        rp = _step_params(engine.params, dt, self.termination, self.residual_tolerance, profiling_on)
        _check_status(world.step(rp))
        x, u = world.state()
        engine_io.write_back(engine, x, u)
        c = world.contacts()
        bodies = list(engine.bodies.values())
        engine.contact_points = ContactPoints(bodies, c["ids"], c["p"], c["n"], c["g"], _contact_factory(engine))
        if profiling_on:
            st = world.stats()[0]
            times = world.profile_times()
            d = {}
            d["update_bvh"] = times[0]
            d["narrow_phase"] = times[1]
            d["number_of_overlaps"] = int(st.n_leaf_overlaps)
            d["contact_determination"] = times[2]
            # the model-space transform, Frank-Wolfe search and contact generation run fused in one kernel
            d["model_space_update"] = 0.0
            d["contact_optimization"] = times[2]
            d["contact_point_generation"] = 0.0
            d["contact_point_reduction"] = times[3]
            d["collision_detection_time"] = times[0] + times[1] + times[2] + times[3]
            if st.n_contacts > 0:
                res = world.residual_history(0)[: int(engine.params.max_iterations)]
                d["residuals"] = res
                d["iterations"] = int(st.iterations)
                d["exitcode"] = int(st.exitcode)
                d["solver_time"] = times[4]
                if st.post_iterations >= 0:
                    d["post_stabilization_iterations"] = int(st.post_iterations)
                    d["post_stabilization_exitcode"] = int(st.post_exitcode)
            d["stepper_time"] = time.perf_counter() - t0
            d["gpu_step_time"] = times[6]
            d["dt"] = dt
            d["contact_points"] = int(st.n_contacts)
            d["kinetic_energy"] = float(st.kinetic_energy)
            d["potential_energy"] = float(st.potential_energy)
            d["max_penetration"] = float(st.max_penetration)
            self.log.append(d)


class BatchStepper:
    """Steps many engines as one batch: one ``rb_step`` per time step advances all of them.

    The batched form of :class:`GpuStepper` for many independent scenes (``api.simulate_batch`` drives it).
    Each engine's step reads only its own bodies, so every engine ends in the state a :class:`GpuStepper`
    of its own would give it (bit-identical in FP64).  The engines must agree on the parameters the step
    reads (``engine.params``, the reference's fields and the optional solver attributes); their bodies,
    shapes, forces and materials are their own.

    Each ``step`` uploads the bodies' ``r, q, v, w`` (only the arrays that were replaced since the last step
    are read; arrays edited in place are already in the staging copy), runs the step, and writes the new
    state back as row views of one fresh array per quantity (a body's arrays are its own; the next step
    allocates new ones).  Bodies added, removed or replaced in an engine rebuild the batch; after changing a
    body's shape, mass, inertia, material or forces call :meth:`invalidate`.
    """

    def __init__(self, device="cuda", termination="merit", residual_tolerance=1e-6, residual_interval=1,
                 launch_shapes=None):
        self.device = device
        self.termination = termination
        self.residual_tolerance = residual_tolerance
        self.residual_interval = residual_interval
        self.launch_shapes = launch_shapes   # optional autotune setting (speed only; see rainbow_b200.autotune)
        self.log = []
        self.invalidate()

    def invalidate(self):
        """Forget the device copy: the next step rebuilds the batch from the engines."""
        self._world = None
        self._engines = None
        self._bodies = None

    def _build(self, engines):
        vecs = [np.array([float(getattr(e.params, f)) for f in W.PARAM_FIELDS]) for e in engines]
        for k, v in enumerate(vecs):
            if not np.array_equal(v, vecs[0]):
                f = W.PARAM_FIELDS[int(np.flatnonzero(v != vecs[0])[0])]
                raise ValueError("simulate_batch: engine %d differs from engine 0 in params.%s" % (k, f))
        for name in ("proximal_solver", "warm_start", "contact_ordering", "solver_precision"):
            vals = {repr(getattr(e.params, name, None)) for e in engines}
            if len(vals) > 1:
                raise ValueError("simulate_batch: the engines differ in params.%s" % name)
        arrays = [engine_io.scene_arrays(e) for e in engines]
        self._world = W.DeviceWorld(arrays, device=self.device,
                                    max_iterations=max(1, int(engines[0].params.max_iterations)))
        self._engines = list(engines)
        self._scene_bodies = [list(e.bodies.values()) for e in engines]
        self._bodies = [b for bl in self._scene_bodies for b in bl]
        self._x = np.concatenate([np.concatenate([a["body_r"], a["body_q"]], axis=1) for a in arrays])
        self._u = np.concatenate([np.concatenate([a["body_v"], a["body_w"]], axis=1) for a in arrays])
        self._rows = None   # the arrays last written into the bodies (r, q, v, w lists)
        self._factories = [_contact_factory(e) for e in engines]

    def _gather(self):
        """Host state of every body; False when the bodies no longer match the batch."""
        x, u, rows = self._x, self._u, self._rows
        k = 0
        for e, bl in zip(self._engines, self._scene_bodies):
            if len(e.bodies) != len(bl):
                return False
        if rows is None:
            for k, b in enumerate(self._bodies):
                x[k, :3] = b.r; x[k, 3:] = b.q; u[k, :3] = b.v; u[k, 3:] = b.w
            return True
        rl, ql, vl, wl = rows
        for e, bl in zip(self._engines, self._scene_bodies):
            for b, b2 in zip(e.bodies.values(), bl):
                if b is not b2:
                    return False
                if b.r is not rl[k]:
                    x[k, :3] = b.r
                if b.q is not ql[k]:
                    x[k, 3:] = b.q
                if b.v is not vl[k]:
                    u[k, :3] = b.v
                if b.w is not wl[k]:
                    u[k, 3:] = b.w
                k += 1
        return True

    def step(self, dt, engines, profiling_on=False):
        """Advance every engine by dt (steppers.py:47 SemiImplicitStepper.step, for all of them at once).
        An engine without bodies only gets an empty contact list, as the reference stepper gives it."""
        engines = list(engines)
        for e in engines:
            if not e.bodies:
                e.contact_points = []
        engines = [e for e in engines if e.bodies]
        if not engines:
            return
        if (self._world is None or len(engines) != len(self._engines)
                or any(a is not b for a, b in zip(engines, self._engines)) or not self._gather()):
            self._build(engines)
            self._gather()
        world = self._world
        t0 = time.perf_counter()
        rp = _step_params(engines[0].params, dt, self.termination, self.residual_tolerance, profiling_on,
                          self.residual_interval)
        if self.launch_shapes:
            from .autotune import DEFAULTS, apply
            apply(rp, {k: v for k, v in self.launch_shapes.items() if k in DEFAULTS})
        world.set_state(self._x, self._u)
        _check_status(world.step(rp))
        x, u = world.state()
        self._x, self._u = x, u
        rl, ql, vl, wl = list(x[:, :3]), list(x[:, 3:]), list(u[:, :3]), list(u[:, 3:])
        for b, r, q, v, w in zip(self._bodies, rl, ql, vl, wl):
            b.r = r
            b.q = q
            b.v = v
            b.w = w
        self._rows = (rl, ql, vl, wl)
        c = world.contacts()
        # the contacts come grouped by scene, in scene order: split them at the scenes' first bodies
        scene_of = np.searchsorted(world.scene_start, c["ids"][:, 0], side="right") - 1
        if np.any(np.diff(scene_of) < 0):
            raise NativeError("rb_step returned contacts out of scene order")
        ends = np.searchsorted(scene_of, np.arange(1, len(self._engines) + 1), side="left")
        k0 = 0
        for s, (e, bl) in enumerate(zip(self._engines, self._scene_bodies)):
            k1 = int(ends[s])
            e.contact_points = ContactPoints(bl, c["ids"][k0:k1], c["p"][k0:k1], c["n"][k0:k1], c["g"][k0:k1],
                                             self._factories[s], offset=int(world.scene_start[s]))
            k0 = k1
        if profiling_on:
            times = world.profile_times()
            self.log.append({"gpu_step_time": times[6], "stepper_time": time.perf_counter() - t0, "dt": dt,
                             "scenes": len(engines), "contact_points": int(len(c["g"]))})
