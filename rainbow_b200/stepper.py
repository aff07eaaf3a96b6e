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

    def __init__(self, bodies, ids, p, n, g, factory):
        self._bodies = bodies
        self._ids, self._p, self._n, self._g = ids, p, n, g
        self._factory = factory
        self._items = None

    def __len__(self):
        return len(self._g)

    def _build(self):
        if self._items is None:
            b = self._bodies
            self._items = [self._factory(b[int(i)], b[int(j)], self._p[k].copy(), self._n[k].copy(), float(self._g[k]))
                           for k, (i, j) in enumerate(self._ids)]
        return self._items

    def __getitem__(self, i):
        return self._build()[i]

    def __iter__(self):
        return iter(self._build())

    def __bool__(self):
        return len(self) > 0

    def arrays(self):
        """The contact set as arrays: body indices (SDF owner, mesh owner), positions, normals, gaps."""
        return self._ids, self._p, self._n, self._g


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
        scheme = getattr(engine.params, "proximal_solver", None) or "rigid_gauss_seidel"
        rp = W.make_rb_params(engine.params, dt=dt, scheme=scheme, termination=self.termination,
                              residual_tolerance=self.residual_tolerance, profiling=profiling_on,
                              warm_start=bool(getattr(engine.params, "warm_start", False)),
                              ordering=getattr(engine.params, "contact_ordering", None) or "serial",
                              precision=getattr(engine.params, "solver_precision", None) or "fp64")
        status = world.step(rp)
        if status & 16:
            raise RuntimeError("ContactPoint.init() was called with non-unit size normal")
        if status & 8:
            raise NativeError("the step produced a non-finite body state")
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
