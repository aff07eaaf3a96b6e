"""Generate golden fixtures by running the reference rigid-body time step itself.

Run in a container where the reference checkout is available (default ``/root/reference``, or the
``RAINBOW_REFERENCE`` environment variable)::

    python tests/golden/make_golden.py            # all fixtures
    python tests/golden/make_golden.py boxes8     # one fixture

Two reference dependencies are absent from this image and are replaced by the stand-ins under
``tests/golden/shims``: ``pyparsing`` (import-time only) and ``igl.signed_distance`` (shape set-up only; the grid
values it produces are stored in the fixture and read back by every consumer).  ``np.Inf`` (removed in NumPy 2)
is restored for ``rainbow/simulators/proximal_contact/solver_interface.py:41``.

Each fixture is an ``.npz`` holding the scene (shapes, bodies, forces, materials, parameters) in the reference's
body order, and per time step the contact set, the solver result, the solver statistics and the body state after
the step.  The scene builders follow the reference's own API calls (``api.py``) so that the shapes go through
``create_mesh`` / ``create_shape`` / ``connect_shape`` exactly as a user scene would.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("RAINBOW_REFERENCE", "/root/reference")
sys.path[:0] = [os.path.join(HERE, "shims"), REF]
np.Inf = np.inf  # NumPy 2 removed the alias the reference's proximal_contact package still uses

import rainbow.math.vector3 as V3  # noqa: E402
import rainbow.math.quaternion as Q  # noqa: E402
import rainbow.simulators.prox_rigid_bodies.api as API  # noqa: E402
import rainbow.simulators.prox_rigid_bodies.collision_detection as CD  # noqa: E402
import rainbow.simulators.prox_rigid_bodies.constraints as PROBLEMS  # noqa: E402
import rainbow.simulators.prox_rigid_bodies.state_storage as STORAGE  # noqa: E402
import rainbow.simulators.prox_rigid_bodies.types as TYPES  # noqa: E402
from rainbow.geometry.surface_mesh import create_box, create_sphere  # noqa: E402

PARAM_FIELDS = [
    "time_step", "max_iterations", "use_bounce", "use_pre_stabilization", "use_post_stabilization",
    "gap_reduction", "min_gap_value", "max_gap_value", "absolute_tolerance", "relative_tolerance",
    "nu_reduce", "nu_increase", "too_small_merit_change", "contact_optimization_max_iterations",
    "contact_optimization_tolerance", "bvh_chunk_size", "K", "envelope", "resolution",
]


# ---------------------------------------------------------------------------------------------------------------
# scene builders (reference API calls only)
# ---------------------------------------------------------------------------------------------------------------
def _ground(engine, size=(20.0, 1.0, 20.0), material=None):
    V, T = create_box(*size)
    API.create_shape(engine, "ground_shape", API.create_mesh(V, T))
    API.create_rigid_body(engine, "ground")
    API.connect_shape(engine, "ground", "ground_shape")
    API.set_position(engine, "ground", V3.make(0.0, -size[1] / 2.0, 0.0), True)
    API.set_orientation(engine, "ground", Q.identity(), True)
    API.set_body_type(engine, "ground", "fixed")
    API.set_mass_properties(engine, "ground", 1.0)
    if material is not None:
        API.set_body_material(engine, "ground", material)


def _unit_quaternion(rng):
    q = rng.uniform(-1.0, 1.0, 4)
    return q / np.linalg.norm(q)


def scene_box_lattice(n, spacing, jitter, res, seed, params=None, mu=0.5, two_materials=False):
    rng = np.random.default_rng(seed)
    engine = API.create_engine()
    engine.params.resolution = res
    for k, v in (params or {}).items():
        setattr(engine.params, k, v)
    API.create_surfaces_interaction(engine, "m", "m", 0.0, V3.make(mu, mu, mu))
    if two_materials:
        API.create_surfaces_interaction(engine, "m", "w", 0.0, V3.make(0.3, 0.3, 0.3))
        API.create_surfaces_interaction(engine, "w", "w", 0.0, V3.make(0.7, 0.7, 0.7))
    _ground(engine, material="m")
    V, T = create_box(1.0, 1.0, 1.0)
    API.create_shape(engine, "box", API.create_mesh(V, T))
    API.create_gravity_force(engine, "gravity", 9.81, V3.j())
    k = 0
    for i in range(n):
        for j in range(n):
            for l in range(n):
                name = "b%d" % k
                API.create_rigid_body(engine, name)
                API.connect_shape(engine, name, "box")
                r = V3.make(i * spacing, 0.5 + j * spacing, l * spacing) + rng.uniform(-jitter, jitter, 3)
                API.set_position(engine, name, r, True)
                API.set_orientation(engine, name, Q.identity(), True)
                API.set_mass_properties(engine, name, 1.0)
                API.connect_force(engine, name, "gravity")
                API.set_body_material(engine, name, "w" if (two_materials and k % 2) else "m")
                k += 1
    return engine


def scene_spheres(res, seed):
    rng = np.random.default_rng(seed)
    engine = API.create_engine()
    engine.params.resolution = res
    API.create_surfaces_interaction(engine, "m", "m", 0.0, V3.make(0.5, 0.5, 0.5))
    _ground(engine, material="m")
    V, T = create_sphere(0.5, 16, 16)
    API.create_shape(engine, "sphere", API.create_mesh(V, T))
    V, T = create_box(1.0, 1.0, 1.0)
    API.create_shape(engine, "box", API.create_mesh(V, T))
    API.create_gravity_force(engine, "gravity", 9.81, V3.j())
    positions = [(0.0, 0.47, 0.0), (0.98, 0.46, 0.0), (0.0, 1.42, 0.1), (0.5, 0.48, 0.97), (1.6, 0.5, 1.2)]
    for k, p in enumerate(positions):
        name = "s%d" % k
        API.create_rigid_body(engine, name)
        API.connect_shape(engine, name, "box" if k == 4 else "sphere")
        API.set_position(engine, name, V3.make(*p), True)
        API.set_orientation(engine, name, _unit_quaternion(rng), True)
        API.set_mass_properties(engine, name, 1000.0)
        API.connect_force(engine, name, "gravity")
        API.set_body_material(engine, name, "m")
    return engine


def scene_tower(height, res):
    engine = API.create_engine()
    engine.params.resolution = res
    engine.params.time_step = 0.005
    engine.params.max_iterations = 100
    engine.params.relative_tolerance = 1e-6
    API.create_surfaces_interaction(engine, "m", "m", 0.0, V3.make(0.6, 0.6, 0.6))
    _ground(engine, material="m")
    V, T = create_box(1.0, 1.0, 1.0)
    API.create_shape(engine, "box", API.create_mesh(V, T))
    API.create_gravity_force(engine, "gravity", 9.81, V3.j())
    for k in range(height):
        name = "t%d" % k
        API.create_rigid_body(engine, name)
        API.connect_shape(engine, name, "box")
        API.set_position(engine, name, V3.make(0.01 * k, 0.5 + k, 0.0), True)
        API.set_orientation(engine, name, Q.identity(), True)
        API.set_mass_properties(engine, name, 1.0 if k % 2 == 0 else 1000.0)
        API.connect_force(engine, name, "gravity")
        API.set_body_material(engine, name, "m")
    return engine


def scene_flags(res, seed):
    """Boxes with initial motion, damping, bounce and both stabilisation passes switched on."""
    rng = np.random.default_rng(seed)
    engine = API.create_engine()
    engine.params.resolution = res
    engine.params.use_bounce = True
    engine.params.use_pre_stabilization = True
    engine.params.use_post_stabilization = True
    API.create_surfaces_interaction(engine, "m", "m", 0.3, V3.make(0.4, 0.4, 0.4))
    _ground(engine, material="m")
    V, T = create_box(1.0, 0.6, 1.4)
    API.create_shape(engine, "slab", API.create_mesh(V, T))
    API.create_gravity_force(engine, "gravity", 9.81, V3.j())
    API.create_damping_force(engine, "damping", 0.01, 0.02)
    for k in range(4):
        name = "f%d" % k
        API.create_rigid_body(engine, name)
        API.connect_shape(engine, name, "slab")
        API.set_position(engine, name, V3.make(1.3 * (k % 2), 0.25 + 0.62 * (k // 2), 0.05 * k), True)
        API.set_orientation(engine, name, Q.Ry(0.1 * k), True)
        API.set_velocity(engine, name, rng.uniform(-0.5, 0.5, 3))
        API.set_spin(engine, name, rng.uniform(-1.0, 1.0, 3))
        API.set_mass_properties(engine, name, 2.0 + k)
        API.connect_force(engine, name, "gravity")
        API.connect_force(engine, name, "damping")
        API.set_body_material(engine, name, "m")
    return engine


def scene_hinge_chain(links, res, stab=False, tilt=0.0, ledge=False):
    """Cubes rotated 45 degrees about z, side by side along x, joined by hinges at the midpoints between
    neighbours; the first link is fixed and gravity pulls the rest down, so the chain swings about the hinge
    axes (world z, turned by `tilt` about x).  With `ledge` a fixed box under the outer links catches them,
    so hinges and contacts are solved together."""
    engine = API.create_engine()
    engine.params.resolution = res
    engine.params.use_pre_stabilization = stab
    API.create_surfaces_interaction(engine, "m", "m", 0.0, V3.make(0.4, 0.4, 0.4))
    V, T = create_box(1.0, 1.0, 1.0)
    API.create_shape(engine, "cube", API.create_mesh(V, T))
    API.create_gravity_force(engine, "gravity", 9.81, V3.j())
    diameter = np.sqrt(2.0)
    margin = 0.1 * diameter / 2.0
    names = []
    for k in range(links):
        name = "link%d" % k
        names.append(name)
        API.create_rigid_body(engine, name)
        API.connect_shape(engine, name, "cube")
        API.set_position(engine, name, V3.make(k * (diameter + margin), 0.0, 0.0), True)
        API.set_orientation(engine, name, Q.Rz(np.pi / 4), True)
        API.set_mass_properties(engine, name, 1.0)
        API.set_body_material(engine, name, "m")
        if k == 0:
            API.set_body_type(engine, name, "fixed")
        else:
            API.connect_force(engine, name, "gravity")
    if ledge:
        V, T = create_box(6.0, 1.0, 2.0)
        API.create_shape(engine, "ledge_shape", API.create_mesh(V, T))
        API.create_rigid_body(engine, "ledge")
        API.connect_shape(engine, "ledge", "ledge_shape")
        API.set_position(engine, "ledge", V3.make(2.0 * (diameter + margin) + 1.5, -1.3, 0.0), True)
        API.set_orientation(engine, "ledge", Q.identity(), True)
        API.set_body_type(engine, "ledge", "fixed")
        API.set_mass_properties(engine, "ledge", 1.0)
        API.set_body_material(engine, "ledge", "m")
    axis = Q.rotate(Q.Rx(tilt), V3.k())
    for k in range(links - 1):
        hinge = names[k] + "_" + names[k + 1]
        API.create_hinge(engine, hinge)
        o = (API.get_position(engine, names[k]) + API.get_position(engine, names[k + 1])) / 2.0
        API.set_hinge(engine=engine, hinge_name=hinge, parent_name=names[k], child_name=names[k + 1], origin=o,
                      axis=axis, mode="world")
    return engine


# ---------------------------------------------------------------------------------------------------------------
# serialisation
# ---------------------------------------------------------------------------------------------------------------
def scene_arrays(engine):
    out = {}
    shapes = list(engine.shapes.values())
    shape_index = {s.name: i for i, s in enumerate(shapes)}
    out["shape_names"] = np.array([s.name for s in shapes])
    v_off, t_off, g_off = [0], [0], [0]
    Vs, Ts, Gs, meta = [], [], [], []
    for s in shapes:
        Vs.append(np.asarray(s.mesh.V, dtype=np.float64))
        Ts.append(np.asarray(s.mesh.T, dtype=np.int32))
        vals = np.asarray(s.grid.values, dtype=np.float64).ravel()
        Gs.append(vals)
        v_off.append(v_off[-1] + len(Vs[-1]))
        t_off.append(t_off[-1] + len(Ts[-1]))
        g_off.append(g_off[-1] + len(vals))
        meta.append(np.concatenate([s.grid.min_coord, s.grid.max_coord, s.grid.spacing,
                                    [s.grid.I, s.grid.J, s.grid.K]]).astype(np.float64))
        out["shape_%s_mass" % s.name] = np.float64(s.mass)
    out["shape_V"] = np.concatenate(Vs)
    out["shape_T"] = np.concatenate(Ts)
    out["shape_grid"] = np.concatenate(Gs)
    out["shape_v_off"] = np.array(v_off, dtype=np.int64)
    out["shape_t_off"] = np.array(t_off, dtype=np.int64)
    out["shape_g_off"] = np.array(g_off, dtype=np.int64)
    out["shape_grid_meta"] = np.array(meta)

    bodies = list(engine.bodies.values())
    assert [b.idx for b in bodies] == list(range(len(bodies)))
    forces = list(engine.forces.values())
    force_index = {f.name: i for i, f in enumerate(forces)}
    materials = sorted({b.material for b in bodies} | {m for key in engine.surfaces_interactions.storage
                                                        for m in key})
    mat_index = {m: i for i, m in enumerate(materials)}
    out["body_names"] = np.array([b.name for b in bodies])
    out["body_shape"] = np.array([shape_index[b.shape.name] for b in bodies], dtype=np.int32)
    out["body_r"] = np.array([b.r for b in bodies], dtype=np.float64)
    out["body_q"] = np.array([b.q for b in bodies], dtype=np.float64)
    out["body_v"] = np.array([b.v for b in bodies], dtype=np.float64)
    out["body_w"] = np.array([b.w for b in bodies], dtype=np.float64)
    out["body_mass"] = np.array([b.mass for b in bodies], dtype=np.float64)
    out["body_inertia"] = np.array([b.inertia for b in bodies], dtype=np.float64)
    out["body_fixed"] = np.array([b.is_fixed for b in bodies], dtype=np.uint8)
    out["body_material"] = np.array([mat_index[b.material] for b in bodies], dtype=np.int32)
    out["body_forces"] = np.array([[force_index[f.name] in [force_index[g.name] for g in b.forces]
                                    for f in forces] for b in bodies], dtype=np.uint8).reshape(len(bodies),
                                                                                              len(forces))
    out["body_force_order"] = np.array([[force_index[f.name] for f in b.forces] + [-1] * (len(forces) - len(b.forces))
                                        for b in bodies], dtype=np.int32).reshape(len(bodies), len(forces))
    kinds, fparams = [], []
    for f in forces:
        if isinstance(f, TYPES.Gravity):
            kinds.append(0)
            fparams.append([f.g, f.up[0], f.up[1], f.up[2]])
        else:
            kinds.append(1)
            fparams.append([f.alpha, f.beta, 0.0, 0.0])
    out["force_kind"] = np.array(kinds, dtype=np.int32)
    out["force_params"] = np.array(fparams, dtype=np.float64).reshape(len(forces), 4)
    out["force_names"] = np.array([f.name for f in forces])
    out["material_names"] = np.array(materials)
    M = len(materials)
    mu = np.zeros((M, M, 3))
    eps = np.zeros((M, M))
    for a in range(M):
        for b in range(M):
            it = engine.surfaces_interactions.get_interaction(materials[a], materials[b])
            mu[a, b] = it.mu
            eps[a, b] = it.epsilon
    out["material_mu"] = mu
    out["material_epsilon"] = eps
    out["params"] = np.array([float(getattr(engine.params, f)) for f in PARAM_FIELDS])
    out["param_names"] = np.array(PARAM_FIELDS)
    hinges = sorted(engine.hinges.values(), key=lambda h: h.idx)
    assert [h.idx for h in hinges] == list(range(len(hinges)))
    out["hinge_bodies"] = np.array([[h.parent.idx, h.child.idx] for h in hinges], dtype=np.int32).reshape(-1, 2)
    out["hinge_frames"] = np.array([np.concatenate([h.arm_p, h.arm_c, h.axis_p, h.axis_c]) for h in hinges],
                                   dtype=np.float64).reshape(-1, 12)
    return out


class Recorder:
    """Captures the contact problem of each step through thin wrappers around reference methods."""

    def __init__(self):
        self.reset()
        orig_finalize = PROBLEMS.Contacts.finalize_solution
        orig_init = PROBLEMS.Contacts.initialize
        orig_copy = STORAGE.StateStorage.copy_from_engine
        rec = self

        def initialize(problem, dt, state, engine):
            orig_init(problem, dt, state, engine)
            rec.b = problem.b.copy()
            rec.diag = problem.diag.copy()
            rec.mu = problem.mu.copy()

        def finalize(problem):
            out = orig_finalize(problem)
            rec.sol = problem.sol.copy()
            return out

        def copy_from_engine(state, engine):
            orig_copy(state, engine)
            if rec.delta_u_ext is None:
                rec.delta_u_ext = state.delta_u_ext.copy()

        orig_h_init = PROBLEMS.Hinges.initialize
        orig_h_finalize = PROBLEMS.Hinges.finalize_solution

        def h_initialize(problem, dt, state, engine):
            orig_h_init(problem, dt, state, engine)
            rec.hinge_b = problem.b.copy()
            rec.hinge_diag = problem.diag.copy()

        def h_finalize(problem):
            out = orig_h_finalize(problem)
            rec.hinge_sol = problem.sol.copy()
            return out

        PROBLEMS.Contacts.initialize = initialize
        PROBLEMS.Contacts.finalize_solution = finalize
        PROBLEMS.Hinges.initialize = h_initialize
        PROBLEMS.Hinges.finalize_solution = h_finalize
        STORAGE.StateStorage.copy_from_engine = copy_from_engine

    def reset(self):
        self.b = self.diag = self.mu = self.sol = self.delta_u_ext = None
        self.hinge_b = self.hinge_diag = self.hinge_sol = None


def run_fixture(name, engine, steps):
    rec = RECORDER
    data = scene_arrays(engine)
    per_step = {k: [] for k in ["contacts_ids", "contacts_p", "contacts_n", "contacts_g", "b", "diag", "sol",
                                "iterations", "exitcode", "residuals", "x", "u", "delta_u_ext", "dt",
                                "post_iterations", "post_exitcode", "hinge_b", "hinge_diag", "hinge_sol"]}
    t0 = time.perf_counter()
    for s in range(steps):
        rec.reset()
        dt = engine.params.time_step
        engine.stepper.step(dt, engine, True)
        log = engine.stepper.log[-1]
        cps = engine.contact_points
        per_step["contacts_ids"].append(np.array([[c.bodyA.idx, c.bodyB.idx] for c in cps], dtype=np.int32)
                                        .reshape(-1, 2))
        per_step["contacts_p"].append(np.array([c.p for c in cps], dtype=np.float64).reshape(-1, 3))
        per_step["contacts_n"].append(np.array([c.n for c in cps], dtype=np.float64).reshape(-1, 3))
        per_step["contacts_g"].append(np.array([c.g for c in cps], dtype=np.float64).reshape(-1))
        K = len(cps)
        per_step["b"].append(rec.b if K else np.zeros(0))
        per_step["diag"].append(rec.diag if K else np.zeros(0))
        per_step["sol"].append(rec.sol if K else np.zeros(0))
        H = len(engine.hinges)
        per_step["hinge_b"].append(rec.hinge_b if H else np.zeros(0))
        per_step["hinge_diag"].append(rec.hinge_diag if H else np.zeros(0))
        per_step["hinge_sol"].append(rec.hinge_sol if H else np.zeros(0))
        per_step["iterations"].append(log.get("iterations", -1))
        per_step["exitcode"].append(log.get("exitcode", -1))
        per_step["residuals"].append(np.asarray(log.get("residuals", np.zeros(0)), dtype=np.float64))
        per_step["post_iterations"].append(log.get("post_stabilization_iterations", -1))
        per_step["post_exitcode"].append(log.get("post_stabilization_exitcode", -1))
        per_step["x"].append(np.concatenate([np.concatenate([b.r, b.q]) for b in engine.bodies.values()]))
        per_step["u"].append(np.concatenate([np.concatenate([b.v, b.w]) for b in engine.bodies.values()]))
        per_step["delta_u_ext"].append(rec.delta_u_ext)
        per_step["dt"].append(dt)
        print("  %s step %d: %d contacts, iterations %s exit %s (%.1fs)" % (
            name, s, K, log.get("iterations"), log.get("exitcode"), time.perf_counter() - t0), flush=True)
    for k, v in per_step.items():
        if k in ("iterations", "exitcode", "post_iterations", "post_exitcode"):
            data["step_" + k] = np.array(v, dtype=np.int32)
        elif k == "dt":
            data["step_dt"] = np.array(v, dtype=np.float64)
        elif k in ("x", "u", "delta_u_ext"):
            data["step_" + k] = np.array(v)
        else:
            lens = np.array([len(a) for a in v], dtype=np.int64)
            data["step_%s_len" % k] = lens
            data["step_" + k] = np.concatenate(v) if sum(lens) else np.zeros((0,) + v[0].shape[1:])
    data["steps"] = np.int64(steps)
    return data


def solver_fixture(engine, name):
    """One contact problem from the scene's current state, solved by every proximal_contact scheme."""
    import rainbow.simulators.proximal_contact.prox_solvers as PS
    state = STORAGE.StateStorage()
    state.copy_from_engine(engine)
    CD.run_collision_detection(engine, {}, False)
    problem = PROBLEMS.Contacts()
    problem.initialize(engine.params.time_step, state, engine)
    data = scene_arrays(engine)
    data["contacts_ids"] = np.array([[c.bodyA.idx, c.bodyB.idx] for c in engine.contact_points], dtype=np.int32)
    data["contacts_p"] = np.array([c.p for c in engine.contact_points])
    data["contacts_n"] = np.array([c.n for c in engine.contact_points])
    data["contacts_g"] = np.array([c.g for c in engine.contact_points])
    data["b"] = problem.b
    data["mu"] = problem.mu
    data["diag"] = problem.diag
    for scheme in ["gauss_seidel", "parallel_jacobi", "parallel_jacboi_hybrid"]:
        stats = {}
        sol, stats = PS.solve(problem.J, problem.WJT, problem.b, problem.mu, PS.prox_sphere, engine, stats, True,
                              scheme=scheme)
        key = scheme.replace("parallel_jacboi_hybrid", "parallel_jacobi_hybrid")
        data["sol_" + key] = np.asarray(sol)
        data["iterations_" + key] = np.int64(stats[scheme + "_iterations"])
        data["exitcode_" + key] = np.int64(stats[scheme + "_exitcode"])
        data["residuals_" + key] = np.asarray(stats[scheme + "_residuals"])
        print("  %s %s: iterations %s exit %s" % (name, scheme, stats[scheme + "_iterations"],
                                                  stats[scheme + "_exitcode"]), flush=True)
    return data


FIXTURES = {
    "boxes8": lambda: (scene_box_lattice(2, 1.05, 0.02, 16, seed=1, two_materials=True), 12),
    "c1_boxes64": lambda: (scene_box_lattice(4, 1.05, 0.02, 32, seed=0,
                                             params=dict(max_iterations=100, relative_tolerance=1e-6)), 4),
    "spheres": lambda: (scene_spheres(16, seed=3), 8),
    "tower6": lambda: (scene_tower(6, 16), 20),
    "flags": lambda: (scene_flags(16, seed=5), 10),
    "hinges": lambda: (scene_hinge_chain(5, 16, ledge=True), 30),
    "hinges_stab": lambda: (scene_hinge_chain(4, 16, stab=True, tilt=0.3), 25),
}


def main(names):
    out_dir = HERE
    for name in names:
        if name == "solvers":
            engine = scene_box_lattice(2, 1.05, 0.02, 16, seed=2, params=dict(max_iterations=60,
                                                                              relative_tolerance=1e-6,
                                                                              absolute_tolerance=1e-9))
            for _ in range(3):
                engine.stepper.step(engine.params.time_step, engine, False)
            data = solver_fixture(engine, name)
        else:
            engine, steps = FIXTURES[name]()
            data = run_fixture(name, engine, steps)
        path = os.path.join(out_dir, name + ".npz")
        np.savez_compressed(path, **data)
        print("wrote %s (%.0f KB)" % (path, os.path.getsize(path) / 1024.0), flush=True)


RECORDER = Recorder()

if __name__ == "__main__":
    main(sys.argv[1:] or list(FIXTURES) + ["solvers"])
