"""Synthetic benchmark scenes, built with the reference-compatible API (seeded, no external data).

* ``box_lattice``  -- unit boxes in an n x n x n lattice with jittered positions on a fixed ground box
                       (64 boxes at spacing 1.05, SDF resolution 32: the reference's CPU-sized case);
* ``mixed_lattice`` -- n^3 bodies alternating unit boxes and r = 0.5 spheres (16 x 16 sweep), uniformly random
                       orientations, density 1000, dropped from spacing 1.2 onto a ground box;
* ``box_tower``    -- a column of unit boxes with alternating densities (mass ratio 1e3);
* ``random_scene`` -- a small scene of random boxes and spheres (random sizes, random friction) on a ground box,
                       the unit of the batched and served workloads.
Each returns an engine; :func:`rainbow_b200.engine_io.scene_arrays` turns it into device-ready arrays.
"""
import numpy as np

from . import api as API


def _ground(engine, size, material="m"):
    V, T = API.create_box(*size)
    API.create_shape(engine, "ground_shape", API.create_mesh(V, T))
    API.create_rigid_body(engine, "ground")
    API.connect_shape(engine, "ground", "ground_shape")
    API.set_position(engine, "ground", np.array([0.0, -size[1] / 2.0, 0.0]), True)
    API.set_orientation(engine, "ground", np.array([1.0, 0.0, 0.0, 0.0]), True)
    API.set_body_type(engine, "ground", "fixed")
    API.set_mass_properties(engine, "ground", 1.0)
    API.set_body_material(engine, "ground", material)


def _random_unit_quaternion(rng):
    q = rng.normal(size=4)
    return q / np.linalg.norm(q)


def box_lattice(n=4, spacing=1.05, jitter=0.02, resolution=32, seed=0, mu=0.5, device="cuda"):
    rng = np.random.default_rng(seed)
    engine = API.create_engine(device)
    engine.params.resolution = resolution
    engine.params.max_iterations = 100
    engine.params.relative_tolerance = 1e-6
    API.create_surfaces_interaction(engine, "m", "m", 0.0, np.array([mu, mu, mu]))
    _ground(engine, (20.0, 1.0, 20.0))
    V, T = API.create_box(1.0, 1.0, 1.0)
    API.create_shape(engine, "box", API.create_mesh(V, T))
    API.create_gravity_force(engine, "gravity", 9.81, np.array([0.0, 1.0, 0.0]))
    k = 0
    for i in range(n):
        for j in range(n):
            for l in range(n):
                name = "b%d" % k
                API.create_rigid_body(engine, name)
                API.connect_shape(engine, name, "box")
                r = np.array([i * spacing, 0.5 + j * spacing, l * spacing]) + rng.uniform(-jitter, jitter, 3)
                API.set_position(engine, name, r, True)
                API.set_orientation(engine, name, np.array([1.0, 0.0, 0.0, 0.0]), True)
                API.set_mass_properties(engine, name, 1.0)
                API.connect_force(engine, name, "gravity")
                API.set_body_material(engine, name, "m")
                k += 1
    return engine


def mixed_lattice(n=16, spacing=1.2, resolution=64, seed=0, mu=0.5, device="cuda"):
    rng = np.random.default_rng(seed)
    engine = API.create_engine(device)
    engine.params.resolution = resolution
    engine.params.max_iterations = 100
    engine.params.relative_tolerance = 1e-6
    API.create_surfaces_interaction(engine, "m", "m", 0.0, np.array([mu, mu, mu]))
    extent = n * spacing + 4.0
    _ground(engine, (extent, 1.0, extent))
    V, T = API.create_box(1.0, 1.0, 1.0)
    API.create_shape(engine, "box", API.create_mesh(V, T))
    V, T = API.create_sphere(0.5, 16, 16)
    API.create_shape(engine, "sphere", API.create_mesh(V, T))
    API.create_gravity_force(engine, "gravity", 9.81, np.array([0.0, 1.0, 0.0]))
    off = -0.5 * (n - 1) * spacing
    k = 0
    for i in range(n):
        for j in range(n):
            for l in range(n):
                name = "b%d" % k
                API.create_rigid_body(engine, name)
                API.connect_shape(engine, name, "box" if k % 2 == 0 else "sphere")
                r = np.array([off + i * spacing, 0.6 + j * spacing, off + l * spacing])
                API.set_position(engine, name, r, True)
                API.set_orientation(engine, name, _random_unit_quaternion(rng), True)
                API.set_mass_properties(engine, name, 1000.0)
                API.connect_force(engine, name, "gravity")
                API.set_body_material(engine, name, "m")
                k += 1
    return engine


def box_tower(height=32, resolution=32, mu=0.6, dt=0.005, device="cuda"):
    engine = API.create_engine(device)
    engine.params.resolution = resolution
    engine.params.time_step = dt
    engine.params.max_iterations = 100
    engine.params.relative_tolerance = 1e-6
    API.create_surfaces_interaction(engine, "m", "m", 0.0, np.array([mu, mu, mu]))
    _ground(engine, (20.0, 1.0, 20.0))
    V, T = API.create_box(1.0, 1.0, 1.0)
    API.create_shape(engine, "box", API.create_mesh(V, T))
    API.create_gravity_force(engine, "gravity", 9.81, np.array([0.0, 1.0, 0.0]))
    for k in range(height):
        name = "t%d" % k
        API.create_rigid_body(engine, name)
        API.connect_shape(engine, name, "box")
        API.set_position(engine, name, np.array([0.0, 0.5 + k, 0.0]), True)
        API.set_orientation(engine, name, np.array([1.0, 0.0, 0.0, 0.0]), True)
        API.set_mass_properties(engine, name, 1.0 if k % 2 == 0 else 1000.0)
        API.connect_force(engine, name, "gravity")
        API.set_body_material(engine, name, "m")
    return engine


def random_scene(n_bodies, rng, resolution=32, device="cuda", size_pool=None):
    """Random boxes (side U(0.5, 2)) and spheres (radius U(0.25, 1)) dropped on a ground box; mu U(0.2, 0.8).

    ``size_pool``: optional number of distinct sizes per shape kind drawn once per scene (fewer SDFs)."""
    engine = API.create_engine(device)
    engine.params.resolution = resolution
    engine.params.max_iterations = 100
    engine.params.relative_tolerance = 1e-6
    mu = rng.uniform(0.2, 0.8)
    API.create_surfaces_interaction(engine, "m", "m", 0.0, np.array([mu, mu, mu]))
    side = int(np.ceil(n_bodies ** (1.0 / 3.0)))
    spacing = 2.3
    _ground(engine, (side * spacing + 4.0, 1.0, side * spacing + 4.0))
    API.create_gravity_force(engine, "gravity", 9.81, np.array([0.0, 1.0, 0.0]))
    kinds = rng.integers(0, 2, n_bodies)
    sizes = np.where(kinds == 0, rng.uniform(0.5, 2.0, n_bodies), rng.uniform(0.25, 1.0, n_bodies))
    if size_pool:
        pool = {0: rng.uniform(0.5, 2.0, size_pool), 1: rng.uniform(0.25, 1.0, size_pool)}
        sizes = np.array([pool[k][rng.integers(0, size_pool)] for k in kinds])
    made = {}
    off = -0.5 * (side - 1) * spacing
    for b in range(n_bodies):
        key = (int(kinds[b]), float(sizes[b]))
        if key not in made:
            name = "shape%d" % len(made)
            V, T = API.create_box(sizes[b], sizes[b], sizes[b]) if kinds[b] == 0 else API.create_sphere(sizes[b], 16, 16)
            API.create_shape(engine, name, API.create_mesh(V, T))
            made[key] = name
        i, j, l = b % side, (b // side) % side, b // (side * side)
        name = "b%d" % b
        API.create_rigid_body(engine, name)
        API.connect_shape(engine, name, made[key])
        API.set_position(engine, name, np.array([off + i * spacing, 1.2 + j * spacing, off + l * spacing]), True)
        API.set_orientation(engine, name, _random_unit_quaternion(rng), True)
        API.set_mass_properties(engine, name, 1000.0)
        API.connect_force(engine, name, "gravity")
        API.set_body_material(engine, name, "m")
    return engine


# ------------------------------------------------------------------------------------------------------------
# batched workload: many independent scenes built directly as arrays (no per-body Python objects)
# ------------------------------------------------------------------------------------------------------------
def _shape_arrays(V, T, resolution, envelope, device):
    """One shape through the reference's set-up chain (create_mesh, create_shape): body-frame mesh, mass
    properties at unit density, frame transform and signed distance grid."""
    from . import geometry as GEO
    mesh = GEO.create_mesh(V, T)
    mass, com, I = GEO.compute_mass_properties(mesh.V, mesh.T, 1.0)
    r, q, inertia = GEO.xform_model_2_body_space(mass, com, I)
    Vb = GEO.quat_rotate_array(GEO.quat_conj(q), mesh.V - r)
    max_length = (Vb.max(axis=0) - Vb.min(axis=0)).max()
    grid = GEO.create_signed_distance(Vb, mesh.T, resolution, resolution, resolution,
                                      max(max_length * 0.1, envelope * 2), device=device)
    return dict(V=Vb, T=np.asarray(mesh.T, np.int32), grid=grid.values, meta=grid.meta(), mass=mass,
                inertia=np.asarray(inertia, np.float64), r=np.asarray(r, np.float64), q=np.asarray(q, np.float64))


def batch_arrays(n_scenes=1024, seed=0, pool=64, body_range=(8, 256), resolution=32, device="cuda", ground=24.0):
    """``n_scenes`` independent scenes: body count log-uniform in body_range, random boxes (side U(0.5, 2))
    and spheres (radius U(0.25, 1), 16 x 16 sweep) with uniformly random orientations, density 1000, dropped
    onto a fixed ground box (ground x 1 x ground); friction mu U(0.2, 0.8) per scene; dt 0.01.

    With ``pool`` set, shape sizes are drawn from a pool of ``pool`` boxes and ``pool`` spheres shared by all
    scenes, so the signed distance grids are built once per pool entry; with ``pool=None`` every body gets a
    shape and a grid of its own (:func:`batch_arrays_per_body`).  Returns the list of per-scene arrays
    (sharing the pool's shape arrays by ``shape_key``) and the Parameters mapping used."""
    if pool is None:
        return batch_arrays_per_body(n_scenes, seed, body_range, resolution, device, ground)
    from . import geometry as GEO
    from .types import Parameters
    rng = np.random.default_rng(seed)
    params = Parameters()
    params.resolution = resolution
    params.max_iterations = 100
    params.relative_tolerance = 1e-6
    shapes = [_shape_arrays(*GEO.create_box(ground, 1.0, ground), resolution, params.envelope, device)]
    kind = [2]
    for s in rng.uniform(0.5, 2.0, pool):
        shapes.append(_shape_arrays(*GEO.create_box(s, s, s), resolution, params.envelope, device))
        kind.append(0)
    for rad in rng.uniform(0.25, 1.0, pool):
        shapes.append(_shape_arrays(*GEO.create_sphere(rad, 16, 16), resolution, params.envelope, device))
        kind.append(1)
    common = {
        "shape_V": np.concatenate([s["V"] for s in shapes]),
        "shape_T": np.concatenate([s["T"] for s in shapes]),
        "shape_grid": np.concatenate([s["grid"] for s in shapes]),
        "shape_v_off": np.concatenate([[0], np.cumsum([len(s["V"]) for s in shapes])]).astype(np.int64),
        "shape_t_off": np.concatenate([[0], np.cumsum([len(s["T"]) for s in shapes])]).astype(np.int64),
        "shape_g_off": np.concatenate([[0], np.cumsum([len(s["grid"]) for s in shapes])]).astype(np.int64),
        "shape_grid_meta": np.array([s["meta"] for s in shapes]),
        "shape_key": np.array(["pool%d:%d:%d:%g:%d" % (seed, pool, resolution, ground, k) for k in range(len(shapes))]),
    }
    from .world import PARAM_FIELDS
    pvec = np.array([float(getattr(params, f)) for f in PARAM_FIELDS])
    out = []
    lo, hi = np.log(body_range[0]), np.log(body_range[1])
    for _ in range(n_scenes):
        n = int(round(np.exp(rng.uniform(lo, hi))))
        side = int(np.ceil(n ** (1.0 / 3.0)))
        spacing = 2.3
        off = -0.5 * (side - 1) * spacing
        idx = rng.integers(1, 2 * pool + 1, n)
        body_shape = np.concatenate([[0], idx]).astype(np.int32)
        pos = np.zeros((n + 1, 3))
        quat = np.zeros((n + 1, 4))
        # ground: model frame at (0, -0.5, 0), identity orientation
        g = shapes[0]
        quat[0] = GEO.quat_prod(np.array([1.0, 0.0, 0.0, 0.0]), g["q"])
        pos[0] = GEO.quat_rotate(np.array([1.0, 0.0, 0.0, 0.0]), g["r"]) + np.array([0.0, -0.5, 0.0])
        for b in range(n):
            i, j, l = b % side, (b // side) % side, b // (side * side)
            qu = rng.normal(size=4)
            qu /= np.linalg.norm(qu)
            sh = shapes[idx[b]]
            quat[b + 1] = GEO.quat_prod(qu, sh["q"])
            pos[b + 1] = GEO.quat_rotate(qu, sh["r"]) + np.array([off + i * spacing, 1.2 + j * spacing, off + l * spacing])
        mass = np.array([shapes[k]["mass"] for k in body_shape]) * 1000.0
        inertia = np.array([shapes[k]["inertia"] for k in body_shape]) * 1000.0
        fixed = np.zeros(n + 1, np.uint8)
        fixed[0] = 1
        mu = rng.uniform(0.2, 0.8)
        scene = dict(common)
        scene.update({
            "body_shape": body_shape, "body_r": pos, "body_q": quat, "body_v": np.zeros((n + 1, 3)),
            "body_w": np.zeros((n + 1, 3)), "body_mass": mass, "body_inertia": inertia, "body_fixed": fixed,
            "body_material": np.zeros(n + 1, np.int32),
            "body_force_order": np.concatenate([[[-1]], np.zeros((n, 1), np.int32)]).astype(np.int32),
            "force_kind": np.array([0], np.int32), "force_params": np.array([[9.81, 0.0, 1.0, 0.0]]),
            "material_mu": np.full((1, 1, 3), mu), "material_epsilon": np.zeros((1, 1)), "params": pvec,
        })
        out.append(scene)
    return out, params


def _per_body_draws(rng, lo, hi):
    """One scene's draws of the per-body workload: body count, kinds, sizes, orientations, friction."""
    n = int(round(np.exp(rng.uniform(lo, hi))))
    kinds = rng.integers(0, 2, n)
    sizes = np.where(kinds == 0, rng.uniform(0.5, 2.0, n), rng.uniform(0.25, 1.0, n))
    quats = rng.normal(size=(n, 4))
    quats /= np.linalg.norm(quats, axis=1, keepdims=True)
    mu = rng.uniform(0.2, 0.8)
    return n, kinds, sizes, quats, mu


def per_body_counts(n_scenes=1024, seed=0, body_range=(8, 256)):
    """Bodies (ground included) of each scene of :func:`batch_arrays_per_body`, without building anything."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(body_range[0]), np.log(body_range[1])
    return [_per_body_draws(rng, lo, hi)[0] + 1 for _ in range(n_scenes)]


def batch_arrays_per_body(n_scenes=1024, seed=0, body_range=(8, 256), resolution=32, device="cuda", ground=24.0,
                          select=None):
    """The batched workload with a shape and signed distance grid of its own for every body: body counts,
    kinds (box or sphere), sizes (box side U(0.5, 2), sphere radius U(0.25, 1)), orientations and friction
    drawn per scene from ``seed``.  A body's shape is the unit box (side 1) or unit sphere (radius 1, 16 x 16
    sweep), taken through the reference's set-up chain once, scaled by the body's size (body-frame vertices
    and centre of mass by s, mass by s^3, inertia by s^5); its grid (grid3.py:320: bounding box grown by
    max(0.1 x longest side, 2 x envelope), ``resolution`` nodes per axis) is computed on the device from its
    own mesh.  All grids live in one device tensor; each scene's ``shape_grid`` is a view of it (its ground's
    grid first, then its bodies' in body order), so nothing of the ~18.8 GB (73k grids of 32^3 doubles) passes
    through host memory.  ``select``: build only these scene indices (every scene's draws are still made, so a
    scene is the same whichever others are built; ranks of a multi-GPU run build their own share)."""
    from . import geometry as GEO
    from .types import Grid, Parameters
    from .world import PARAM_FIELDS
    rng = np.random.default_rng(seed)
    params = Parameters()
    params.resolution = resolution
    params.max_iterations = 100
    params.relative_tolerance = 1e-6
    env = float(params.envelope)
    unit = [_shape_arrays(*GEO.create_box(1.0, 1.0, 1.0), resolution, env, device),
            _shape_arrays(*GEO.create_sphere(1.0, 16, 16), resolution, env, device)]
    g = _shape_arrays(*GEO.create_box(ground, 1.0, ground), resolution, env, device)
    unit_len = [float((u["V"].max(axis=0) - u["V"].min(axis=0)).max()) for u in unit]
    pvec = np.array([float(getattr(params, f)) for f in PARAM_FIELDS])
    lo, hi = np.log(body_range[0]), np.log(body_range[1])
    V_list, T_list, metas, plans = [], [], [], []
    wanted = set(range(n_scenes)) if select is None else set(int(i) for i in select)
    for si in range(n_scenes):
        n, kinds, sizes, quats, mu = _per_body_draws(rng, lo, hi)
        if si not in wanted:
            continue
        V_list.append(g["V"]); T_list.append(g["T"]); metas.append(g["meta"])
        for b in range(n):
            u, sz = unit[kinds[b]], float(sizes[b])
            Vb = u["V"] * sz
            boundary = max(0.1 * unit_len[kinds[b]] * sz, 2.0 * env)
            V_list.append(Vb)
            T_list.append(u["T"])
            metas.append(Grid(Vb.min(axis=0) - boundary, Vb.max(axis=0) + boundary, resolution, resolution,
                              resolution).meta())
        plans.append((si, n, kinds, sizes, quats, mu))
    values, g_off = GEO.signed_distance_grids(V_list, T_list, metas, device=device)
    out = []
    shape0 = 0
    for si, n, kinds, sizes, quats, mu in plans:
        sh = slice(shape0, shape0 + n + 1)
        Vs, Ts = V_list[sh], T_list[sh]
        side = int(np.ceil(n ** (1.0 / 3.0)))
        spacing = 2.3
        off = -0.5 * (side - 1) * spacing
        pos = np.zeros((n + 1, 3))
        quat = np.zeros((n + 1, 4))
        quat[0] = GEO.quat_prod(np.array([1.0, 0.0, 0.0, 0.0]), g["q"])
        pos[0] = GEO.quat_rotate(np.array([1.0, 0.0, 0.0, 0.0]), g["r"]) + np.array([0.0, -0.5, 0.0])
        mass = np.zeros(n + 1)
        inertia = np.zeros((n + 1, 3))
        mass[0], inertia[0] = g["mass"] * 1000.0, g["inertia"] * 1000.0
        for b in range(n):
            i, j, l = b % side, (b // side) % side, b // (side * side)
            u, sz = unit[kinds[b]], float(sizes[b])
            quat[b + 1] = GEO.quat_prod(quats[b], u["q"])
            pos[b + 1] = GEO.quat_rotate(quats[b], u["r"] * sz) + np.array([off + i * spacing, 1.2 + j * spacing,
                                                                         off + l * spacing])
            mass[b + 1] = u["mass"] * sz ** 3 * 1000.0
            inertia[b + 1] = u["inertia"] * sz ** 5 * 1000.0
        fixed = np.zeros(n + 1, np.uint8)
        fixed[0] = 1
        g0, g1 = int(g_off[shape0]), int(g_off[shape0 + n + 1])
        out.append({
            "shape_V": np.concatenate(Vs), "shape_T": np.concatenate(Ts),
            "shape_grid": values[g0:g1],
            "shape_v_off": np.concatenate([[0], np.cumsum([len(v) for v in Vs])]).astype(np.int64),
            "shape_t_off": np.concatenate([[0], np.cumsum([len(t) for t in Ts])]).astype(np.int64),
            "shape_g_off": (g_off[shape0:shape0 + n + 2] - g_off[shape0]).astype(np.int64),
            "shape_grid_meta": np.array(metas[sh]),
            "shape_key": np.array(["perbody%d:%d:%g:ground" % (seed, resolution, ground)] +
                                  ["perbody%d:%d:%d:%d" % (seed, resolution, si, b) for b in range(n)]),
            "body_shape": np.arange(n + 1, dtype=np.int32), "body_r": pos, "body_q": quat,
            "body_v": np.zeros((n + 1, 3)), "body_w": np.zeros((n + 1, 3)), "body_mass": mass,
            "body_inertia": inertia, "body_fixed": fixed, "body_material": np.zeros(n + 1, np.int32),
            "body_force_order": np.concatenate([[[-1]], np.zeros((n, 1), np.int32)]).astype(np.int32),
            "force_kind": np.array([0], np.int32), "force_params": np.array([[9.81, 0.0, 1.0, 0.0]]),
            "material_mu": np.full((1, 1, 3), mu), "material_epsilon": np.zeros((1, 1)), "params": pvec,
        })
        shape0 += n + 1
    return out, params
