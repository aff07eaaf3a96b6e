"""Host-side logic that needs no GPU: scene packing, engine conversion, and reading the reference's own
engine objects (the drop-in read path) when the reference checkout is present."""
import os
import sys

import numpy as np
import pytest

from conftest import FIXTURES, ROOT, load_fixture

from rainbow_b200 import engine_io, world as W

SCENE_KEYS = ["shape_V", "shape_T", "shape_grid", "shape_v_off", "shape_t_off", "shape_g_off", "shape_grid_meta",
              "body_shape", "body_r", "body_q", "body_v", "body_w", "body_mass", "body_inertia", "body_fixed",
              "body_material", "body_force_order", "force_kind", "force_params", "material_mu", "material_epsilon",
              "params"]


@pytest.mark.parametrize("name", FIXTURES)
def test_engine_round_trip(name):
    d = load_fixture(name)
    engine = engine_from = engine_io.engine_from_arrays(d)
    a = engine_io.scene_arrays(engine_from)
    for k in SCENE_KEYS:
        np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(d[k]).reshape(np.asarray(a[k]).shape), err_msg=k)
    x, u = engine_io.body_state(engine)
    np.testing.assert_array_equal(x[:, :3], d["body_r"])
    np.testing.assert_array_equal(u[:, 3:], d["body_w"])


def test_pack_two_scenes():
    a, b = load_fixture("boxes8"), load_fixture("spheres")
    P = W.pack_scenes([a, b])
    na, nb = len(a["body_mass"]), len(b["body_mass"])
    assert P["n_bodies"] == na + nb
    np.testing.assert_array_equal(P["scene_start"], [0, na, na + nb])
    sa = len(a["shape_v_off"]) - 1
    np.testing.assert_array_equal(P["body_shape"][na:], b["body_shape"] + sa)
    # topology prefix sums follow the body -> shape map
    v_cnt = np.diff(P["shape_v_off"])
    t_cnt = np.diff(P["shape_t_off"])
    np.testing.assert_array_equal(np.diff(P["body_v0"]), v_cnt[P["body_shape"]])
    np.testing.assert_array_equal(np.diff(P["body_t0"]), t_cnt[P["body_shape"]])
    np.testing.assert_array_equal(np.diff(P["body_c0"]), (t_cnt[P["body_shape"]] + 31) // 32)
    assert len(P["vert_body"]) == P["body_v0"][-1] and P["vert_body"][-1] == na + nb - 1
    # per-scene material tables and force ranges
    Ma, Mb = len(a["material_epsilon"]), len(b["material_epsilon"])
    np.testing.assert_array_equal(P["scene_material_offset"], [0, Ma * Ma])
    np.testing.assert_array_equal(P["scene_material_count"], [Ma, Mb])
    np.testing.assert_array_equal(P["scene_force_start"], [0, len(a["force_kind"]), len(a["force_kind"]) + len(b["force_kind"])])
    # state layout of state_storage.py: 7 (r, q) and 6 (v, w) per body
    np.testing.assert_array_equal(P["x"].reshape(-1, 7)[na:, 3:], b["body_q"])
    np.testing.assert_array_equal(P["u"].reshape(-1, 6)[:na, :3], a["body_v"])


def test_hinges_round_trip_through_engines_and_packing():
    """Hinge joints (types.py:304) survive engine -> arrays -> engine, and packing rebases their body indices
    onto each scene's body range."""
    from rainbow_b200 import world as W
    d = load_fixture("hinges")
    back = engine_io.scene_arrays(engine_io.engine_from_arrays(d))
    np.testing.assert_array_equal(back["hinge_bodies"], d["hinge_bodies"])
    np.testing.assert_array_equal(back["hinge_frames"], d["hinge_frames"])
    e = load_fixture("hinges_stab")
    P = W.pack_scenes([load_fixture("boxes8"), d, e])
    nb0 = len(load_fixture("boxes8")["body_mass"])
    nb1 = len(d["body_mass"])
    H1, H2 = len(d["hinge_bodies"]), len(e["hinge_bodies"])
    np.testing.assert_array_equal(P["scene_hinge_start"], [0, 0, H1, H1 + H2])
    hb = P["hinge_bodies"].reshape(-1, 2)
    np.testing.assert_array_equal(hb[:H1], d["hinge_bodies"] + nb0)
    np.testing.assert_array_equal(hb[H1:], e["hinge_bodies"] + nb0 + nb1)


def test_massless_body_is_rejected():
    engine = engine_io.engine_from_arrays(load_fixture("boxes8"))
    list(engine.bodies.values())[1].mass = 0.0
    with pytest.raises(ValueError):
        engine_io.scene_arrays(engine)


REFERENCE = os.environ.get("RAINBOW_REFERENCE", "/root/reference")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REFERENCE, "rainbow")), reason="reference checkout not present")
def test_reads_reference_engine_objects():
    """scene_arrays on an engine built by the reference's own API gives the arrays the reference recorded."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden as MG
    engine = MG.scene_box_lattice(2, 1.05, 0.02, 16, seed=1, two_materials=True)
    a = engine_io.scene_arrays(engine)
    d = load_fixture("boxes8")
    for k in SCENE_KEYS:
        np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(d[k]).reshape(np.asarray(a[k]).shape), err_msg=k)


def test_api_set_hinge_matches_the_reference_frames():
    """api.create_hinge / set_hinge (api.py:71-156) give the arms and axes the reference stored for the
    golden hinge chain (world-mode origin and axis, sockets in both bodies' frames)."""
    from rainbow_b200 import api as A
    d = load_fixture("hinges")
    engine = engine_io.engine_from_arrays(d)
    names = list(engine.bodies)
    engine.hinges = {}
    for k in range(len(d["hinge_bodies"])):
        p, c = names[d["hinge_bodies"][k][0]], names[d["hinge_bodies"][k][1]]
        A.create_hinge(engine, "h%d" % k)
        origin = (engine.bodies[p].r + engine.bodies[c].r) / 2.0
        A.set_hinge(engine, "h%d" % k, p, c, origin, np.array([0.0, 0.0, 1.0]), mode="world")
    back = engine_io.scene_arrays(engine)
    np.testing.assert_array_equal(back["hinge_bodies"], d["hinge_bodies"])
    np.testing.assert_allclose(back["hinge_frames"], d["hinge_frames"], rtol=0, atol=1e-15)
    with pytest.raises(RuntimeError):
        A.create_hinge(engine, "h0")
    with pytest.raises(ValueError):
        A.set_hinge(engine, "h0", names[0], names[1], np.zeros(3), np.array([0.0, 0.0, 1.0]), mode="nope")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REFERENCE, "rainbow")), reason="reference checkout not present")
def test_mirror_api_builds_the_reference_scene(monkeypatch):
    """The same user script through the reference's api.py:159-281 calls (create_mesh, create_shape,
    connect_shape, set_position / set_orientation with use_model_frame, set_mass_properties, set_body_type,
    materials, gravity) and through rainbow_b200.api gives equal body-frame meshes (vertex and triangle order),
    shape mass, inertia and frame (shape.r, shape.q), grid extents, body placement (r, q), masses, inertias,
    fixed flags, materials and forces.  The grid values are compared on the GPU (tests/test_gpu_sdf.py); here
    the mirror's grid construction is replaced by its extents only, as this container has no GPU."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden as MG   # puts the reference (with its two import stand-ins) on sys.path
    from rainbow_b200 import api as A, geometry as GEO
    from rainbow_b200.types import Grid

    def extents_only(V, T, I, J, K, boundary=0.5, device="cuda"):
        V = np.asarray(V, np.float64)
        return Grid(V.min(axis=0) - boundary, V.max(axis=0) + boundary, I, J, K)
    monkeypatch.setattr(GEO, "create_signed_distance", extents_only)

    rng = np.random.default_rng(3)
    placements = [(kind, size, rng.uniform(-3, 3, 3), rng.normal(size=4))
                  for kind, size in (("box", (1.0, 0.6, 2.0)), ("sphere", 0.7), ("box", (0.5, 0.5, 0.5)),
                                     ("sphere", 0.3))]

    def build(api, create_box, create_sphere, vec, quat_identity):
        engine = api.create_engine() if api is MG.API else api.create_engine("cpu")
        engine.params.resolution = 6
        api.create_surfaces_interaction(engine, "m", "m", 0.1, vec(0.4, 0.4, 0.4))
        api.create_surfaces_interaction(engine, "m", "w", 0.0, vec(0.3, 0.2, 0.1))
        V, T = create_box(20.0, 1.0, 20.0)
        api.create_shape(engine, "ground_shape", api.create_mesh(V, T))
        api.create_rigid_body(engine, "ground")
        api.connect_shape(engine, "ground", "ground_shape")
        api.set_position(engine, "ground", vec(0.0, -0.5, 0.0), True)
        api.set_orientation(engine, "ground", quat_identity(), True)
        api.set_body_type(engine, "ground", "fixed")
        api.set_mass_properties(engine, "ground", 1.0)
        api.set_body_material(engine, "ground", "m")
        api.create_gravity_force(engine, "gravity", 9.81, vec(0.0, 1.0, 0.0))
        for k, (kind, size, r, q) in enumerate(placements):
            V, T = create_box(*size) if kind == "box" else create_sphere(size, 8, 8)
            api.create_shape(engine, "s%d" % k, api.create_mesh(V, T))
            api.create_rigid_body(engine, "b%d" % k)
            api.connect_shape(engine, "b%d" % k, "s%d" % k)
            api.set_position(engine, "b%d" % k, vec(*r), True)
            api.set_orientation(engine, "b%d" % k, np.asarray(q / np.linalg.norm(q)), True)
            api.set_mass_properties(engine, "b%d" % k, 1000.0 if k % 2 else 1.0)
            api.connect_force(engine, "b%d" % k, "gravity")
            api.set_body_material(engine, "b%d" % k, "w" if k == 2 else "m")
        return engine

    ref = build(MG.API, MG.create_box, MG.create_sphere, MG.V3.make, MG.Q.identity)
    mine = build(A, A.create_box, A.create_sphere, lambda *a: np.array(a, np.float64),
                 lambda: np.array([1.0, 0.0, 0.0, 0.0]))
    assert list(ref.shapes) == list(mine.shapes) and list(ref.bodies) == list(mine.bodies)
    for name in ref.shapes:
        a, b = ref.shapes[name], mine.shapes[name]
        np.testing.assert_array_equal(b.mesh.V, a.mesh.V, err_msg=name)
        np.testing.assert_array_equal(b.mesh.T, a.mesh.T, err_msg=name)
        np.testing.assert_array_equal(b.mass, a.mass, err_msg=name)
        np.testing.assert_array_equal(b.inertia, a.inertia, err_msg=name)
        np.testing.assert_array_equal(b.r, a.r, err_msg=name)
        np.testing.assert_array_equal(b.q, a.q, err_msg=name)
        for f in ("min_coord", "max_coord", "spacing"):
            np.testing.assert_array_equal(getattr(b.grid, f), getattr(a.grid, f), err_msg=name)
        assert (b.grid.I, b.grid.J, b.grid.K) == (a.grid.I, a.grid.J, a.grid.K)
    for name in ref.bodies:
        a, b = ref.bodies[name], mine.bodies[name]
        np.testing.assert_array_equal(b.r, a.r, err_msg=name)
        np.testing.assert_array_equal(b.q, a.q, err_msg=name)
        np.testing.assert_array_equal(b.mass, a.mass, err_msg=name)
        np.testing.assert_array_equal(b.inertia, a.inertia, err_msg=name)
        assert (b.is_fixed, b.material, [f.name for f in b.forces]) == (a.is_fixed, a.material,
                                                                        [f.name for f in a.forces])
    for key in (("m", "m"), ("m", "w")):
        ia, ib = ref.surfaces_interactions.get_interaction(*key), mine.surfaces_interactions.get_interaction(*key)
        np.testing.assert_array_equal(ib.mu, ia.mu)
        assert ib.epsilon == ia.epsilon


def test_simulate_batch_refuses_engines_with_different_parameters():
    """The batched drop-in steps engines that share the step's parameters; a differing one is named before any
    device work (api.simulate_batch, BatchStepper)."""
    from rainbow_b200 import api as A
    from rainbow_b200.stepper import BatchStepper
    a, b = (engine_io.engine_from_arrays(load_fixture("boxes8")) for _ in range(2))
    b.params.time_step = 0.005
    with pytest.raises(ValueError, match="time_step"):
        A.simulate_batch([a, b], 0.01, BatchStepper())
    b.params.time_step = a.params.time_step
    b.params.solver_precision = "fp32_refine"
    with pytest.raises(ValueError, match="solver_precision"):
        A.simulate_batch([a, b], 0.01, BatchStepper())
    with pytest.raises(ValueError):
        A.simulate_batch([a, b], 0.0, BatchStepper())



def test_batch_stepper_host_state_traffic(monkeypatch):
    """BatchStepper's host side against a stand-in world: the state it uploads holds every body's current
    r, q, v, w (arrays edited in place and arrays replaced since the last step alike), the bodies receive the
    world's new state as their own arrays, each engine gets its own contact points (scene-local body indices),
    and adding a body to an engine rebuilds the batch."""
    from rainbow_b200 import api as A, stepper as ST, world as W

    class FakeWorld:
        built = 0

        def __init__(self, arrays, device=None, max_iterations=None):
            FakeWorld.built += 1
            self.scene_start = np.concatenate([[0], np.cumsum([len(a["body_mass"]) for a in arrays])])
            self.n = int(self.scene_start[-1])
            self.uploaded = None

        def set_state(self, x, u):
            self.uploaded = (np.array(x, copy=True), np.array(u, copy=True))

        def step(self, rp):
            return 0

        def state(self):
            x, u = self.uploaded
            return x + 1.0, u + 2.0   # a recognisable "new" state

        def contacts(self):
            # one contact in each scene, between its first two bodies
            ids = np.array([[int(s0), int(s0) + 1] for s0 in self.scene_start[:-1]], dtype=np.int32)
            K = len(ids)
            return dict(ids=ids, p=np.zeros((K, 3)), n=np.tile([0.0, 1.0, 0.0], (K, 1)), g=np.zeros(K),
                        sol=np.zeros(4 * K))

    monkeypatch.setattr(W, "DeviceWorld", FakeWorld)
    monkeypatch.setattr(ST, "_check_status", lambda s: s)
    engines = [engine_io.engine_from_arrays(load_fixture("boxes8")) for _ in range(2)]
    before = [engine_io.body_state(e) for e in engines]
    bs = ST.BatchStepper()
    A.simulate_batch(engines, engines[0].params.time_step, bs)
    world = bs._world
    x0 = np.concatenate([b[0] for b in before])
    np.testing.assert_array_equal(world.uploaded[0], x0)
    for e, (x, u) in zip(engines, before):
        xn, un = engine_io.body_state(e)
        np.testing.assert_array_equal(xn, x + 1.0)
        np.testing.assert_array_equal(un, u + 2.0)
        ids, _, _, _ = e.contact_points.arrays()
        np.testing.assert_array_equal(ids, [[0, 1]])
        names = list(e.bodies)
        assert (e.contact_points[0].bodyA.name, e.contact_points[0].bodyB.name) == (names[0], names[1])
    # edit one body's velocity in place and replace another's spin: the next upload carries both
    b1 = list(engines[1].bodies.values())[3]
    b1.v[0] += 0.25
    b2 = list(engines[0].bodies.values())[2]
    b2.w = np.array([0.0, 0.5, 0.0])
    v_edited = b1.v.copy()
    A.simulate_batch(engines, engines[0].params.time_step, bs)
    assert bs._world is world and FakeWorld.built == 1
    n0 = len(engines[0].bodies)
    np.testing.assert_array_equal(world.uploaded[1][n0 + 3, :3], v_edited)
    np.testing.assert_array_equal(world.uploaded[1][2, 3:], [0.0, 0.5, 0.0])
    np.testing.assert_array_equal(b2.w, [2.0, 2.5, 2.0])   # and the step's result went back into the body
    # a body added to an engine: the batch is rebuilt from the engines
    from rainbow_b200.types import RigidBody
    extra = RigidBody("extra")
    src = list(engines[0].bodies.values())[1]
    for f in ("shape", "mass", "inertia", "is_fixed", "material", "forces"):
        setattr(extra, f, getattr(src, f))
    extra.idx = len(engines[0].bodies)
    extra.r, extra.q, extra.v, extra.w = src.r + 5.0, src.q.copy(), src.v.copy(), src.w.copy()
    engines[0].bodies[extra.name] = extra
    A.simulate_batch(engines, engines[0].params.time_step, bs)
    assert FakeWorld.built == 2 and bs._world.n == sum(len(e.bodies) for e in engines)
    # an engine without bodies is left out of the batch and gets an empty contact list
    from rainbow_b200.types import Engine
    empty = Engine()
    empty.params = engines[0].params
    empty.contact_points = None
    A.simulate_batch(engines + [empty], engines[0].params.time_step, bs)
    assert empty.contact_points == [] and bs._world.n == sum(len(e.bodies) for e in engines)
