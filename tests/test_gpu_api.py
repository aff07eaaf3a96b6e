"""The reference-compatible API on the GPU: drop-in stepper, scene building, signed distance grids."""
import numpy as np
import pytest

from conftest import load_fixture, step_slice

pytestmark = pytest.mark.gpu


def test_stepper_drop_in_on_engine_objects():
    """GpuStepper installed on an engine object reproduces the reference trajectory through API.simulate."""
    from rainbow_b200 import api as API, engine_io
    from rainbow_b200.stepper import GpuStepper
    d = load_fixture("flags")
    engine = engine_io.engine_from_arrays(d)
    engine.stepper = GpuStepper()
    steps = int(d["steps"])
    for s in range(steps):
        API.simulate(engine, float(d["step_dt"][s]), True)
    x, u = engine_io.body_state(engine)
    np.testing.assert_array_equal(x.ravel(), d["step_x"][-1])
    np.testing.assert_array_equal(u.ravel(), d["step_u"][-1])
    log = API.get_log(engine)
    assert len(log) == steps
    for key in ("update_bvh", "narrow_phase", "number_of_overlaps", "contact_determination",
                "contact_point_reduction", "collision_detection_time", "residuals", "iterations", "exitcode",
                "solver_time", "stepper_time", "dt", "contact_points", "kinetic_energy", "potential_energy",
                "max_penetration"):
        assert key in log[-1], key
    assert log[-1]["iterations"] == d["step_iterations"][-1]
    cps = engine.contact_points
    assert len(cps) == len(step_slice(d, "contacts_g", steps - 1))
    names = list(engine.bodies)
    ids = step_slice(d, "contacts_ids", steps - 1)
    for k, cp in enumerate(cps):
        assert cp.bodyA.name == names[ids[k, 0]] and cp.bodyB.name == names[ids[k, 1]]
    np.testing.assert_array_equal(np.array([cp.p for cp in cps]), step_slice(d, "contacts_p", steps - 1))


def test_signed_distance_grid_of_a_box():
    """rb_signed_distance_grid against the closed-form distance of an axis-aligned box."""
    from rainbow_b200 import geometry as GEO
    V, T = GEO.create_box(1.0, 0.6, 2.0)
    grid = GEO.create_signed_distance(V, T, 17, 13, 21, 0.3)
    h = np.array([0.5, 0.3, 1.0])
    I, J, K = grid.I, grid.J, grid.K
    ii, jj, kk = np.meshgrid(np.arange(I), np.arange(J), np.arange(K), indexing="ij")
    p = grid.min_coord + grid.spacing * np.stack([ii, jj, kk], axis=-1)
    q = np.abs(p) - h
    outside = np.linalg.norm(np.maximum(q, 0.0), axis=-1)
    inside = np.minimum(np.max(q, axis=-1), 0.0)
    expected = (outside + inside).transpose(2, 1, 0).ravel()   # i runs fastest (grid3.py:71)
    np.testing.assert_allclose(grid.values, expected, atol=1e-12)


def test_api_scene_matches_oracle(oracle_lib):
    """A scene built through the mirrored API steps identically on the GPU and in the oracle."""
    from rainbow_b200 import engine_io, scenes
    from rainbow_b200 import world as W
    engine = scenes.box_lattice(n=2, resolution=16, seed=3)
    arrays = engine_io.scene_arrays(engine)
    world = W.DeviceWorld(arrays)
    sc = oracle_lib.OracleScene(arrays)
    for _ in range(5):
        world.step(W.make_rb_params(engine.params))
        o = sc.step()
    x, u = world.state()
    np.testing.assert_array_equal(x.ravel(), o["x"])
    np.testing.assert_array_equal(u.ravel(), o["u"])
    assert o["n_contacts"] > 0


def test_simulate_batch_matches_each_engine_stepped_alone():
    """api.simulate_batch over three engines (random boxes and spheres on a ground; 6, 12 and 20 bodies) gives
    every engine the body states and contact points that a GpuStepper of its own gives it through
    api.simulate, bit for bit, also after one body's velocity is edited in place and another body's spin array
    is replaced between two calls."""
    from rainbow_b200 import api as API, scenes
    from rainbow_b200.stepper import BatchStepper, GpuStepper

    def make():
        return [scenes.random_scene(n, np.random.default_rng(seed), resolution=16)
                for n, seed in ((6, 1), (12, 2), (20, 3))]

    def edit(engines):
        list(engines[1].bodies.values())[2].v[1] += 0.5
        list(engines[2].bodies.values())[3].w = np.array([0.0, 1.0, 0.0])

    batch, alone = make(), make()
    for e in alone:
        e.stepper = GpuStepper()
    stepper = BatchStepper()
    dt = batch[0].params.time_step
    contacts = 0
    for k in range(8):
        if k == 4:
            edit(batch)
            edit(alone)
        API.simulate_batch(batch, dt, stepper)
        for e in alone:
            API.simulate(e, dt)
        for eb, ea in zip(batch, alone):
            for b1, b2 in zip(eb.bodies.values(), ea.bodies.values()):
                for f in ("r", "q", "v", "w"):
                    np.testing.assert_array_equal(getattr(b1, f), getattr(b2, f), err_msg="step %d %s" % (k, f))
            for x1, x2 in zip(eb.contact_points.arrays(), ea.contact_points.arrays()):
                np.testing.assert_array_equal(x1, x2)
            assert ([(c.bodyA.name, c.bodyB.name) for c in eb.contact_points] ==
                    [(c.bodyA.name, c.bodyB.name) for c in ea.contact_points])
            contacts += len(eb.contact_points)
    assert contacts > 0


def test_engines_with_device_grids_step_like_their_arrays():
    """Scenes whose grids live on the device (the per-body workload builds them there) go through
    engine_io.engine_from_arrays and api.simulate_batch without a host copy of the grids (each engine's grids
    are views of the workload's tensor) and step bit for bit like the same arrays given to DeviceWorld."""
    import torch
    from rainbow_b200 import api as API, engine_io, scenes, world as W
    from rainbow_b200.stepper import BatchStepper
    arrays, params = scenes.batch_arrays_per_body(n_scenes=1024, seed=0, resolution=32, device="cuda:0",
                                                  select=[3, 11])
    engines = [engine_io.engine_from_arrays(a) for a in arrays]
    grid = next(iter(engines[0].shapes.values())).grid.values
    assert isinstance(grid, torch.Tensor) and grid.is_cuda
    back = engine_io.scene_arrays(engines[0])
    assert isinstance(back["shape_grid"], torch.Tensor) and back["shape_grid"].is_cuda
    world = W.DeviceWorld(arrays, device="cuda:0", max_iterations=100)
    rp = W.make_rb_params(params)
    stepper = BatchStepper()
    for _ in range(5):
        assert world.step(rp) == 0
        API.simulate_batch(engines, engines[0].params.time_step, stepper)
    x, u = world.state()
    xb = np.concatenate([engine_io.body_state(e)[0] for e in engines])
    ub = np.concatenate([engine_io.body_state(e)[1] for e in engines])
    np.testing.assert_array_equal(xb, x)
    np.testing.assert_array_equal(ub, u)
