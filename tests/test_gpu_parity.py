"""GPU step (through the C ABI) against the reference's recorded steps and against the oracle.

FP64 parity target: bit-identical contact sets (body indices, positions, normals, gaps), solver impulses,
iteration counts and body states.  The required bound is 1e-9 relative; the kernels reproduce NumPy's
rounding sequence, so the tests demand exact equality."""
import numpy as np
import pytest

from conftest import FIXTURES, load_fixture, step_slice

pytestmark = pytest.mark.gpu


def _world(d, **kw):
    from rainbow_b200 import world as W
    return W.DeviceWorld(d, **kw)


def _params(d, dt=None, scheme="rigid_gauss_seidel", profiling=True):
    from rainbow_b200 import world as W
    return W.make_rb_params(W.params_from_vector(d["params"]), dt=dt, scheme=scheme, profiling=profiling)


def _assert_step(world, d, s, scene=0):
    st = world.stats()[scene]
    c = world.contacts()
    k0, K = st.contact_start, st.n_contacts
    ids = c["ids"][k0:k0 + K] - world.scene_start[scene]
    np.testing.assert_array_equal(ids, step_slice(d, "contacts_ids", s), err_msg="step %d contact ids" % s)
    for key, ref in (("p", "contacts_p"), ("n", "contacts_n"), ("g", "contacts_g")):
        np.testing.assert_array_equal(c[key][k0:k0 + K], step_slice(d, ref, s), err_msg="step %d %s" % (s, key))
    np.testing.assert_array_equal(c["sol"][4 * k0:4 * (k0 + K)], step_slice(d, "sol", s), err_msg="step %d sol" % s)
    assert st.iterations == d["step_iterations"][s]
    assert st.exitcode == d["step_exitcode"][s]
    assert st.post_iterations == d["step_post_iterations"][s]
    if world.n_hinges and "step_hinge_sol_len" in d:
        np.testing.assert_array_equal(world.hinge_solution(), step_slice(d, "hinge_sol", s),
                                      err_msg="step %d hinge sol" % s)
    x, u = world.state()
    b0, b1 = world.scene_start[scene], world.scene_start[scene + 1]
    np.testing.assert_array_equal(x[b0:b1].ravel(), d["step_x"][s], err_msg="step %d x" % s)
    np.testing.assert_array_equal(u[b0:b1].ravel(), d["step_u"][s], err_msg="step %d u" % s)


@pytest.mark.parametrize("name", FIXTURES)
def test_gpu_matches_reference_step_by_step(name):
    d = load_fixture(name)
    world = _world(d)
    N = world.n_bodies
    for s in range(int(d["steps"])):
        if s > 0:
            world.set_state(d["step_x"][s - 1].reshape(N, 7), d["step_u"][s - 1].reshape(N, 6))
        status = world.step(_params(d, dt=float(d["step_dt"][s])))
        assert status == 0
        _assert_step(world, d, s)


def test_gpu_free_run_matches_reference():
    d = load_fixture("boxes8")
    world = _world(d)
    for s in range(int(d["steps"])):
        world.step(_params(d, dt=float(d["step_dt"][s])))
    _assert_step(world, d, int(d["steps"]) - 1)


@pytest.mark.parametrize("scheme", ["gauss_seidel", "parallel_jacobi", "parallel_jacobi_hybrid"])
def test_gpu_proximal_contact_schemes_match_reference(scheme):
    d = load_fixture("solvers")
    world = _world(d)
    world.step(_params(d, scheme=scheme))
    st = world.stats()[0]
    c = world.contacts()
    np.testing.assert_array_equal(c["ids"], d["contacts_ids"])
    np.testing.assert_array_equal(c["sol"], d["sol_" + scheme])
    assert st.iterations == d["iterations_" + scheme]
    assert st.exitcode == d["exitcode_" + scheme]


@pytest.mark.parametrize("scheme", ["parallel_jacobi", "gauss_seidel"])
def test_gpu_schemes_match_oracle_over_steps(oracle_lib, scheme):
    """Several chained steps with a proximal_contact scheme: GPU and oracle stay bit-identical."""
    d = load_fixture("spheres")
    world = _world(d)
    sc = oracle_lib.OracleScene(d)
    for s in range(4):
        world.step(_params(d, scheme=scheme))
        o = sc.step(scheme=scheme)
        c = world.contacts()
        np.testing.assert_array_equal(c["ids"], o["ids"])
        np.testing.assert_array_equal(c["sol"], o["sol"])
        x, u = world.state()
        np.testing.assert_array_equal(x.ravel(), o["x"])
        np.testing.assert_array_equal(u.ravel(), o["u"])


def test_batched_scenes_equal_alone():
    """Every scene gives the same bits alone and packed with the other fixtures into one launch."""
    from rainbow_b200 import world as W
    ds = [load_fixture(n) for n in ("boxes8", "spheres", "tower6", "c1_boxes64")]
    # one parameter set for the whole batch: the tower's dt and tolerances
    params = W.params_from_vector(ds[2]["params"])
    alone = []
    for d in ds:
        w = _world(d, max_iterations=100)
        for _ in range(3):
            w.step(W.make_rb_params(params))
        alone.append((w.state(), w.contacts(), w.stats()[0]))
    batch = W.DeviceWorld(ds, max_iterations=100)
    for _ in range(3):
        batch.step(W.make_rb_params(params))
    x, u = batch.state()
    c = batch.contacts()
    for i, ((xa, ua), ca, sa) in enumerate(alone):
        b0, b1 = batch.scene_start[i], batch.scene_start[i + 1]
        np.testing.assert_array_equal(x[b0:b1], xa)
        np.testing.assert_array_equal(u[b0:b1], ua)
        st = batch.stats()[i]
        assert (st.n_contacts, st.iterations, st.exitcode) == (sa.n_contacts, sa.iterations, sa.exitcode)
        k0 = st.contact_start
        np.testing.assert_array_equal(c["ids"][k0:k0 + st.n_contacts] - b0, ca["ids"])
        np.testing.assert_array_equal(c["sol"][4 * k0:4 * (k0 + st.n_contacts)], ca["sol"])


def test_capacity_growth_repeats_step():
    """Work lists far too small: the step reports the overflow, leaves the state alone, grows and repeats."""
    d = load_fixture("spheres")
    ref = _world(d)
    ref.step(_params(d))
    small = _world(d, caps={"pairs": 2, "items": 8, "contacts": 4})
    small.step(_params(d))
    assert small.caps.pair_capacity > 2 and small.caps.contact_capacity > 4
    np.testing.assert_array_equal(small.state()[0], ref.state()[0])
    np.testing.assert_array_equal(small.contacts()["sol"], ref.contacts()["sol"])


def test_profile_counts_match_oracle(oracle_lib):
    d = load_fixture("c1_boxes64")
    world = _world(d)
    world.step(_params(d, profiling=True))
    st = world.stats()[0]
    o = oracle_lib.OracleScene(d).step()
    assert st.n_leaf_overlaps == o["n_leaf_overlaps"]
    assert st.n_candidates == o["n_candidates"]
    assert abs(st.kinetic_energy - o["kinetic"]) <= 1e-12 * max(1.0, abs(o["kinetic"]))
    assert st.potential_energy == o["potential"]
    assert st.max_penetration == o["max_penetration"]
    times = world.profile_times()
    assert len(times) == 7 and times[6] > 0.0


@pytest.mark.parametrize("termination,mode", [("residual", 1), ("residual_fixed_r", 2)])
@pytest.mark.parametrize("scheme", ["rigid_gauss_seidel", "gauss_seidel"])
def test_residual_termination_matches_oracle(oracle_lib, termination, mode, scheme):
    """Solves stopped by the complementarity residual (tolerance 1e-6) stay bit-identical to the oracle."""
    from rainbow_b200 import world as W
    d = load_fixture("c1_boxes64")
    p = W.params_from_vector(d["params"])
    p["max_iterations"] = 200
    world = _world(d, max_iterations=200)
    sc = oracle_lib.OracleScene(d)
    sc.set_param("max_iterations", 200)
    for _ in range(3):
        world.step(W.make_rb_params(p, scheme=scheme, termination=termination, residual_tolerance=1e-6))
        o = sc.step(scheme=scheme, tol_mode=mode, tol=1e-6)
        st = world.stats()[0]
        assert (st.iterations, st.exitcode) == (o["iterations"], o["exitcode"])
        np.testing.assert_array_equal(world.contacts()["sol"], o["sol"])
        x, u = world.state()
        np.testing.assert_array_equal(x.ravel(), o["x"])
        np.testing.assert_array_equal(u.ravel(), o["u"])


def test_warm_start_reuses_previous_impulses():
    """Warm-started solves reach the same residual tolerance in fewer sweeps; the cache holds every contact."""
    from rainbow_b200 import world as W
    d = load_fixture("c1_boxes64")
    p = W.params_from_vector(d["params"])
    p["max_iterations"] = 200
    sweeps = {}
    for warm in (False, True):
        world = _world(d, max_iterations=200)
        total = 0
        for s in range(int(d["steps"])):
            world.step(W.make_rb_params(p, termination="residual_fixed_r", residual_tolerance=1e-6, warm_start=warm))
            st = world.stats()[0]
            assert st.exitcode == 3 and st.residual <= 1e-6
            total += st.iterations + 1
        assert int(world.t_cache_count.item()) == st.n_contacts
        keys = world.t_cache_key[:2 * st.n_contacts].view(-1, 2).cpu().numpy()
        assert all(tuple(keys[i]) < tuple(keys[i + 1]) for i in range(len(keys) - 1))
        sweeps[warm] = total
    assert sweeps[True] < sweeps[False]


def test_residual_interval_matches_oracle(oracle_lib):
    """Fixed-r solves that test the residual every fourth sweep stay bit-identical to the oracle."""
    from rainbow_b200 import world as W
    d = load_fixture("c1_boxes64")
    p = W.params_from_vector(d["params"])
    p["max_iterations"] = 200
    world = _world(d, max_iterations=200)
    sc = oracle_lib.OracleScene(d)
    sc.set_param("max_iterations", 200)
    for _ in range(3):
        world.step(W.make_rb_params(p, termination="residual_fixed_r", residual_tolerance=1e-6, residual_interval=4))
        o = sc.step(tol_mode=2, tol=1e-6, residual_interval=4)
        st = world.stats()[0]
        assert (st.iterations, st.exitcode) == (o["iterations"], o["exitcode"])
        assert st.exitcode == 3 and (st.iterations + 1) % 4 == 0
        np.testing.assert_array_equal(world.contacts()["sol"], o["sol"])
        np.testing.assert_array_equal(world.state()[0].ravel(), o["x"])


@pytest.mark.parametrize("name", ["c1_boxes64", "spheres"])
def test_fp32_refine_meets_the_fp64_tolerance(name):
    """FP32 sweeps on chip followed by FP64 refinement: the FP64 residual meets the tolerance and the step's
    velocities agree with the FP64 solve to a small fraction of their scale."""
    from rainbow_b200 import world as W
    d = load_fixture(name)
    p = W.params_from_vector(d["params"])
    p["max_iterations"] = 400
    kw = dict(termination="residual_fixed_r", residual_tolerance=1e-6, residual_interval=4)
    w64 = _world(d, max_iterations=400)
    w32 = _world(d, max_iterations=400)
    w64.step(W.make_rb_params(p, precision="fp64", **kw))
    w32.step(W.make_rb_params(p, precision="fp32_refine", refine_iterations=100, **kw))
    s64, s32 = w64.stats()[0], w32.stats()[0]
    assert s64.exitcode == 3 and s32.exitcode == 3
    assert s32.residual <= 1e-6 and s32.fp32_sweeps > 0
    np.testing.assert_array_equal(w32.contacts()["ids"], w64.contacts()["ids"])
    u64, u32 = w64.state()[1], w32.state()[1]
    scale = np.abs(u64).max()
    assert np.abs(u32 - u64).max() <= 1e-3 * scale + 1e-9


def test_fp32_only_reports_its_fp64_residual():
    from rainbow_b200 import world as W
    d = load_fixture("c1_boxes64")
    p = W.params_from_vector(d["params"])
    w32 = _world(d)
    w32.step(W.make_rb_params(p, precision="fp32", termination="residual_fixed_r", residual_tolerance=1e-6))
    st = w32.stats()[0]
    assert st.fp32_sweeps > 0 and np.isfinite(st.residual) and st.residual < 1e-2
    assert st.exitcode in (0, 3) and (st.exitcode == 3) == (st.residual <= 1e-6)


def test_graph_replay_equals_direct_steps():
    """A step captured into a CUDA graph and replayed advances the batch with the same bits as direct calls."""
    import torch
    from rainbow_b200 import world as W
    ds = [load_fixture(n) for n in ("boxes8", "spheres", "tower6")]
    params = W.params_from_vector(ds[2]["params"])
    rp = W.make_rb_params(params, warm_start=True, termination="residual_fixed_r", residual_tolerance=1e-6)
    direct = W.DeviceWorld(ds, max_iterations=100)
    graphed = W.DeviceWorld(ds, max_iterations=100)
    for _ in range(4):
        direct.step(rp)
    graphed.step(rp)                       # uncaptured first step: sizes the work lists
    graph = graphed.capture(rp)
    graphed.t_status.zero_()
    for _ in range(3):
        graph.replay()
    torch.cuda.synchronize()
    assert int(graphed.t_status[0].item()) == 0
    for a, b in zip(direct.state(), graphed.state()):
        np.testing.assert_array_equal(b, a)
    ca, cb = direct.contacts(), graphed.contacts()
    for key in ("ids", "p", "sol"):
        np.testing.assert_array_equal(cb[key], ca[key], err_msg=key)


def test_pinned_state_views_round_trip():
    """state(copy=False) hands out the pinned staging buffers; passing them back to set_state uploads them
    without a host copy, and the steps that follow are the same bits as with copied arrays."""
    from rainbow_b200 import world as W
    ds = [load_fixture(n) for n in ("boxes8", "spheres")]
    p = W.params_from_vector(ds[0]["params"])
    p["max_iterations"] = 100
    rp = W.make_rb_params(p)
    copied = W.DeviceWorld(ds, max_iterations=100)
    viewed = W.DeviceWorld(ds, max_iterations=100)
    x, u = copied.state()
    hx, hu = viewed.state(copy=False)
    np.testing.assert_array_equal(hx, x)
    for _ in range(3):
        copied.set_state(x, u)
        copied.step(rp)
        x, u = copied.state()
        viewed.set_state(hx, hu)
        viewed.step(rp)
        hx, hu = viewed.state(copy=False)
        np.testing.assert_array_equal(hx, x)
        np.testing.assert_array_equal(hu, u)


def test_fp32_refine_spends_the_same_sweep_budget():
    """Unconverged FP32+FP64 solves use exactly max_iterations sweeps, like the FP64 solve they stand in for,
    with the reserved FP64 sweeps at the end."""
    from rainbow_b200 import world as W
    d = load_fixture("c1_boxes64")
    p = W.params_from_vector(d["params"])
    p["max_iterations"] = 30
    w = _world(d, max_iterations=30)
    w.step(W.make_rb_params(p, precision="fp32_refine", refine_iterations=10, termination="residual_fixed_r",
                            residual_tolerance=1e-12))
    st = w.stats()[0]
    assert st.exitcode == 0 and st.iterations == 30
    assert 0 < st.fp32_sweeps <= 20


@pytest.mark.parametrize("scheme,ordering,termination,mode", [
    ("parallel_gauss_seidel", "serial", "merit", 0),
    ("rigid_gauss_seidel", "coloured", "merit", 0),
    ("rigid_gauss_seidel", "coloured", "residual_fixed_r", 2),
    ("gauss_seidel", "coloured", "residual", 1),
])
@pytest.mark.parametrize("name", ["c1_boxes64", "tower6", "spheres"])
def test_coloured_gauss_seidel_matches_oracle(oracle_lib, name, scheme, ordering, termination, mode):
    """Graph-coloured sweeps: the GPU colours the contacts like the oracle (same number of colours) and the
    chained steps stay bit-identical to it."""
    from rainbow_b200 import world as W
    d = load_fixture(name)
    p = W.params_from_vector(d["params"])
    world = _world(d)
    sc = oracle_lib.OracleScene(d)
    for _ in range(3):
        world.step(W.make_rb_params(p, scheme=scheme, ordering=ordering, termination=termination,
                                    residual_tolerance=1e-6))
        o = sc.step(scheme=scheme, ordering=ordering, tol_mode=mode, tol=1e-6)
        st = world.stats()[0]
        assert st.n_contacts == o["n_contacts"]
        if o["n_contacts"]:
            assert st.n_levels == o["n_colours"]
        assert (st.iterations, st.exitcode) == (o["iterations"], o["exitcode"])
        np.testing.assert_array_equal(world.contacts()["sol"], o["sol"])
        x, u = world.state()
        np.testing.assert_array_equal(x.ravel(), o["x"])
        np.testing.assert_array_equal(u.ravel(), o["u"])


def test_coloured_fp32_refine_meets_the_tolerance():
    from rainbow_b200 import world as W
    d = load_fixture("c1_boxes64")
    p = W.params_from_vector(d["params"])
    p["max_iterations"] = 400
    w = _world(d, max_iterations=400)
    w.step(W.make_rb_params(p, precision="fp32_refine", ordering="coloured", refine_iterations=100,
                            termination="residual_fixed_r", residual_tolerance=1e-6))
    st = w.stats()[0]
    assert st.exitcode == 3 and st.residual <= 1e-6 and st.fp32_sweeps > 0


def test_hinge_scenes_batched_with_others_equal_alone():
    """Hinge chains packed with contact-only scenes: every scene gives the same bits as alone (the hinge
    problem of one scene never sees another scene's bodies)."""
    from rainbow_b200 import world as W
    ds = [load_fixture(n) for n in ("boxes8", "hinges", "tower6", "hinges_stab")]
    params = W.params_from_vector(ds[1]["params"])
    cap = int(params["max_iterations"])
    alone = []
    for d in ds:
        w = _world(d, max_iterations=cap)
        for _ in range(5):
            w.step(W.make_rb_params(params))
        alone.append((w.state(), w.hinge_solution() if w.n_hinges else None))
    batch = W.DeviceWorld(ds, max_iterations=cap)
    for _ in range(5):
        batch.step(W.make_rb_params(params))
    x, u = batch.state()
    hs = batch.hinge_solution()
    h = 0
    for i, ((xa, ua), ha) in enumerate(alone):
        b0, b1 = batch.scene_start[i], batch.scene_start[i + 1]
        np.testing.assert_array_equal(x[b0:b1], xa)
        np.testing.assert_array_equal(u[b0:b1], ua)
        if ha is not None:
            np.testing.assert_array_equal(hs[h:h + len(ha)], ha)
            h += len(ha)


def test_hinges_reject_other_solver_settings():
    from rainbow_b200 import _native as N
    from rainbow_b200 import world as W
    d = load_fixture("hinges")
    w = _world(d)
    with pytest.raises(N.NativeError, match="hinge"):
        w.step(W.make_rb_params(W.params_from_vector(d["params"]), termination="residual_fixed_r"))
