"""GPU step against the oracle on the benchmarked workloads, FP64, bit for bit.

The golden fixtures pin the oracle to the reference's own NumPy step on scenes of up to 65 bodies.  These
tests carry the GPU step's parity to the scenes and settings the benchmark times, where the kernels take
paths the fixtures never reach (block teams with thousands of bodies on chip, long contact lists per body,
work-list growth, the warm-start cache):

* eight scenes of the batched workload (8..256 random boxes and spheres; the 185- and 225-body scenes among
  them), batched together and each alone, with the benchmark's FP64 solver settings (complementarity
  residual 1e-6 tested every 4 sweeps, fixed r, warm start) and with the reference's own settings (merit
  rule, no warm start);
* the 32-box tower with mass ratio 1e3 (dt 0.005) over 60 steps;
* the 4096-body box/sphere lattice at SDF resolution 64;
* a 2048-body scene of the serving workload (the top of its 16..2048 body range);
* the 64-box lattice run freely for 100 steps with the reference's parameters;
* four scenes of the default benchmark workload, which gives every body a shape and grid of its own.

Every compared step asserts equal contact ids, positions, normals, gaps, impulses, iteration counts, exit
codes and body states.  The reference steps these scenes through steppers.py:47-106; the oracle restates that
step operation by operation."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BENCH = dict(termination="residual_fixed_r", residual_tolerance=1e-6, residual_interval=4, warm_start=True)
BENCH_ORACLE = dict(tol_mode=2, tol=1e-6, residual_interval=4, warm_start=True)
BATCH_SCENES = [0, 1, 4, 7, 8, 12, 13, 14]   # 12, 95, 41, 185, 97, 54, 225, 155 bodies (+ ground)


def _check(world, o, scene, tag):
    """GPU results of `scene` in `world` against the oracle's step result `o`."""
    st = world.stats()[scene]
    c = world.contacts()
    k0, K = st.contact_start, st.n_contacts
    b0, b1 = world.scene_start[scene], world.scene_start[scene + 1]
    assert K == o["n_contacts"], "%s: %d contacts, oracle %d" % (tag, K, o["n_contacts"])
    np.testing.assert_array_equal(c["ids"][k0:k0 + K] - b0, o["ids"], err_msg=tag + " ids")
    for key in ("p", "n", "g"):
        np.testing.assert_array_equal(c[key][k0:k0 + K], o[key], err_msg=tag + " " + key)
    np.testing.assert_array_equal(c["sol"][4 * k0:4 * (k0 + K)], o["sol"], err_msg=tag + " sol")
    if K:
        assert (st.iterations, st.exitcode) == (o["iterations"], o["exitcode"]), tag
    x, u = world.state()
    np.testing.assert_array_equal(x[b0:b1].ravel(), o["x"], err_msg=tag + " x")
    np.testing.assert_array_equal(u[b0:b1].ravel(), o["u"], err_msg=tag + " u")


def _rb(params, bench):
    from rainbow_b200 import world as W
    return W.make_rb_params(params, **(BENCH if bench else {}))


@pytest.fixture(scope="module")
def batch_scenes():
    from rainbow_b200 import scenes
    arrays, params = scenes.batch_arrays(n_scenes=max(BATCH_SCENES) + 1, seed=0, pool=64, resolution=32,
                                         device="cuda:0")
    return [arrays[i] for i in BATCH_SCENES], params


@pytest.mark.parametrize("bench", [True, False], ids=["bench_settings", "reference_settings"])
def test_batch_scenes_match_oracle_batched_and_alone(oracle_lib, batch_scenes, bench):
    from rainbow_b200 import world as W
    arrays, params = batch_scenes
    steps = 25 if bench else 12
    okw = BENCH_ORACLE if bench else {}
    rp = _rb(params, bench)
    batch = W.DeviceWorld(arrays, device="cuda:0", max_iterations=100)
    alone = [W.DeviceWorld(a, device="cuda:0", max_iterations=100) for a in arrays]
    ors = [oracle_lib.OracleScene(a) for a in arrays]
    contacts = 0
    for s in range(steps):
        assert batch.step(rp) == 0
        for i, (w1, sc) in enumerate(zip(alone, ors)):
            assert w1.step(rp) == 0
            o = sc.step(**okw)
            contacts += o["n_contacts"]
            _check(batch, o, i, "step %d scene %d batched" % (s, BATCH_SCENES[i]))
            _check(w1, o, 0, "step %d scene %d alone" % (s, BATCH_SCENES[i]))
    assert contacts > 0


def test_tower32_matches_oracle(oracle_lib):
    from rainbow_b200 import engine_io, scenes, world as W
    arrays = engine_io.scene_arrays(scenes.box_tower(32, device="cuda:0"))
    params = W.params_from_vector(arrays["params"])
    world = W.DeviceWorld(arrays, device="cuda:0", max_iterations=100)
    sc = oracle_lib.OracleScene(arrays)
    rp = _rb(params, True)
    for s in range(60):
        assert world.step(rp) == 0
        _check(world, sc.step(**BENCH_ORACLE), 0, "tower step %d" % s)


def test_mixed_lattice_4096_matches_oracle(oracle_lib):
    from rainbow_b200 import engine_io, scenes, world as W
    arrays = engine_io.scene_arrays(scenes.mixed_lattice(n=16, spacing=1.2, resolution=64, seed=0, device="cuda:0"))
    params = W.params_from_vector(arrays["params"])
    world = W.DeviceWorld(arrays, device="cuda:0", max_iterations=100)
    sc = oracle_lib.OracleScene(arrays)
    rp = _rb(params, True)
    total = 0
    for s in range(6):
        assert world.step(rp) == 0
        o = sc.step(**BENCH_ORACLE)
        total += o["n_contacts"]
        _check(world, o, 0, "lattice step %d" % s)
    assert total > 1000


def test_serving_scene_2048_matches_oracle(oracle_lib):
    from rainbow_b200 import scenes, world as W
    arrays, params = scenes.batch_arrays(n_scenes=1, seed=1, pool=64, body_range=(2048, 2048), resolution=32,
                                         device="cuda:0", ground=40.0)
    assert len(arrays[0]["body_mass"]) == 2049
    world = W.DeviceWorld(arrays, device="cuda:0", max_iterations=100)
    sc = oracle_lib.OracleScene(arrays[0])
    rp = _rb(params, True)
    total = 0
    for s in range(12):
        assert world.step(rp) == 0
        o = sc.step(**BENCH_ORACLE)
        total += o["n_contacts"]
        _check(world, o, 0, "serving scene step %d" % s)
    assert total > 0


def test_c1_free_run_100_steps_matches_oracle(oracle_lib):
    """The 64-box lattice (spacing 1.05, jitter 0.02) on its ground, 100 steps, the reference's parameters
    (merit rule, at most 100 iterations, relative tolerance 1e-6, no warm start): GPU and oracle run freely
    from the same initial state and stay bit-identical throughout."""
    from rainbow_b200 import engine_io, scenes, world as W
    arrays = engine_io.scene_arrays(scenes.box_lattice(n=4, spacing=1.05, jitter=0.02, resolution=32, seed=0,
                                                       device="cuda:0"))
    params = W.params_from_vector(arrays["params"])
    world = W.DeviceWorld(arrays, device="cuda:0", max_iterations=100)
    sc = oracle_lib.OracleScene(arrays)
    rp = W.make_rb_params(params)
    for s in range(100):
        assert world.step(rp) == 0
        o = sc.step()
        if s % 10 == 9:
            _check(world, o, 0, "C1 step %d" % s)
    assert o["n_contacts"] > 0


def test_per_body_workload_scenes_match_oracle(oracle_lib):
    """The default benchmark workload gives every body a shape and grid of its own.  Four of its scenes --
    the largest of all 1024 (257 bodies) and three of the first twenty (179, 145 and 11 bodies) -- built alone
    (the draws of the other scenes replayed, their shapes not built), batched together and stepped 20 steps
    with the bench's FP64 settings: bit-identical to the oracle on host copies at every step."""
    from rainbow_b200 import scenes, world as W
    pick = [3, 9, 11, 419]
    arrays, params = scenes.batch_arrays_per_body(n_scenes=1024, seed=0, resolution=32, device="cuda:0", select=pick)
    assert sorted(len(a["body_mass"]) for a in arrays) == [11, 145, 179, 257]
    host = [{k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in a.items()} for a in arrays]
    world = W.DeviceWorld(arrays, device="cuda:0", max_iterations=100)
    ors = [oracle_lib.OracleScene(h) for h in host]
    rp = _rb(params, True)
    contacts = 0
    for s in range(20):
        assert world.step(rp) == 0
        for i, sc in enumerate(ors):
            o = sc.step(**BENCH_ORACLE)
            contacts += o["n_contacts"]
            _check(world, o, i, "per-body step %d scene %d" % (s, i))
    assert contacts > 0
