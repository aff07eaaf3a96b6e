"""Failure paths, made on the host: a non-finite body state and requests the server cannot take.

A NaN written into a body's velocity on the host flows through one step without deciding any index or loop
count: it enters the contact problem's b and the impulses of that body's contacts, and the solver's loops end
at the sweep cap (a NaN residual counts as unconverged).  Positions decide indices only through bounding boxes,
whose min/max reductions skip NaN (a NaN body joins no pair), and grid cells, where a NaN coordinate clamps to
cell 0.  The step's integration flags the state, the device status carries RB_STATUS_NONFINITE, and the
Python layers raise (the reference would carry the NaN on silently)."""
import numpy as np
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu


def test_nan_state_sets_the_status_bit_and_raises():
    from rainbow_b200 import _native as N
    from rainbow_b200 import api as API, engine_io, world as W
    from rainbow_b200.stepper import GpuStepper
    d = load_fixture("boxes8")
    world = W.DeviceWorld(d)
    rp = W.make_rb_params(W.params_from_vector(d["params"]))
    assert world.step(rp) == 0
    x, u = world.state()
    u[3, 0] = np.nan                       # one body's velocity on the host
    world.set_state(x, u)
    status = world.step(rp)
    assert status & N.STATUS_NONFINITE
    assert not np.isfinite(world.state()[0][3]).all()
    # the same through the drop-in stepper: the step raises and the engine keeps its last good state
    engine = engine_io.engine_from_arrays(d)
    engine.stepper = GpuStepper()
    API.simulate(engine, engine.params.time_step)
    body = list(engine.bodies.values())[3]
    body.v = np.array([np.nan, 0.0, 0.0])
    r_before = body.r.copy()
    with pytest.raises(N.NativeError, match="non-finite"):
        API.simulate(engine, engine.params.time_step)
    np.testing.assert_array_equal(body.r, r_before)


def test_server_rejects_a_request_it_cannot_run_and_serves_the_rest():
    """A scene with a shape beyond the 16384-triangle limit is rejected at admission with the reason; the
    requests before and after it are served as if it had never come."""
    from rainbow_b200 import geometry as GEO
    from rainbow_b200 import serving as S
    from rainbow_b200 import world as W
    good1, good2 = load_fixture("boxes8"), load_fixture("tower6")
    bad = dict(load_fixture("spheres"))
    V, T = GEO.create_sphere(1.0, 100, 100)                # 19800 triangles
    assert len(T) > W.MAX_TRIANGLES_PER_SHAPE
    sv, st = np.asarray(bad["shape_v_off"]), np.asarray(bad["shape_t_off"])
    bad["shape_V"] = np.concatenate([np.asarray(bad["shape_V"]).reshape(-1, 3)[:sv[-2]], V])
    bad["shape_T"] = np.concatenate([np.asarray(bad["shape_T"]).reshape(-1, 3)[:st[-2]], T])
    bad["shape_v_off"] = np.concatenate([sv[:-1], [sv[-2] + len(V)]])
    bad["shape_t_off"] = np.concatenate([st[:-1], [st[-2] + len(T)]])
    params = W.params_from_vector(good2["params"])
    rp = W.make_rb_params(params)
    srv = S.Server(rp, max_iterations=100)
    u1 = srv.submit(good1, 3)
    ub = srv.submit(bad, 3)
    u2 = srv.submit(good2, 2)
    srv.run()
    assert [r.uid for r in srv.rejected] == [ub]
    assert "triangles" in srv.rejected[0].error
    assert sorted(r.uid for r in srv.finished) == [u1, u2]
    assert srv.report()["rejected"] == 1
    done = {r.uid: r for r in srv.finished}
    for r, d in ((done[u1], good1), (done[u2], good2)):
        w = W.DeviceWorld(d, max_iterations=int(rp.max_iterations))
        for _ in range(r.horizon):
            w.step(rp)
        np.testing.assert_array_equal(r.result[0], w.state()[0])


def test_server_holds_requests_beyond_its_memory_budget():
    """With a budget too small for two scenes, the second request waits in the queue until the first has
    left, then runs; both results equal their scenes stepped alone."""
    from rainbow_b200 import serving as S
    from rainbow_b200 import world as W
    a, b = load_fixture("boxes8"), load_fixture("spheres")
    rp = W.make_rb_params(W.params_from_vector(a["params"]))
    srv = S.Server(rp, max_iterations=100, hbm_fraction=1e-9)   # only an empty server admits (its first scene)
    ua, ub = srv.submit(a, 3), srv.submit(b, 2)
    srv.tick()
    assert len(srv.active) == 1 and len(srv.queue) == 1
    srv.run()
    assert [t["scenes"] for t in srv.ticks] == [1, 1, 1, 1, 1]
    done = {r.uid: r for r in srv.finished}
    assert sorted(done) == [ua, ub]
    assert done[ub].admitted >= done[ua].admitted
    for uid, d, h in ((ua, a, 3), (ub, b, 2)):
        w = W.DeviceWorld(d, max_iterations=int(rp.max_iterations))
        for _ in range(h):
            w.step(rp)
        np.testing.assert_array_equal(done[uid].result[0], w.state()[0])
