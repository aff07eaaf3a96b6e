"""Continuous batching on the GPU: the device-built layout equals the host packing, and every scene served in
a changing mix gives the same result as the scene stepped alone (FP64 and FP32+FP64 refinement: bit-identical,
tolerance 0)."""
import ctypes

import numpy as np
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu

NAMES = ("boxes8", "spheres", "tower6", "c1_boxes64")


def test_device_topology_equals_host_packing():
    from rainbow_b200 import serving as S
    from rainbow_b200 import world as W
    ds = [load_fixture(n) for n in NAMES]
    lib = S.ShapeLibrary("cuda")
    blocks = [S.SceneBlock(d, lib) for d in ds]
    batch = S.ServingBatch(lib, blocks, "cuda", (4096, 65536, 4096), 100)
    ref = W.pack_scenes(ds)
    for key in ("body_v0", "body_t0", "body_c0", "vert_body", "tri_body", "clu_body"):
        np.testing.assert_array_equal(batch.tensors[key].cpu().numpy(), ref[key], err_msg=key)


def _alone(d, rp, steps):
    from rainbow_b200 import world as W
    w = W.DeviceWorld(d, max_iterations=100)
    for _ in range(steps):
        w.step(rp)
    return w.state()


@pytest.mark.parametrize("precision,ordering", [("fp64", "serial"), ("fp32_refine", "serial"),
                                                ("fp64", "coloured")])
def test_each_scene_is_the_same_alone_and_in_the_mix(precision, ordering):
    from rainbow_b200 import serving as S
    from rainbow_b200 import world as W
    ds = [load_fixture(n) for n in NAMES]
    params = W.params_from_vector(ds[2]["params"])
    rp = W.make_rb_params(params, warm_start=True, termination="residual_fixed_r", residual_tolerance=1e-6,
                          residual_interval=2, precision=precision, ordering=ordering)
    horizons = [6, 4, 5, 3]
    # at most 80 resident bodies: the 65-body lattice waits in the queue until the others have left
    srv = S.Server(rp, max_iterations=100, max_active_bodies=80)
    uids = [srv.submit(ds[0], horizons[0]), srv.submit(ds[1], horizons[1])]
    srv.tick()
    srv.tick()
    uids.append(srv.submit(ds[2], horizons[2]))   # joins a batch already in flight
    srv.tick()
    uids.append(srv.submit(ds[3], horizons[3]))
    srv.run()
    assert srv.idle()
    done = {r.uid: r for r in srv.finished}
    assert sorted(done) == sorted(uids)
    mixes = {t["scenes"] for t in srv.ticks}
    assert max(mixes) >= 2 and len(srv.ticks) > max(horizons)
    for uid, d, h in zip(uids, ds, horizons):
        x, u = done[uid].result
        xa, ua = _alone(d, rp, h)
        np.testing.assert_array_equal(x, xa, err_msg="scene %d x" % uid)
        np.testing.assert_array_equal(u, ua, err_msg="scene %d u" % uid)
    rep = srv.report()
    assert rep["finished"] == 4 and rep["scene_steps"] == sum(horizons)


def test_repack_carries_the_warm_start_cache():
    """After a scene leaves, the staying scene's cached impulses are found again under its new body indices:
    its next solve starts from them and needs no more sweeps than when stepped alone."""
    from rainbow_b200 import serving as S
    from rainbow_b200 import world as W
    ds = [load_fixture(n) for n in ("boxes8", "tower6")]
    params = W.params_from_vector(ds[1]["params"])
    rp = W.make_rb_params(params, warm_start=True, termination="residual_fixed_r", residual_tolerance=1e-6)
    srv = S.Server(rp, max_iterations=100)
    srv.submit(ds[0], 2)
    srv.submit(ds[1], 4)
    srv.run()
    # the tower was relaid out (boxes left after 2 ticks) at body offset 0 instead of 9
    assert [t["scenes"] for t in srv.ticks] == [2, 2, 1, 1]
    kept = int(srv.batch.t_cache_count.item())
    assert kept > 0
