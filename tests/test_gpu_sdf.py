"""Signed distance grids built on the GPU (grid3.py:320 create_signed_distance, whose igl.signed_distance call
at grid3.py:338 rb_signed_distance_grid replaces) against the grids the reference step consumed in the golden
fixtures, and the batched construction of the per-body workload."""
import numpy as np
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu


def _shapes(d):
    sv, st, sg = (np.asarray(d[k]) for k in ("shape_v_off", "shape_t_off", "shape_g_off"))
    V, T, G = np.asarray(d["shape_V"]).reshape(-1, 3), np.asarray(d["shape_T"]).reshape(-1, 3), np.asarray(d["shape_grid"]).ravel()
    meta = np.asarray(d["shape_grid_meta"]).reshape(-1, 12)
    for k in range(len(sv) - 1):
        yield V[sv[k]:sv[k + 1]], T[st[k]:st[k + 1]], G[sg[k]:sg[k + 1]], meta[k]


def _grid_on_gpu(V, T, meta):
    import ctypes
    import torch
    from rainbow_b200 import _native as N
    tV = torch.from_numpy(np.ascontiguousarray(V, np.float64)).cuda()
    tT = torch.from_numpy(np.ascontiguousarray(T, np.int32)).cuda()
    tM = torch.from_numpy(np.ascontiguousarray(meta, np.float64)).cuda()
    n = int(meta[9] * meta[10] * meta[11])
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    N.check(N.load().rb_signed_distance_grid(tV.data_ptr(), len(V), tT.data_ptr(), len(T), tM.data_ptr(),
                                             out.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
            "rb_signed_distance_grid")
    return out.cpu().numpy()


@pytest.mark.parametrize("name", ["spheres", "c1_boxes64", "boxes8", "tower6"])
def test_gpu_grids_match_the_grids_the_reference_consumed(name):
    """Every shape of the fixture (boxes of several sizes, the ground slab, 16 x 16 spheres): the GPU grid equals
    the grid the reference's own step used, node for node, to 1e-12 (the fixtures' grids came from the NumPy
    restatement of igl.signed_distance: closest point by Ericson's case analysis, sign by the generalized
    winding number)."""
    d = load_fixture(name)
    n = 0
    for V, T, G, meta in _shapes(d):
        got = _grid_on_gpu(V, T, meta)
        np.testing.assert_allclose(got, G, rtol=0.0, atol=1e-12)
        n += 1
    assert n >= 2


def test_batched_grids_equal_single_grids():
    """rb_signed_distance_grids over several meshes equals rb_signed_distance_grid on each, bit for bit."""
    from rainbow_b200 import geometry as GEO
    from rainbow_b200.types import Grid
    meshes = [GEO.create_box(1.0, 0.6, 2.0), GEO.create_sphere(0.7, 16, 16), GEO.create_box(24.0, 1.0, 24.0),
              GEO.create_sphere(0.3, 8, 8)]
    Vs, Ts, metas = [], [], []
    for i, (V, T) in enumerate(meshes):
        V = np.asarray(V, np.float64)
        res = (17, 32, 9, 20)[i]
        metas.append(Grid(V.min(0) - 0.2, V.max(0) + 0.2, res, res + 1, res + 2).meta())
        Vs.append(V)
        Ts.append(np.asarray(T, np.int32))
    values, g_off = GEO.signed_distance_grids(Vs, Ts, metas)
    values = values.cpu().numpy()
    for i in range(len(meshes)):
        np.testing.assert_array_equal(values[g_off[i]:g_off[i + 1]], _grid_on_gpu(Vs[i], Ts[i], metas[i]))


def test_per_body_workload_steps_like_the_oracle(oracle_lib):
    """The batch workload with a shape and grid per body: every body's grid is its own mesh's grid, masses scale
    with size, and the batch steps bit-identically to the oracle on host copies of the same scenes."""
    from rainbow_b200 import scenes, world as W
    arrays, params = scenes.batch_arrays(n_scenes=3, seed=5, pool=None, body_range=(8, 24), resolution=16,
                                         device="cuda:0")
    for a in arrays:
        host = {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in a.items()}
        shapes = list(_shapes(host))
        assert len(shapes) == len(a["body_mass"])          # the ground and one shape per body
        for V, T, G, meta in shapes[1:4]:
            np.testing.assert_array_equal(G, _grid_on_gpu(V, T, meta))
        assert len(set(np.round(a["body_mass"][1:], 9))) == len(a["body_mass"]) - 1   # sizes differ per body
    world = W.DeviceWorld(arrays, device="cuda:0", max_iterations=100)
    ors = [oracle_lib.OracleScene({k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in a.items()})
           for a in arrays]
    rp = W.make_rb_params(params)
    for s in range(8):
        assert world.step(rp) == 0
        x, u = world.state()
        for i, sc in enumerate(ors):
            o = sc.step()
            b0, b1 = world.scene_start[i], world.scene_start[i + 1]
            np.testing.assert_array_equal(x[b0:b1].ravel(), o["x"], err_msg="step %d scene %d" % (s, i))
            np.testing.assert_array_equal(u[b0:b1].ravel(), o["u"], err_msg="step %d scene %d" % (s, i))


def test_per_body_scenes_do_not_depend_on_which_others_are_built():
    """A multi-GPU rank builds only its share of the per-body workload: a selected scene's arrays (shapes,
    grids, bodies) equal the same scene built with all the others, and the counts without building match."""
    from rainbow_b200 import scenes
    every, _ = scenes.batch_arrays_per_body(n_scenes=5, seed=2, body_range=(8, 16), resolution=8, device="cuda:0")
    some, _ = scenes.batch_arrays_per_body(n_scenes=5, seed=2, body_range=(8, 16), resolution=8, device="cuda:0",
                                           select=[1, 4])
    assert [len(a["body_mass"]) for a in every] == scenes.per_body_counts(5, 2, (8, 16))
    for a, b in zip([every[1], every[4]], some):
        for k in a:
            va = a[k].cpu().numpy() if hasattr(a[k], "cpu") else np.asarray(a[k])
            vb = b[k].cpu().numpy() if hasattr(b[k], "cpu") else np.asarray(b[k])
            np.testing.assert_array_equal(va, vb, err_msg=k)
