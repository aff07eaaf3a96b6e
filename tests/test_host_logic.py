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
