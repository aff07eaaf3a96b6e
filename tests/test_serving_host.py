"""Host side of the serving loop (no GPU): shape library deduplication and the body layout of a batch."""
import numpy as np

from conftest import load_fixture


def test_pack_blocks_matches_pack_scenes_body_layout():
    from rainbow_b200 import serving as S
    from rainbow_b200 import world as W
    ds = [load_fixture(n) for n in ("boxes8", "spheres", "tower6", "c1_boxes64")]
    lib = S.ShapeLibrary("cpu")
    blocks = [S.SceneBlock(d, lib) for d in ds]
    P = S.pack_blocks(blocks, lib)
    R = W.pack_scenes(ds)
    # the fixtures repeat shapes (ground, unit box): the library keeps one copy of each distinct shape
    assert len(lib.V) < R["n_shapes"]
    for b, (ls, rs) in enumerate(zip(P["body_shape"], R["body_shape"])):
        v0, v1 = R["shape_v_off"][rs], R["shape_v_off"][rs + 1]
        np.testing.assert_array_equal(lib.V[ls], R["shape_V"][3 * v0:3 * v1], err_msg="body %d" % b)
        g0, g1 = R["shape_g_off"][rs], R["shape_g_off"][rs + 1]
        np.testing.assert_array_equal(lib.G[ls], R["shape_grid"][g0:g1], err_msg="body %d" % b)
    for key in ("scene_start", "body_mass", "body_inertia", "body_fixed", "body_material",
                "force_ptr", "force_list", "scene_force_start", "force_kind", "force_params",
                "scene_material_offset", "scene_material_count", "material_mu", "material_eps"):
        np.testing.assert_array_equal(P[key], R[key], err_msg=key)
    assert (P["n_body_vertices"], P["n_body_triangles"], P["n_clusters"]) == \
        (int(R["body_v0"][-1]), int(R["body_t0"][-1]), int(R["body_c0"][-1]))
    x0 = np.concatenate([b.x0 for b in blocks]).reshape(-1)
    np.testing.assert_array_equal(x0, R["x"])


def test_shape_library_stores_a_shape_once_across_scenes():
    from rainbow_b200 import serving as S
    d = load_fixture("boxes8")
    lib = S.ShapeLibrary("cpu")
    a = lib.add(d)
    b = lib.add(dict(d))                         # the same shapes again (content keys): no new entries
    np.testing.assert_array_equal(a, b)
    assert len(lib.V) == len(np.asarray(d["shape_v_off"])) - 1
