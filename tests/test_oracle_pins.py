"""The oracle's primitives against the known answers of the reference's own unit tests.

Each case restates an input and expected output of ``unit_tests/test_math_quaternion.py``,
``unit_tests/test_math_vector3.py``, ``unit_tests/test_geometry_grid3.py`` and
``unit_tests/test_random_graph_coloring.py`` (tolerances as ``rainbow/util/test_tools.py:9``: rtol = atol = 1e-8).
"""
import numpy as np
import pytest

TOL = dict(rtol=1e-8, atol=1e-8)


def test_quaternion_prod_against_definition(oracle_lib):
    # test_math_quaternion.py:31-85: q (x) conjugate(q) by definition 18.41
    for q in ([1, 2, 3, 4], [3, 1, 6, -4], [0.3, 0.1, 0.00006, -8]):
        q = np.array(q, dtype=np.float64)
        qc = q * np.array([1, -1, -1, -1])
        expected = np.empty(4)
        expected[0] = q[0] * qc[0] - np.dot(q[1:], qc[1:])
        expected[1:] = q[0] * qc[1:] + qc[0] * q[1:] + np.cross(q[1:], qc[1:])
        np.testing.assert_allclose(oracle_lib.quat_prod(q, qc), expected, **TOL)


def test_quaternion_rotate(oracle_lib):
    # test_math_quaternion.py:163-172: rotating x by 90 degrees about y gives -z
    radian = (0.5 * np.pi) / 2
    q = np.array([np.cos(radian), 0.0, np.sin(radian), 0.0])
    np.testing.assert_allclose(oracle_lib.quat_rotate(q, [1.0, 0.0, 0.0]), [0.0, 0.0, -1.0], **TOL)
    # test_math_quaternion.py:174-183: rotating x by 90 degrees about z gives y
    q = np.array([np.cos(radian), 0.0, 0.0, np.sin(radian)])
    np.testing.assert_allclose(oracle_lib.quat_rotate(q, [1.0, 0.0, 0.0]), [0.0, 1.0, 0.0], **TOL)


def test_quaternion_rotate_array(oracle_lib):
    # test_math_quaternion.py:450-467
    radian = (0.5 * np.pi) / 2
    q = np.array([np.cos(radian), 0.0, np.sin(radian), 0.0])
    rs = np.eye(3)
    expected = np.array([[0, 0, -1], [0, 1, 0], [1, 0, 0]], dtype=np.float64)
    np.testing.assert_allclose(oracle_lib.quat_rotate_array(q, rs), expected, **TOL)


def test_quaternion_to_matrix(oracle_lib):
    # test_math_quaternion.py:363-378 (theorem 18.44)
    radian = (0.5 * np.pi) / 2
    q = np.array([np.cos(radian), np.sin(radian), 0, 0])
    c, s = np.cos(radian), np.sin(radian)
    expected = np.array([[1, 0, 0], [0, 1 - 2 * s * s, -2 * c * s], [0, 2 * c * s, 1 - 2 * s * s]])
    np.testing.assert_allclose(oracle_lib.quat_to_matrix(q), expected, **TOL)


def test_quaternion_unit(oracle_lib):
    q = np.array([2.0, 2.0, 3.0, 4.0])
    np.testing.assert_allclose(oracle_lib.quat_unit(q), q / np.linalg.norm(q), **TOL)
    np.testing.assert_array_equal(oracle_lib.quat_unit(np.zeros(4)), [1.0, 0.0, 0.0, 0.0])


@pytest.mark.parametrize("n", [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0], [1.0, 1.0, 1.0], [0.3, -2.0, 0.7]])
def test_make_orthonormal_vectors(oracle_lib, n):
    # test_math_vector3.py:272-370: t, b, n form a right-handed orthonormal frame with n along the input
    t, b, nn = oracle_lib.make_orthonormal_vectors(n)
    n = np.asarray(n) / np.linalg.norm(n)
    np.testing.assert_allclose(nn, n, **TOL)
    for u, v in ((t, b), (t, nn), (b, nn)):
        assert abs(np.dot(u, v)) < 1e-12
    for u in (t, b, nn):
        assert abs(np.linalg.norm(u) - 1.0) < 1e-12
    np.testing.assert_allclose(np.cross(t, b), nn, **TOL)


def test_make_orthonormal_vectors_axis_choice(oracle_lib):
    # vector3.py:94-99: the tangent guess is the axis of the smallest |n_i|, later tests winning ties
    t, b, n = oracle_lib.make_orthonormal_vectors([0.0, 0.0, 1.0])
    # smallest components x and y tie; y wins -> t_guess = j, b = n x j = -i, t = b x n = j
    np.testing.assert_allclose(b, [-1.0, 0.0, 0.0], **TOL)
    np.testing.assert_allclose(t, [0.0, 1.0, 0.0], **TOL)


def _linear_grid(oracle_lib, I=5):
    # test_geometry_grid3.py:108-120: func(p) = p[0] on [-1, 1]^3, I = J = K = 5
    meta = oracle_lib.grid_meta([-1, -1, -1], [1, 1, 1], I, I, I)
    vals = np.zeros(I ** 3)
    sp = meta[6:9]
    for k in range(I):
        for j in range(I):
            for i in range(I):
                vals[i + I * (j + I * k)] = -1.0 + sp[0] * i
    return vals, meta


@pytest.mark.parametrize("p", [[0, 0, 0], [-0.5, -0.5, -0.5], [0.5, 0.5, 0.5], [-1, -1, -1], [1, 1, 1],
                               [-2, -2, -2], [2, 2, 2]])
def test_grid_value_and_gradient_linear_field(oracle_lib, p):
    # test_geometry_grid3.py:108-191: value reproduces p[0], gradient is (1, 0, 0), also outside the grid
    vals, meta = _linear_grid(oracle_lib)
    assert abs(oracle_lib.grid_value(vals, meta, p) - p[0]) < 1e-7
    np.testing.assert_allclose(oracle_lib.grid_gradient(vals, meta, p), [1.0, 0.0, 0.0], **TOL)


def test_grid_enclosing_cell(oracle_lib):
    # test_geometry_grid3.py:56-91: cell index with projection of outside points onto the border cells
    meta = oracle_lib.grid_meta([-1, -1, -1], [1, 1, 1], 5, 5, 5)
    assert oracle_lib.grid_cell(meta, [-1, -1, -1]) == (0, 0, 0)
    assert oracle_lib.grid_cell(meta, [1, 1, 1]) == (3, 3, 3)
    assert oracle_lib.grid_cell(meta, [-5, 0.1, 7]) == (0, 2, 3)
    assert oracle_lib.grid_cell(meta, [-0.4, -0.6, 0.6]) == (1, 0, 3)


def test_grid_is_inside(oracle_lib):
    # test_geometry_grid3.py:193-239: boundary width shrinks the accepted box
    meta = oracle_lib.grid_meta([-1, -1, -1], [1, 1, 1], 4, 4, 4)
    assert oracle_lib.grid_is_inside(meta, [0, 0, 0], 0.0)
    assert oracle_lib.grid_is_inside(meta, [1, 1, 1], 0.0)
    assert not oracle_lib.grid_is_inside(meta, [1.01, 0, 0], 0.0)
    assert not oracle_lib.grid_is_inside(meta, [0.6, 0, 0], 0.5)
    assert oracle_lib.grid_is_inside(meta, [0.4, -0.4, 0.4], 0.5)


def test_prox_sphere(oracle_lib):
    # prox_operators.py:14-34: zero when x_n <= 0, identity inside the ball, radial projection outside
    assert oracle_lib.prox_sphere(1.0, 2.0, 3.0, 0.5, 0.0) == (0.0, 0.0, 0.0)
    assert oracle_lib.prox_sphere(0.1, 0.1, 0.0, 0.5, 1.0) == (0.1, 0.1, 0.0)
    out = np.array(oracle_lib.prox_sphere(3.0, 4.0, 0.0, 0.5, 2.0))
    np.testing.assert_allclose(out, [0.6, 0.8, 0.0], **TOL)


def test_colouring_is_valid(oracle_lib):
    # test_random_graph_coloring.py:20-32 checks that neighbours get different colours; here contacts that
    # share a non-fixed body are neighbours
    rng = np.random.default_rng(4)
    n_bodies = 40
    fixed = np.zeros(n_bodies, np.uint8)
    fixed[0] = 1
    ids = rng.integers(0, n_bodies, size=(300, 2)).astype(np.int32)
    ids = ids[ids[:, 0] != ids[:, 1]]
    colour, nc = oracle_lib.colour_contacts(ids, fixed, n_bodies)
    assert nc == colour.max() + 1
    for c in range(nc):
        members = ids[colour == c]
        bodies = members[~fixed[members].astype(bool)]
        assert len(bodies) == len(np.unique(bodies)), "colour %d has two contacts on one body" % c
    # a path of contacts alternates two colours at most ... plus the greedy bound deg + 1
    path = np.array([[i, i + 1] for i in range(1, 20)], np.int32)
    colour, nc = oracle_lib.colour_contacts(path, fixed, n_bodies)
    assert nc <= 3


def test_coloured_order_is_a_valid_gauss_seidel_order(oracle_lib):
    """The coloured sweep visits colour classes in order; inside a class no two contacts share a non-fixed body,
    so the class order is a valid parallel schedule.  With the lattice scene the colouring needs far fewer
    classes than the serial order's dependency levels."""
    from conftest import load_fixture
    d = load_fixture("c1_boxes64")
    sc = oracle_lib.OracleScene(d)
    o = sc.step(scheme="rigid_gauss_seidel", ordering="coloured")
    ids, fixed = o["ids"], np.asarray(d["body_fixed"], np.uint8)
    colour, nc = oracle_lib.colour_contacts(ids, fixed, len(fixed))
    assert o["n_colours"] == nc
    for c in range(nc):
        bodies = [b for b in ids[colour == c].ravel() if not fixed[b]]
        assert len(bodies) == len(set(bodies))
