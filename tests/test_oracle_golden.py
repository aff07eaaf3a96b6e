"""The oracle pinned against the reference itself: every step of every golden fixture, bit for bit.

The fixtures were recorded by running the reference step (tests/golden/make_golden.py).  Each step starts from
the reference's state after the previous step, so a difference is attributed to the step where it appears.
"""
import numpy as np
import pytest

from conftest import FIXTURES, load_fixture, step_slice


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_reference_step_by_step(oracle_lib, name):
    d = load_fixture(name)
    sc = oracle_lib.OracleScene(d)
    N = sc.n_bodies
    for s in range(int(d["steps"])):
        if s > 0:
            x = d["step_x"][s - 1].reshape(N, 7)
            u = d["step_u"][s - 1].reshape(N, 6)
            sc.r[:], sc.q[:], sc.v[:], sc.w[:] = x[:, :3], x[:, 3:], u[:, :3], u[:, 3:]
        o = sc.step(dt=float(d["step_dt"][s]))
        np.testing.assert_array_equal(o["ids"], step_slice(d, "contacts_ids", s), err_msg="step %d contact ids" % s)
        for key, ref in (("p", "contacts_p"), ("n", "contacts_n"), ("g", "contacts_g"), ("b", "b"), ("diag", "diag"),
                         ("sol", "sol")):
            np.testing.assert_array_equal(o[key].ravel(), step_slice(d, ref, s).ravel(), err_msg="step %d %s" % (s, key))
        assert o["iterations"] == d["step_iterations"][s]
        assert o["exitcode"] == d["step_exitcode"][s]
        assert o["post_iterations"] == d["step_post_iterations"][s]
        np.testing.assert_array_equal(o["delta_u_ext"], d["step_delta_u_ext"][s])
        np.testing.assert_array_equal(o["x"], d["step_x"][s], err_msg="step %d x" % s)
        np.testing.assert_array_equal(o["u"], d["step_u"][s], err_msg="step %d u" % s)


def test_oracle_free_run_matches_reference(oracle_lib):
    """Twelve steps chained inside the oracle stay bit-identical to the reference's trajectory."""
    d = load_fixture("boxes8")
    sc = oracle_lib.OracleScene(d)
    for s in range(int(d["steps"])):
        o = sc.step(dt=float(d["step_dt"][s]))
    np.testing.assert_array_equal(o["x"], d["step_x"][-1])
    np.testing.assert_array_equal(o["u"], d["step_u"][-1])


@pytest.mark.parametrize("scheme", ["gauss_seidel", "parallel_jacobi", "parallel_jacobi_hybrid"])
def test_oracle_proximal_contact_schemes(oracle_lib, scheme):
    """The proximal_contact solvers (solver_interface.py, jacobi_solver.py, gauss_seidel_solver.py) on one
    contact problem: sixty iterations without convergence, bit-identical solutions."""
    d = load_fixture("solvers")
    sc = oracle_lib.OracleScene(d)
    o = sc.step(scheme=scheme)
    np.testing.assert_array_equal(o["ids"], d["contacts_ids"])
    np.testing.assert_array_equal(o["b"], d["b"])
    np.testing.assert_array_equal(o["sol"], d["sol_" + scheme])
    assert o["iterations"] == d["iterations_" + scheme]
    assert o["exitcode"] == d["exitcode_" + scheme]


@pytest.mark.parametrize("name", ["hinges", "hinges_stab"])
def test_oracle_hinges_match_reference_step_by_step(oracle_lib, name):
    """Hinge chains (constraints/hinges.py), one with contacts against a ledge and one with pre-stabilisation:
    the hinge problem's b, Delassus diagonal and solution, the solver statistics and the state, bit for bit."""
    d = load_fixture(name)
    sc = oracle_lib.OracleScene(d)
    N = sc.n_bodies
    for s in range(int(d["steps"])):
        if s > 0:
            x = d["step_x"][s - 1].reshape(N, 7)
            u = d["step_u"][s - 1].reshape(N, 6)
            sc.r[:], sc.q[:], sc.v[:], sc.w[:] = x[:, :3], x[:, 3:], u[:, :3], u[:, 3:]
        o = sc.step(dt=float(d["step_dt"][s]))
        np.testing.assert_array_equal(o["ids"], step_slice(d, "contacts_ids", s), err_msg="step %d contact ids" % s)
        for key, ref in (("b", "b"), ("diag", "diag"), ("sol", "sol"), ("hinge_b", "hinge_b"),
                         ("hinge_diag", "hinge_diag"), ("hinge_sol", "hinge_sol")):
            np.testing.assert_array_equal(o[key].ravel(), step_slice(d, ref, s).ravel(), err_msg="step %d %s" % (s, key))
        assert (o["iterations"], o["exitcode"]) == (d["step_iterations"][s], d["step_exitcode"][s]), s
        np.testing.assert_array_equal(o["x"], d["step_x"][s], err_msg="step %d x" % s)
        np.testing.assert_array_equal(o["u"], d["step_u"][s], err_msg="step %d u" % s)


def test_oracle_warm_start_cache():
    """Warm start in the oracle: contact keys come out ascending, a step with an empty cache equals a cold
    step, and warm-started solves meet the residual tolerance in fewer sweeps over a trajectory."""
    from oracle import oracle as O
    d = load_fixture("c1_boxes64")
    cold, warm = O.OracleScene(d), O.OracleScene(d)
    for sc in (cold, warm):
        sc.set_param("max_iterations", 2000)
    kw = dict(tol_mode=2, tol=1e-6, residual_interval=1)
    a, b = cold.step(**kw), warm.step(warm_start=True, **kw)
    np.testing.assert_array_equal(a["sol"], b["sol"])
    np.testing.assert_array_equal(a["x"], b["x"])
    sweeps = {False: a["iterations"], True: b["iterations"]}
    for _ in range(6):
        a, b = cold.step(**kw), warm.step(warm_start=True, **kw)
        assert a["exitcode"] == 3 and b["exitcode"] == 3
        sweeps[False] += a["iterations"]
        sweeps[True] += b["iterations"]
        k = b["keys"]
        assert len(k) == b["n_contacts"]
        assert all(tuple(k[i]) < tuple(k[i + 1]) for i in range(len(k) - 1))
        lo = np.minimum(b["ids"][:, 0], b["ids"][:, 1]).astype(np.int64)
        hi = np.maximum(b["ids"][:, 0], b["ids"][:, 1]).astype(np.int64)
        np.testing.assert_array_equal(k[:, 0], (lo << 31) | hi)
        np.testing.assert_array_equal(k[:, 1] >> 30, (b["ids"][:, 1] == hi).astype(np.int64))
    assert sweeps[True] < sweeps[False]
