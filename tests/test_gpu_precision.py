"""Precision stress: the 32-high box tower with alternating masses 1 and 1000 (mass ratio 1e3), mu 0.6,
dt 0.005, stepped in FP64, FP32 + FP64 refinement and FP32 only.  The FP32 modes must track the FP64
trajectory while the tower is intact (position drift <= 1e-6 m over the first 50 steps) and meet the 1e-6
residual tolerance as often as the FP64 solve (within 5 % of the steps; median residual at most the
tolerance or twice the FP64 median).  Later the tower
collapses (its boxes sink into each other, as in the reference) and the trajectories of unconverged solves
part ways; the bench's tower32 workload reports residual and drift per step over 500 steps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(arrays, params, precision, steps):
    from rainbow_b200 import world as W
    w = W.DeviceWorld(arrays, max_iterations=100)
    rp = W.make_rb_params(params, precision=precision, termination="residual_fixed_r", residual_tolerance=1e-6,
                          residual_interval=4, warm_start=True)
    xs, res = [], []
    for _ in range(steps):
        w.step(rp)
        xs.append(w.state()[0][:, :3].copy())
        res.append(w.stats()[0].residual)
    return np.array(xs), np.array(res)


def test_fp32_modes_track_fp64_on_the_mass_ratio_tower():
    from rainbow_b200 import engine_io, scenes
    from rainbow_b200 import world as W
    arrays = engine_io.scene_arrays(scenes.box_tower(32))
    params = W.params_from_vector(arrays["params"])
    x64, r64 = _run(arrays, params, "fp64", 50)
    for mode in ("fp32_refine", "fp32"):
        xm, rm = _run(arrays, params, mode, 50)
        drift = np.abs(xm - x64).max()
        assert drift <= 1e-6, (mode, drift)
        # converged steps: the same share meets the 1e-6 tolerance; the rest: residuals of the FP64 size
        assert np.mean(rm <= 1e-6) >= np.mean(r64 <= 1e-6) - 0.05, (mode, np.mean(rm <= 1e-6), np.mean(r64 <= 1e-6))
        assert np.median(rm) <= max(1e-6, 2.0 * np.median(r64)), (mode, np.median(rm), np.median(r64))


def test_fp32_solve_of_a_scene_with_more_bodies_than_a_slab_holds():
    """4097 bodies (the 16^3 box/sphere lattice on a ground): too many for one SM's shared memory, so the FP32
    phase keeps contact rows and body records in global memory.  It must run (FP32 sweeps > 0) and agree with
    the FP64 solve of the same step to a small fraction of the velocity scale, at a residual of the same
    size."""
    from rainbow_b200 import engine_io, scenes
    from rainbow_b200 import world as W
    arrays = engine_io.scene_arrays(scenes.mixed_lattice(n=16, resolution=16))
    params = W.params_from_vector(arrays["params"])
    kw = dict(termination="residual_fixed_r", residual_tolerance=1e-6, residual_interval=4)
    w = W.DeviceWorld(arrays, max_iterations=100)
    for _ in range(30):
        w.step(W.make_rb_params(params, **kw))
    x0, u0 = w.state()
    out = {}
    for mode in ("fp64", "fp32_refine"):
        w.set_state(x0, u0)
        w.step(W.make_rb_params(params, precision=mode, **kw))
        out[mode] = (w.state()[1], w.stats()[0])
    (u64, s64), (u32, s32) = out["fp64"], out["fp32_refine"]
    assert s64.n_contacts > 0 and s32.fp32_sweeps > 0
    assert np.abs(u32 - u64).max() <= 1e-3 * np.abs(u64).max()
    assert s32.residual <= 2.0 * s64.residual + 1e-6


def _s32_bytes(K, nb):
    """Shared memory of a scene's whole FP32 copy (the solver's size classes): 48 floats per contact, its
    level-order position (2 B), body list entries (8 B) and body index pair (4 B), 16 floats per body, level
    and list starts; each piece rounded up to 16 bytes."""
    a = lambda v: (v + 15) // 16 * 16  # noqa: E731
    return a(192 * K) + a(2 * K) + a(8 * K) + a(64 * nb) + a(4 * K) + a(2 * (K + 1)) + a(2 * (nb + 1))


def test_fp32_solve_of_scenes_whose_rows_live_in_l2():
    """Piles of 1500-2048 bodies: their contact rows no longer fit one SM's shared memory (more than 224 KB),
    so the FP32 phase keeps the rows in global memory and the body records on chip, in 512-thread teams.  The
    step must agree with the FP64 solve of the same step to a small fraction of the velocity scale, at a
    residual of the same size."""
    from rainbow_b200 import scenes
    from rainbow_b200 import world as W
    arrays, params = scenes.batch_arrays(n_scenes=2, seed=1, pool=8, body_range=(1500, 2048), resolution=16,
                                         device="cuda:0", ground=40.0)
    kw = dict(termination="residual_fixed_r", residual_tolerance=1e-6, residual_interval=4)
    w = W.DeviceWorld(arrays, max_iterations=100)
    for _ in range(100):
        w.step(W.make_rb_params(params, precision="fp32_refine", **kw))
    x0, u0 = w.state()
    out = {}
    for mode in ("fp64", "fp32_refine"):
        w.set_state(x0, u0)
        w.step(W.make_rb_params(params, precision=mode, **kw))
        out[mode] = (w.state()[1], w.stats())
    (u64, s64), (u32, s32) = out["fp64"], out["fp32_refine"]
    nb = [len(a["body_mass"]) for a in arrays]
    in_l2 = [i for i, s in enumerate(s32) if _s32_bytes(s.n_contacts, nb[i]) > 224 * 1024 and 64 * nb[i] < 150 * 1024]
    assert in_l2, [(s.n_contacts, n) for s, n in zip(s32, nb)]
    for i in in_l2:
        b0, b1 = w.scene_start[i], w.scene_start[i + 1]
        assert s32[i].fp32_sweeps > 0
        assert np.abs(u32[b0:b1] - u64[b0:b1]).max() <= 1e-3 * np.abs(u64[b0:b1]).max()
        assert s32[i].residual <= 2.0 * s64[i].residual + 1e-6


def test_fp32_contact_search_finds_the_fp64_contacts():
    """The FP32 modes run the contact search's lookups on the FP32 grid copy, decide near-ties (exact ties of
    coplanar box corners included) on FP64 lookups and accept contacts in FP64.  On 16 scenes of the batched
    workload after a 20-step pre-roll, a profiled step finds exactly the FP64 step's contacts (ids, points,
    normals, gaps), most of its lookups are FP32, and the self-check against the plain FP64 search counts no
    flipped decision."""
    from rainbow_b200 import scenes
    from rainbow_b200 import world as W
    arrays, params = scenes.batch_arrays(n_scenes=16, seed=0, pool=64, resolution=32, device="cuda:0")
    w = W.DeviceWorld(arrays, max_iterations=100)
    kw = dict(termination="residual_fixed_r", residual_tolerance=1e-6, residual_interval=4)
    for _ in range(20):
        w.step(W.make_rb_params(params, **kw))
    x0, u0 = w.state()
    out = {}
    for mode in ("fp64", "fp32_refine"):
        w.set_state(x0, u0)
        w.step(W.make_rb_params(params, precision=mode, profiling=3, **kw))
        out[mode] = (w.stats(), w.contacts())
    (s64, c64), (s32, c32) = out["fp64"], out["fp32_refine"]
    for key in ("ids", "p", "n", "g"):
        np.testing.assert_array_equal(c32[key], c64[key], err_msg=key)
    l32, l64 = sum(s.n_grid_lookups32 for s in s32), sum(s.n_grid_lookups for s in s32)
    assert sum(s.n_grid_lookups32 for s in s64) == 0 and l32 > l64
    assert sum(s.n_search_flips + s.n_accept_flips for s in s32) == 0


@pytest.mark.parametrize("scheme", ["parallel_jacobi", "parallel_jacobi_hybrid"])
def test_fp32_jacobi_agrees_with_fp64_jacobi(scheme):
    """Proximal Jacobi (jacobi_solver.py:41-79) in FP32 + FP64 refinement against the FP64 Jacobi solve of the
    same step: the same share of steps meets the 1e-6 residual, and the velocities agree to 1e-4 of their scale
    on the 64-box lattice over 10 steps from the same states."""
    from rainbow_b200 import world as W
    from conftest import load_fixture
    d = load_fixture("c1_boxes64")
    p = W.params_from_vector(d["params"])
    p["max_iterations"] = 3000
    w = W.DeviceWorld(d, max_iterations=3000)
    kw = dict(scheme=scheme, termination="residual_fixed_r", residual_tolerance=1e-6, residual_interval=4,
              warm_start=True)
    met = {"fp64": 0, "fp32_refine": 0}
    for _ in range(10):
        x0, u0 = w.state()
        cache = (w.t_cache_key.clone(), w.t_cache_sol.clone(), w.t_cache_count.clone())
        out = {}
        for mode in ("fp32_refine", "fp64"):      # FP64 last: the trajectory follows FP64
            w.set_state(x0, u0)
            w.t_cache_key.copy_(cache[0]); w.t_cache_sol.copy_(cache[1]); w.t_cache_count.copy_(cache[2])
            w.step(W.make_rb_params(p, precision=mode, **kw))
            st = w.stats()[0]
            met[mode] += st.exitcode == 3
            out[mode] = (w.state()[1], st)
        (u32, s32), (u64, s64) = out["fp32_refine"], out["fp64"]
        if s64.n_contacts:
            assert s32.fp32_sweeps > 0
            assert np.abs(u32 - u64).max() <= 1e-4 * max(1e-3, np.abs(u64).max())
    assert met["fp32_refine"] >= met["fp64"] - 1
