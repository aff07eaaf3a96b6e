"""Launch shapes change speed only: the same batch stepped with different slabs and grids gives identical
bits (FP32 + refinement and FP64), and the tuner returns a valid setting no slower than the default."""
import numpy as np
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32_refine", "fp64"])
def test_launch_shapes_do_not_change_results(precision):
    from rainbow_b200 import autotune as A
    from rainbow_b200 import world as W
    ds = [load_fixture(n) for n in ("boxes8", "spheres", "tower6", "c1_boxes64")]
    params = W.params_from_vector(ds[2]["params"])
    base = W.make_rb_params(params, warm_start=True, termination="residual_fixed_r", residual_tolerance=1e-6,
                            precision=precision)
    shapes = [A.DEFAULTS,
              {"fp32_small_slab": 8192, "fp32_mid_slab": 40960, "mid_blocks": 37, "narrow_blocks": 5,
               "narrow_threads": 64}]
    results = []
    for sh in shapes:
        w = W.DeviceWorld(ds, max_iterations=100)
        rp = A.apply(type(base).from_buffer_copy(base), sh)
        for _ in range(3):
            w.step(rp)
        results.append((w.state(), w.contacts()["sol"]))
    (xa, ua), sa = results[0]
    (xb, ub), sb = results[1]
    np.testing.assert_array_equal(xb, xa)
    np.testing.assert_array_equal(ub, ua)
    np.testing.assert_array_equal(sb, sa)


def test_tuner_returns_a_valid_setting():
    from rainbow_b200 import autotune as A
    from rainbow_b200 import world as W
    ds = [load_fixture(n) for n in ("boxes8", "spheres", "tower6", "c1_boxes64")] * 4
    params = W.params_from_vector(ds[2]["params"])
    rp = W.make_rb_params(params, warm_start=True, termination="residual_fixed_r", residual_tolerance=1e-6,
                          precision="fp32_refine")
    w = W.DeviceWorld(ds, max_iterations=100)
    w.step(rp)
    x0, u0 = w.state()
    best, info = A.tune(w, rp, steps=2, rounds=1, memo=False)
    assert A.valid(best) and info["trials"] >= 2
    assert info["ms_per_step"] <= info["default_ms_per_step"] * 1.5   # timing noise allowance
    x1, u1 = w.state()
    np.testing.assert_array_equal(x1, x0)        # the world is back in its saved state
