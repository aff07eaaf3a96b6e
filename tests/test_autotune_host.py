"""The autotuner's search (no GPU): coordinate descent finds the minimum of a separable cost and never
proposes a setting rb_step would reject."""
import pytest


def test_coordinate_descent_finds_the_minimum_of_a_separable_cost():
    from rainbow_b200 import autotune as A
    target = {"fp32_small_slab": 16384, "fp32_mid_slab": 49152, "mid_blocks": 148 * 8, "narrow_blocks": 148 * 16,
              "narrow_threads": 128}
    proposed = []

    def cost(s):
        proposed.append(dict(s))
        return sum(abs(s[k] - target[k]) / target[k] for k in target)

    best, c, n = A.coordinate_descent(cost)
    assert best == target and c == 0.0
    assert all(A.valid(s) for s in proposed)
    assert n == len({tuple(sorted(s.items())) for s in proposed})   # every setting timed once


def test_apply_sets_the_rb_params_fields():
    from rainbow_b200 import autotune as A
    from rainbow_b200 import _native as N
    rp = N.RbParams()
    A.apply(rp, A.DEFAULTS)
    assert rp.fp32_small_slab == 28672 and rp.narrow_threads == 256 and rp.mid_blocks == 148 * 16


@pytest.mark.parametrize("small,mid,ok", [(28672, 57344, True), (57344, 57344, False), (2048, 40960, False),
                                          (16384, 65536, False)])
def test_validity_matches_the_library_bounds(small, mid, ok):
    from rainbow_b200 import autotune as A
    assert A.valid(dict(A.DEFAULTS, fp32_small_slab=small, fp32_mid_slab=mid)) == ok
