"""Launch-shape autotuner of the batched step.

The step's launch shapes -- the shared-memory slab of a warp team in the FP32 solve's two warp classes (which
also decides how many scenes share an SM), and the grids of the triangle-candidate and contact searches --
change speed only, never results (every kernel computes each scene's values in the same order whatever the
shape; ``tests/test_gpu_autotune.py`` checks the bits).  The best shapes depend on the batch: how many scenes,
how large, how many contacts.  :func:`tune` times candidates on the batch itself, from one saved state, by
coordinate descent (one knob at a time, the others held) and returns the fastest setting; :func:`apply` writes
it into an ``rb_params``.  Results are remembered per batch signature for the life of the process.
"""
import numpy as np

# knob -> candidate values (0 would mean the built-in default)
CANDIDATES = {
    "fp32_small_slab": [8192, 12288, 16384, 20480, 28672, 40960],
    "fp32_mid_slab": [40960, 49152, 57344],
    "mid_blocks": [148 * 4, 148 * 8, 148 * 16, 148 * 32],
    "narrow_blocks": [148 * 4, 148 * 8, 148 * 16],
    "narrow_threads": [128, 256],
}
DEFAULTS = {"fp32_small_slab": 28672, "fp32_mid_slab": 57344, "mid_blocks": 148 * 16, "narrow_blocks": 148 * 8,
            "narrow_threads": 256}

_memo = {}


def valid(setting):
    """The constraints rb_step checks: 4096 <= small slab < mid slab <= 57344."""
    return 4096 <= setting["fp32_small_slab"] < setting["fp32_mid_slab"] <= 57344


def apply(rb_params, setting):
    """Copy a setting into rb_params (in place) and return it."""
    for k, v in setting.items():
        setattr(rb_params, k, int(v))
    return rb_params


def coordinate_descent(cost, start=None, candidates=None, rounds=2):
    """Minimise cost(setting) one knob at a time over the candidate values, up to `rounds` passes or until a
    pass changes nothing.  Returns (best setting, best cost, number of evaluations)."""
    candidates = candidates or CANDIDATES
    best = dict(start or DEFAULTS)
    seen = {}

    def evaluate(s):
        key = tuple(sorted(s.items()))
        if key not in seen:
            seen[key] = cost(s)
        return seen[key]

    best_cost = evaluate(best)
    for _ in range(rounds):
        changed = False
        for knob, values in candidates.items():
            for v in values:
                trial = dict(best, **{knob: v})
                if trial == best or not valid(trial):
                    continue
                c = evaluate(trial)
                if c < best_cost:
                    best, best_cost, changed = trial, c, True
        if not changed:
            break
    return best, best_cost, len(seen)


def signature(world):
    """Batch signature the memo is keyed by: scenes, bodies (1 % buckets) and the largest scene."""
    nb = np.diff(world.scene_start)
    return (world.n_scenes, int(round(np.log(max(world.n_bodies, 1)) * 100)), int(nb.max()))


def tune(world, rb_params, steps=4, rounds=2, memo=True, repeats=3, start=None, knobs=None):
    """Fastest launch shapes for `world` stepped with `rb_params`: a trial times `steps` steps from the same
    saved state (warm-start cache included) `repeats` times and keeps the median.  ``start`` is the setting
    the descent starts from (the defaults otherwise) and ``knobs`` the knobs it varies (all otherwise).  The
    world is left in its saved state."""
    import torch
    # the best shapes depend on the solve's length too (a 100-sweep step is throughput-bound, a long one is
    # bound by its longest scene), so the memo key holds the sweep cap and the precision
    key = (signature(world), int(rb_params.max_iterations), int(rb_params.precision), steps,
           tuple(sorted((start or {}).items())), tuple(knobs or ())) if memo else None
    if key is not None and key in _memo:
        return dict(_memo[key][0]), _memo[key][1]
    x0, u0 = world.state()
    cache = (world.t_cache_key.clone(), world.t_cache_sol.clone(), world.t_cache_count.clone())

    def restore():
        world.set_state(x0, u0)
        world.t_cache_key.copy_(cache[0])
        world.t_cache_sol.copy_(cache[1])
        world.t_cache_count.copy_(cache[2])

    # size the work lists over the trial horizon first, so no trial repeats a step
    for _ in range(steps):
        world.step(rb_params)
    restore()
    stream = torch.cuda.current_stream(world.device)

    def cost(setting):
        rp = apply(type(rb_params).from_buffer_copy(rb_params), setting)
        restore()
        world.launch(rp)                      # warm
        times = []
        for _ in range(repeats):
            restore()
            torch.cuda.synchronize(world.device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                world.launch(rp)
            e1.record(stream)
            torch.cuda.synchronize(world.device)
            times.append(e0.elapsed_time(e1) / steps)
        return float(np.median(times))

    cands = {k: v for k, v in CANDIDATES.items() if knobs is None or k in knobs}
    best, best_ms, n = coordinate_descent(cost, start=start, candidates=cands, rounds=rounds)
    restore()
    info = {"ms_per_step": best_ms, "default_ms_per_step": cost(DEFAULTS), "trials": n}
    restore()
    torch.cuda.synchronize(world.device)
    if key is not None:
        _memo[key] = (dict(best), info)
    return best, info
