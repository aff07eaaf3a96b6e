#!/usr/bin/env python
"""Benchmark of the prox_rigid_bodies time step on B200: one JSON line on stdout (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]
                    [--max-iterations M]

Workloads (synthetic, seeded; the shapes go through the reference-compatible set-up chain):
  batch1024  1024 independent scenes, 8..256 bodies each (log-uniform), random boxes (side U(0.5, 2)) and spheres
             (radius U(0.25, 1), 16 x 16 sweep) with random orientations, density 1000, mu U(0.2, 0.8) per scene,
             on a fixed ground box; SDF resolution 32; dt 0.01 (default).  --shapes pool draws the sizes from a
             pool of 64 boxes + 64 spheres shared by all scenes; --shapes per-body gives every body a shape and
             signed distance grid of its own (the configuration as stated)
  mixed4096  one scene of 4096 bodies (16^3 lattice, spacing 1.2): alternating unit boxes and r = 0.5 spheres,
             random orientations, density 1000, on a fixed ground box; SDF resolution 64
  boxes64    one scene of 64 unit boxes (4^3 lattice, spacing 1.05, jitter +-0.02) on a 20 x 1 x 20 ground
  tower32    the precision stress alone: 32-box tower, masses 1 / 1000, FP64 vs FP32 + FP64 refinement vs FP32
A step advances every scene of the workload by one semi-implicit time step.  Bodies start in the air; a
pre-roll of --pre-roll untimed steps (at the configuration's own 100-iteration limit) lets them land.

Equal residual.  Every solve of every arm (batched, plain one-scene-per-launch FP64, served, CPU) stops at the
same complementarity residual (--tolerance 1e-6, evaluated in FP64) or at --max-iterations sweeps, whichever
comes first, with the same solver; the line reports how many scenes met the tolerance in each arm and the
residuals of those that did not.  The same measurement at the configuration's own 100-sweep limit is
reported as a second, labelled block (at_100_sweeps).

The metric is scene-steps/s with the p50/p99 step latency, batched and served, against the plain FP64 step.
Scenes do not exchange data: with --gpus N every rank steps its own share (weak scaling, no collective on the
data path) and the value is the total over the max-over-ranks time.

--impl reference times the CPU restatement of the reference step (oracle/rb_oracle.c) on a bounded,
stratified sample of the same workload on all host cores.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM bytes of a phase's kernels per step, from ncu captures of this build (dram__bytes_read.sum +
# dram__bytes_write.sum), keyed by the phase's kernel and the (workload, precision, sweep cap) they hold for.
# k_solve_fp32: 5.84 MB for the four size-class launches of one step of the first 128 scenes (3343 contacts),
# scaled by contacts to the 1024-scene step (78,787 contacts): the traffic is the per-contact copy-in, the FP64
# corrections and the write-back, all proportional to the contacts.
# k_narrow: 66.1 MB for one launch on the first 128 scenes (152,968 candidates) with a grid per body, scaled by
# candidates to the 1024-scene step (4,374,974 candidates).
PROFILED_DRAM_BYTES = {
    "k_solve_fp32": (138_000_000, ("batch_1024_scenes_shape_per_body", "fp32_refine", 4000)),
    "k_narrow": (1_890_000_000, ("batch_1024_scenes_shape_per_body", "fp32_refine", 4000)),
}
# the phases rb_profile_times reports, in its order
PHASE_NAMES = ["bodies_bvh", "pairs_candidates", "contact_search", "dedup", "contact_setup_solve", "integrate", "total"]
EQUAL_RESIDUAL_SWEEPS = 4000   # default sweep cap of the equal-residual measurement


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batch1024", choices=["batch1024", "mixed4096", "boxes64", "tower32"])
    ap.add_argument("--shapes", default="per-body", choices=["pool", "per-body"],
                    help="batch1024: sizes from a shared pool of 64 + 64 shapes, or a shape and SDF per body")
    ap.add_argument("--scheme", default="rigid_gauss_seidel")
    ap.add_argument("--termination", default="residual_fixed_r", choices=["residual_fixed_r", "residual", "merit"])
    ap.add_argument("--scenes", type=int, default=1024, help="scenes of the batch1024 workload")
    ap.add_argument("--tolerance", type=float, default=1e-6)
    ap.add_argument("--max-iterations", type=int, default=EQUAL_RESIDUAL_SWEEPS,
                    help="sweep cap of every solve of every arm (the equal-residual measurement)")
    ap.add_argument("--pre-roll", type=int, default=60)
    ap.add_argument("--plain-scenes", type=int, default=16,
                    help="scenes (stratified by body count) of the one-scene-per-launch baseline")
    ap.add_argument("--plain-steps", type=int, default=3, help="timed steps per plain scene")
    ap.add_argument("--no-warm-start", action="store_true", help="start every solve from zero impulses")
    ap.add_argument("--precision", default="fp32_refine", choices=["fp64", "fp32_refine", "fp32"],
                    help="precision of the batched solve (the plain baseline is always FP64)")
    ap.add_argument("--residual-interval", type=int, default=4)
    ap.add_argument("--ordering", default="serial", choices=["serial", "coloured"],
                    help="contact order of the Gauss-Seidel sweeps (both arms use the same)")
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="budget of the CPU baseline sample")
    ap.add_argument("--cpu-scenes", type=int, default=64, help="scenes in the CPU baseline sample (stratified)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plugin", action="store_true",
                    help="skip the e2e run through api.simulate_batch on engine objects")
    ap.add_argument("--no-autotune", action="store_true", help="keep the built-in launch shapes")
    ap.add_argument("--no-100", action="store_true", help="skip the 100-sweep block")
    ap.add_argument("--no-configs", action="store_true", help="skip the C1 / C2 / C4 sub-results")
    ap.add_argument("--serve-seconds", type=float, default=20.0,
                    help="wall time of the serving run (Poisson arrivals, continuous batching); 0 skips it")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="request arrival rate (requests/s)")
    ap.add_argument("--serve-max-bodies", type=int, default=393216,
                    help="resident-body cap of the server (its step-latency target)")
    ap.add_argument("--serve-templates", type=int, default=192, help="distinct scenes the requests draw from")
    ap.add_argument("--serve-plain-scenes", type=int, default=8)
    return ap.parse_args()


# --------------------------------------------------------------------------------------------------------------
# workloads
# --------------------------------------------------------------------------------------------------------------
def build_workload(name, device, n_scenes=1024, shapes="pool", select=None):
    """The workload's scene arrays (for batch1024 only the scenes in `select`, when given)."""
    from rainbow_b200 import engine_io, scenes
    if name == "batch1024":
        pool = 64 if shapes == "pool" else None
        if pool is None:
            arrays, params = scenes.batch_arrays_per_body(n_scenes=n_scenes, seed=0, resolution=32, device=device,
                                                          select=select)
            bodies = sum(scenes.per_body_counts(n_scenes, 0))
        else:
            arrays, params = scenes.batch_arrays(n_scenes=n_scenes, seed=0, pool=pool, resolution=32, device=device)
            bodies = sum(len(a["body_mass"]) for a in arrays)
            if select is not None:
                arrays = [arrays[i] for i in select]
        cfg = {"workload": "batch_%d_scenes_%s" % (n_scenes, "shape_pool" if pool else "shape_per_body"),
               "scenes": n_scenes, "bodies": int(bodies),
               "bodies_per_scene": "8..256",
               "shapes": ("boxes side U(0.5,2), spheres r U(0.25,1) 16x16, "
                          + ("sizes from a pool of 64+64 shapes" if pool else "a shape and SDF per body")),
               "sdf_resolution": 32, "dt": 0.01}
        return arrays, params, cfg, None
    if name == "mixed4096":
        engine = scenes.mixed_lattice(n=16, spacing=1.2, resolution=64, seed=0, device=device)
        cfg = {"workload": "mixed_lattice_4096", "scenes": 1, "bodies": 4097,
               "shapes": "box 1x1x1 / sphere r=0.5 16x16", "sdf_resolution": 64, "dt": 0.01}
    else:
        engine = scenes.box_lattice(n=4, spacing=1.05, jitter=0.02, resolution=32, seed=0, device=device)
        cfg = {"workload": "box_lattice_64", "scenes": 1, "bodies": 65, "shapes": "box 1x1x1", "sdf_resolution": 32,
               "dt": 0.01}
    return [engine_io.scene_arrays(engine)], engine.params, cfg, engine


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed region: NVML read every 10 ms (one
    sample at the start and one at the end, so short regions still get several), nvidia-smi if NVML is
    unavailable.  Reads only; no setting of the GPU is touched."""
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)
        self._nvml = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(gpu_index).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            self._nvml = (pynvml, h)
        except Exception:
            self._nvml = None

    def _sample(self):
        if self._nvml is not None:
            n, h = self._nvml
            try:
                sm = n.nvmlDeviceGetClockInfo(h, n.NVML_CLOCK_SM)
                mx = n.nvmlDeviceGetMaxClockInfo(h, n.NVML_CLOCK_SM)
                pw = n.nvmlDeviceGetPowerUsage(h) / 1000.0
                r = n.nvmlDeviceGetCurrentClocksEventReasons(h)
                act = lambda bit: "Active" if r & bit else "Not Active"  # noqa: E731
                self.samples.append([str(self.gpu), str(sm), str(mx), "%.1f" % pw, hex(r),
                                     act(n.nvmlClocksEventReasonHwSlowdown),
                                     act(n.nvmlClocksEventReasonHwThermalSlowdown),
                                     act(n.nvmlClocksEventReasonSwThermalSlowdown),
                                     act(n.nvmlClocksEventReasonSwPowerCap)])
                return
            except Exception:
                self._nvml = None
        try:
            out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                  "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
            for line in out.stdout.strip().splitlines():
                self.samples.append([v.strip() for v in line.split(",")])
        except Exception:
            pass

    def _run(self):
        while not self._stop.is_set():
            self._sample()
            self._stop.wait(0.01 if self._nvml is not None else 0.2)

    def __enter__(self):
        self._sample()
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)
        self._sample()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        num = lambda v: v.replace(".", "", 1).isdigit()  # noqa: E731
        sm = [float(s[1]) for s in self.samples if len(s) > 2 and num(s[1])]
        mx = [float(s[2]) for s in self.samples if len(s) > 2 and num(s[2])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 5 + i and s[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# --------------------------------------------------------------------------------------------------------------
# CPU baseline: the oracle (C restatement of the reference step), bounded sample
# --------------------------------------------------------------------------------------------------------------
def _cpu_task(job):
    """One scene of the CPU baseline sample on one host core: bring it to the timed state (the GPU's state
    after its pre-roll when given, else the oracle's own pre-roll), one untimed step (fills the warm-start
    cache), then timed steps until `seconds` have passed (at least one).  Returns (steps, elapsed, bodies)."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    scene, state, pre_roll, pre_cap, max_it, seconds, kw = job
    sc = O.OracleScene(scene)
    if state is not None:
        sc.set_state(*state)
    else:
        sc.set_param("max_iterations", pre_cap)
        for _ in range(pre_roll):
            sc.step(**kw)
    sc.set_param("max_iterations", max_it)
    sc.step(**kw)
    steps, t0 = 0, time.perf_counter()
    while True:
        sc.step(**kw)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            return steps, el, sc.n_bodies


def stratified_sample(body_counts, n):
    """Indices of n scenes spread evenly over the scenes sorted by body count (every size stratum sampled)."""
    order = np.argsort(np.asarray(body_counts), kind="stable")
    n = max(1, min(n, len(order)))
    return [int(order[int((k + 0.5) * len(order) / n)]) for k in range(n)]


def cpu_baseline(arrays, args, workers, states=None, pre_cap=100):
    """scene-steps/s of the oracle on the host cores for the workload's scene mix.

    A stratified sample of the scenes (--cpu-scenes, by body count) goes through a shared task queue, largest
    scenes first, so no core idles while another still has work; each task times one scene's steps on one
    core while the others are busy too.  With t_i the measured time per step of sample scene i, the host
    steps the whole mix (every scene once per step) at cores x n / sum(t_i) scene-steps/s -- the rate of a
    perfectly load-balanced host -- and cores x sum(bodies_i) / sum(t_i) body-steps/s.  `states` gives each
    scene's (x, u) at the start of the timed region (from the GPU run); without it each task pre-rolls its
    scene on the oracle first."""
    import multiprocessing as mp
    from oracle import oracle as O
    O.build()
    tol_mode = {"merit": 0, "residual": 1, "residual_fixed_r": 2}[args.termination]
    idx = stratified_sample([len(a["body_mass"]) for a in arrays], args.cpu_scenes)
    idx.sort(key=lambda i: -len(arrays[i]["body_mass"]))
    kw = {"scheme": args.scheme, "tol_mode": tol_mode, "tol": args.tolerance, "ordering": args.ordering,
          "residual_interval": args.residual_interval if args.termination == "residual_fixed_r" else 1,
          "warm_start": not args.no_warm_start}
    max_it = args.max_iterations or int(arrays[0]["params"][1])
    workers = max(1, min(workers, len(idx)))
    per_task = max(0.05, args.cpu_seconds * workers / len(idx))   # about cpu_seconds of wall time in all
    def host(a):   # grids built on the device (per-body shapes) travel to the workers as host arrays
        return {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in a.items()}
    jobs = [(host(arrays[i]), None if states is None else states[i], args.pre_roll, pre_cap, max_it, per_task, kw)
            for i in idx]
    t0 = time.perf_counter()
    if workers == 1:
        res = [_cpu_task(j) for j in jobs]
    else:
        with mp.get_context("spawn").Pool(workers) as pool:
            res = list(pool.imap_unordered(_cpu_task, jobs))
    wall = time.perf_counter() - t0
    t = np.array([el / st for st, el, _ in res])          # seconds per step of each sample scene
    bodies = np.array([nb for _, _, nb in res])
    steps = int(sum(r[0] for r in res))
    rate = workers * len(res) / t.sum()
    return rate, {"cores": workers, "kind": "port", "body_steps_per_s": float(workers * bodies.sum() / t.sum()),
                  "sample": "%d of %d scenes stratified by body count (%d..%d bodies), %s; %d timed scene-steps "
                            "(%.2f s per scene on one core of %d busy ones, shared queue, %.1f s wall); rate = "
                            "cores x scenes / sum of per-scene step times"
                            % (len(res), len(arrays), int(bodies.min()), int(bodies.max()),
                               "from the GPU's state after its pre-roll" if states is not None
                               else "after a %d-step oracle pre-roll" % args.pre_roll,
                               steps, per_task, workers, wall),
                  "seconds_per_step_p50_max": [float(np.median(t)), float(t.max())]}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    workers = os.cpu_count() or 1
    import torch
    dev = "cuda:0" if torch.cuda.is_available() else "cpu"
    if args.workload == "tower32":
        from rainbow_b200 import engine_io, scenes
        arrays = [engine_io.scene_arrays(scenes.box_tower(32, device=dev))]
        cfg = {"workload": "box_tower_32_mass_ratio_1e3", "bodies": 33, "dt": 0.005}
    else:
        arrays, _, cfg, _ = build_workload(args.workload, dev, args.scenes, args.shapes)
    value, info = cpu_baseline(arrays, args, workers if len(arrays) > 1 else 1)
    cfg.update({"scheme": args.scheme, "ordering": args.ordering, "termination": args.termination,
                "tolerance": args.tolerance, "max_iterations": args.max_iterations})
    line = {
        "impl": "reference", "metric": "scene-steps/s", "value": value, "unit": "scene-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": cfg,
        "cpu_baseline": dict(value=value, unit="scene-steps/s", **info),
        "e2e": {"value": value, "unit": "scene-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------------------------------------------
# helpers of the GPU arms
# --------------------------------------------------------------------------------------------------------------
def scene_cache(key, sol, count, b0, b1):
    """Warm-start cache entries of the scene owning global bodies b0..b1-1 (device tensors of a batch: keys
    (lower << 31 | higher, side << 30 | triangle) ascending, 4 impulses each), re-keyed to the scene's own
    body indices.  Returns host arrays (n, 2) int64 and (n, 4) float64."""
    n = int(count.reshape(-1)[0].item())
    k = key[:2 * n].view(n, 2).cpu().numpy().copy()
    s = sol[:4 * n].view(n, 4).cpu().numpy()
    lo = k[:, 0] >> 31
    m = (lo >= b0) & (lo < b1)
    k = k[m]
    k[:, 0] -= (np.int64(b0) << 31) + np.int64(b0)
    return k, s[m].copy()


def install_cache(world, keys, sols):
    """Warm-start cache of a one-scene DeviceWorld (grown first when it cannot hold the entries)."""
    import torch
    n = len(keys)
    if 2 * n > world.t_cache_key.numel():
        world.caps.contact_capacity = max(n, 2 * world.caps.contact_capacity)
        world._alloc()
    world.t_cache_key[:2 * n].copy_(torch.from_numpy(keys.reshape(-1)))
    world.t_cache_sol[:4 * n].copy_(torch.from_numpy(sols.reshape(-1)))
    world.t_cache_count.fill_(n)


def timed_steps(step_fn, steps, stream, flush):
    """Device time (ms) of each of `steps` calls of step_fn, which enqueues one step on `stream`."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        flush.zero_()                      # evict L2 (126 MB) between timed steps
        ev[k][0].record(stream)
        step_fn()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    return np.array([a.elapsed_time(b) for a, b in ev])   # ms


def solve_summary(stats, cap):
    """Convergence of one step's solves: how many met the tolerance, sweeps, residuals of the others."""
    act = [s for s in stats if s.n_contacts > 0]
    if not act:
        return None
    conv = [s for s in act if s.exitcode == 3]
    unc = np.array([s.residual for s in act if s.exitcode != 3])
    sw = np.array([s.iterations + 1 if s.exitcode == 3 else cap for s in act])
    return {"scenes_with_contacts": len(act), "met_tolerance": len(conv), "unconverged": len(act) - len(conv),
            "unconverged_residual_p50_p99_max": [float(np.percentile(unc, 50)), float(np.percentile(unc, 99)),
                                                 float(unc.max())] if len(unc) else None,
            "sweeps_p50_p90_max": [float(np.percentile(sw, 50)), float(np.percentile(sw, 90)), int(sw.max())],
            "residual_median": float(np.median([s.residual for s in act]))}


def batched_arm(world, rp, steps, warmup, restore, flush, gpu, dist=None):
    """Timed graph replays of the whole batch from the saved state: a sizing pass over the timed horizon (so
    no timed step can overflow a work list), warm-up steps, one CUDA graph of the step, then `steps` replays
    with the L2 flushed between them.  Returns times (ms), kernel launches, clocks, status and the last
    step's statistics."""
    import torch
    from rainbow_b200 import _native
    stream = torch.cuda.current_stream()
    restore()
    for _ in range(steps):
        world.step(rp)
    restore()
    for _ in range(max(3, warmup)):
        world.step(rp)
    lib = _native.load()
    launches0 = lib.rb_launch_count()
    graph = world.capture(rp)
    per_replay = lib.rb_launch_count() - launches0
    restore()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    world.t_status.zero_()
    with ClockSampler(gpu) as clocks:
        times = timed_steps(graph.replay, steps, stream, flush)
    del graph
    if dist is not None:
        dist.barrier()
    return times, per_replay * steps, clocks.summary(), int(world.t_status[0].item()), world.stats()


def plain_arm(world, arrays, idx, x0, u0, cache, rp, steps, flush, max_it):
    """The plain baseline: each sampled scene alone, one rb_step launch sequence per scene-step, FP64, from the
    batch's saved state and warm-start cache; timed with direct launches and with graph replays.  FP64
    results are bit-identical alone and batched, so these are the batched FP64 scene's own steps."""
    import torch
    from rainbow_b200 import world as W
    stream = torch.cuda.current_stream()
    x0r, u0r = x0.reshape(-1, 7), u0.reshape(-1, 6)
    pts, gts, last = [], [], []
    for s in idx:
        b0, b1 = int(world.scene_start[s]), int(world.scene_start[s + 1])
        keys, sols = scene_cache(*cache, b0, b1)
        w1 = W.DeviceWorld(arrays[s], device=world.device, max_iterations=max_it)

        def start():
            w1.set_state(x0r[b0:b1], u0r[b0:b1])
            install_cache(w1, keys, sols)
        start()
        for _ in range(steps):
            w1.step(rp)                  # sizes its work lists over the horizon
        start()
        torch.cuda.synchronize()
        pts.append(timed_steps(lambda: w1.launch(rp), steps, stream, flush))
        last.append(w1.stats()[0])
        g1 = w1.capture(rp)
        start()
        torch.cuda.synchronize()
        gts.append(timed_steps(g1.replay, steps, stream, flush))
        del g1, w1
    pt, gt = np.concatenate(pts), np.concatenate(gts)
    return {"value": len(pt) / (pt.sum() / 1000.0), "unit": "scene-steps/s", "scenes_sampled": len(idx),
            "steps_per_scene": steps,
            "bodies_sampled": [int(world.scene_start[s + 1] - world.scene_start[s]) for s in idx],
            "p50_ms": float(np.percentile(pt, 50)), "p99_ms": float(np.percentile(pt, 99)),
            "graph_value": len(gt) / (gt.sum() / 1000.0),
            "graph_p50_ms": float(np.percentile(gt, 50)), "graph_p99_ms": float(np.percentile(gt, 99)),
            "solve_last_step": solve_summary(last, max_it),
            "method": "scenes stratified by body count, each alone: one rb_step launch sequence per scene-step, "
                      "FP64, same solver settings, from the batch's state and warm-start cache (bit-identical to "
                      "the batch's FP64 step); graph_* = the same steps replayed from a CUDA graph per scene"}


def plugin_arm(arrays, x0, u0, args, dev, flush, prec, warm, cap, shapes=None):
    """The batch through the reference-style drop-in: one engine object per scene (grids kept on the device
    as views of the workload's tensor), stepped by api.simulate_batch with a BatchStepper.  Every step reads
    the bodies' r, q, v, w from the engine objects (host), uploads them, steps, and writes the new state and
    each engine's contact points back into the objects.  Starts from the batch's saved state; the warm-start
    cache fills during the warm-up steps."""
    import torch
    from rainbow_b200 import api as API, engine_io
    from rainbow_b200.stepper import BatchStepper
    t_build = time.perf_counter()
    engines = [engine_io.engine_from_arrays(a) for a in arrays]
    x0r, u0r = x0.reshape(-1, 7), u0.reshape(-1, 6)
    k = 0
    for e in engines:
        e.params.proximal_solver = None if args.scheme == "rigid_gauss_seidel" else args.scheme
        e.params.warm_start = warm
        e.params.solver_precision = prec
        e.params.contact_ordering = args.ordering
        e.params.max_iterations = cap
        for b in e.bodies.values():
            b.r, b.q, b.v, b.w = x0r[k, :3].copy(), x0r[k, 3:].copy(), u0r[k, :3].copy(), u0r[k, 3:].copy()
            k += 1
    stepper = BatchStepper(device=dev, termination=args.termination, residual_tolerance=args.tolerance,
                           residual_interval=args.residual_interval, launch_shapes=shapes)
    dt = engines[0].params.time_step
    API.simulate_batch(engines, dt, stepper)       # builds the batch
    t_build = time.perf_counter() - t_build
    for _ in range(max(0, args.warmup - 1)):
        API.simulate_batch(engines, dt, stepper)
    times = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        API.simulate_batch(engines, dt, stepper)
        times.append(time.perf_counter() - t0)
    t = np.array(times)
    nb = sum(len(e.bodies) for e in engines)
    K = sum(len(e.contact_points) for e in engines)
    out = {"value": len(engines) * len(t) / t.sum(), "unit": "scene-steps/s",
           "p50_ms": float(np.percentile(t, 50) * 1e3), "p99_ms": float(np.percentile(t, 99) * 1e3),
           "h2d_bytes_per_step": 13 * 8 * nb, "d2h_bytes_per_step": 13 * 8 * nb + 64 * K,
           "engines": len(engines), "bodies": nb, "build_s": t_build,
           "api": "api.simulate_batch(engines, dt, BatchStepper) over one engine object per scene: r, q, v, w read "
                  "from and written back to every body, contact points per engine, every step"}
    del stepper, engines
    torch.cuda.empty_cache()
    return out


# --------------------------------------------------------------------------------------------------------------
# serving: Poisson stream of scene simulations through the continuous-batching server
# --------------------------------------------------------------------------------------------------------------
def run_serving(args, dev, rp_kw, max_it, flush, tuning=None):
    """Requests arrive as a Poisson stream (rate --serve-rate) of scenes with 16..2048 bodies (log-uniform) and
    horizons U[50, 500] steps; the server admits them by its memory budget (80 % of the device) and body cap.
    Returns throughput and latency of the run and of resident scenes stepped alone, one per launch, FP64."""
    import torch
    from rainbow_b200 import autotune, scenes, serving, world as W
    templates, params = scenes.batch_arrays(n_scenes=args.serve_templates, seed=1, pool=64,
                                            body_range=(16, 2048), resolution=32, device=dev, ground=40.0)
    rp = W.make_rb_params(params, **rp_kw)
    rp.max_iterations = max_it
    if tuning:
        autotune.apply(rp, {k: v for k, v in tuning.items() if k in autotune.DEFAULTS})
    rng = np.random.default_rng(7)
    srv = serving.Server(rp, device=dev, max_iterations=max_it, hbm_fraction=0.8,
                         max_active_bodies=args.serve_max_bodies)
    t_start = time.perf_counter()
    next_arrival = t_start
    submitted = 0
    while True:
        now = time.perf_counter()
        if now - t_start >= args.serve_seconds:
            break
        while next_arrival <= now:
            srv.submit(templates[int(rng.integers(len(templates)))], int(rng.integers(50, 501)), arrival=next_arrival)
            submitted += 1
            next_arrival += rng.exponential(1.0 / args.serve_rate)
        srv.tick()
    rep = srv.report()
    last = srv.batch.stats() if srv.batch is not None else []
    rep.update({"seconds": args.serve_seconds, "arrival_rate": args.serve_rate, "submitted": submitted,
                "queued_at_end": len(srv.queue), "resident_body_cap": args.serve_max_bodies,
                "memory_budget_gb": srv.budget / 1e9, "solve_last_tick": solve_summary(last, max_it),
                "workload": "Poisson requests, scenes of 16..2048 bodies (log-uniform; %d distinct), horizons "
                            "U[50,500], boxes/spheres as the batch workload on a 40 x 1 x 40 ground"
                            % len(templates)})
    # plain: scenes resident at the end of the run, spread evenly over their body counts (so that the sample's
    # sizes, and with them its rate, do not depend on which scenes happen to be resident), each stepped alone
    # from its current state and warm-start cache, one rb_step per scene-step, FP64, same solver settings
    rp64 = W.make_rb_params(params, **dict(rp_kw, precision="fp64"))
    rp64.max_iterations = max_it
    stream = torch.cuda.current_stream()
    b = srv.batch
    resident = sorted([r for r in srv.active if r.done < r.horizon], key=lambda r: r.uid)
    pick = stratified_sample([len(r.scene["body_mass"]) for r in resident], args.serve_plain_scenes) \
        if resident and args.serve_plain_scenes > 0 else []
    times, last = [], []
    for i in sorted(int(v) for v in pick):
        r = resident[i]
        b0, b1 = int(b.scene_start[r.slot]), int(b.scene_start[r.slot + 1])
        x, u = b.scene_state(r.slot)
        keys, sols = scene_cache(b.t_cache_key, b.t_cache_sol, b.t_cache_count, b0, b1)
        w1 = W.DeviceWorld(r.scene, device=dev, max_iterations=max_it)

        def start():
            w1.set_state(x, u)
            install_cache(w1, keys, sols)
        start()
        for _ in range(args.plain_steps):
            w1.step(rp64)                  # sizes its work lists
        start()
        torch.cuda.synchronize()
        times.append(timed_steps(lambda: w1.launch(rp64), args.plain_steps, stream, flush))
        last.append(w1.stats()[0])
        del w1
    times = np.concatenate(times) if times else np.zeros(0)
    if len(times):
        rep["plain"] = {"value": len(times) / (times.sum() / 1000.0), "unit": "scene-steps/s",
                        "p50_ms": float(np.percentile(times, 50)), "p99_ms": float(np.percentile(times, 99)),
                        "solve_last_step": solve_summary(last, max_it),
                        "bodies_sampled": [len(resident[int(i)].scene["body_mass"]) for i in sorted(pick)],
                        "sample": "%d scenes resident at the end of the run, stratified by body count, %d steps each "
                                  "from their state and warm-start cache, one rb_step per scene-step, FP64"
                                  % (len(pick), args.plain_steps)}
        rep["served_vs_plain"] = rep["scene_steps_per_s"] / rep["plain"]["value"] if rep.get("scene_steps_per_s") else None
    return rep


# --------------------------------------------------------------------------------------------------------------
# the configurations beside the headline: C1 (64 boxes, coloured GS, through API.simulate), C2 (4097-body
# lattice, Gauss-Seidel and Jacobi, FP64 vs FP32 + refinement), C4 (the mass-ratio tower, 500 steps)
# --------------------------------------------------------------------------------------------------------------
def config_c1(dev, cpu=True):
    """64 unit boxes on a ground, coloured proximal Gauss-Seidel, FP64, the reference's merit rule (100
    iterations, relative tolerance 1e-6), 100 steps through the drop-in GpuStepper and api.simulate, with the
    engine's bodies read and written every step (host state in and out)."""
    import torch
    from rainbow_b200 import api as API, engine_io, scenes
    engine = scenes.box_lattice(n=4, spacing=1.05, jitter=0.02, resolution=32, seed=0, device=dev)
    engine.params.proximal_solver = "parallel_gauss_seidel"
    arrays0 = engine_io.scene_arrays(engine)
    dt = engine.params.time_step
    API.simulate(engine, dt)                      # first step: uploads the scene, sizes the work lists
    walls = []
    for _ in range(99):
        t0 = time.perf_counter()
        API.simulate(engine, dt)
        walls.append(time.perf_counter() - t0)
    torch.cuda.synchronize()
    walls = np.array(walls)
    out = {"workload": "box_lattice_64 (4^3, spacing 1.05, jitter 0.02), SDF 32, dt 0.01, mu 0.5",
           "solver": "parallel_gauss_seidel (coloured), FP64, merit rule, max 100 iterations",
           "api": "rainbow_b200.api.simulate -> GpuStepper.step (engine state in and out every step)",
           "steps": 100, "steps_per_s": float(len(walls) / walls.sum()),
           "step_wall_ms_p50_p99": [float(np.percentile(walls, 50) * 1e3), float(np.percentile(walls, 99) * 1e3)],
           "contacts_last_step": len(engine.contact_points)}
    if cpu:   # the oracle on one host core, same 100 steps
        from oracle import oracle as O
        O.build()
        sc = O.OracleScene(arrays0)
        t0 = time.perf_counter()
        for _ in range(100):
            sc.step(scheme="parallel_gauss_seidel")
        el = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 100.0 / el, "unit": "steps/s", "cores": 1, "kind": "port",
                               "sample": "the same 100 steps on the oracle"}
    return out


def config_c2(dev, args, flush):
    """4097-body box/sphere lattice (SDF resolution 64), after a 30-step pre-roll: Gauss-Seidel and proximal
    Jacobi, each in FP64 and in FP32 + FP64 refinement, for a few steps from the same state at the
    equal-residual settings; error of each against Gauss-Seidel FP64 after the first step."""
    import torch
    from rainbow_b200 import engine_io, scenes, world as W
    arrays = engine_io.scene_arrays(scenes.mixed_lattice(n=16, spacing=1.2, resolution=64, seed=0, device=dev))
    params = W.params_from_vector(arrays["params"])
    cap = args.max_iterations
    world = W.DeviceWorld(arrays, device=dev, max_iterations=max(cap, 100))
    kw = dict(termination="residual_fixed_r", residual_tolerance=args.tolerance,
              residual_interval=args.residual_interval, warm_start=True)
    pre = W.make_rb_params(params, precision="fp32_refine", **kw)
    for _ in range(30):
        world.step(pre)
    x0, u0 = world.state()
    cache = (world.t_cache_key.clone(), world.t_cache_sol.clone(), world.t_cache_count.clone())
    stream = torch.cuda.current_stream()
    arms = [("gauss_seidel_fp64", "rigid_gauss_seidel", "fp64"), ("gauss_seidel_fp32_refine", "rigid_gauss_seidel",
                                                                   "fp32_refine"),
            ("jacobi_fp64", "parallel_jacobi", "fp64"), ("jacobi_fp32_refine", "parallel_jacobi", "fp32_refine")]
    out, u_ref = {}, None
    for name, scheme, prec in arms:
        rp = W.make_rb_params(params, scheme=scheme, precision=prec, **kw)
        rp.max_iterations = cap
        times, u1 = [], None
        for k in range(3):
            if k == 0:
                world.set_state(x0, u0)
                world.t_cache_key.copy_(cache[0]); world.t_cache_sol.copy_(cache[1]); world.t_cache_count.copy_(cache[2])
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            world.step(rp)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            st = world.stats()[0]
            if k == 0:
                u1 = world.state()[1]
        if u_ref is None:
            u_ref = u1
        out[name] = {"ms_per_step": float(np.mean(times)), "contacts": int(st.n_contacts), "levels": int(st.n_levels),
                     "sweeps": int(st.iterations + 1 if st.exitcode == 3 else cap), "met_tolerance": st.exitcode == 3,
                     "residual": float(st.residual),
                     "max_rel_velocity_error_vs_gs_fp64_step1": float(np.abs(u1 - u_ref).max() / np.abs(u_ref).max())}
    return {"workload": "mixed_lattice_4096 (16^3 boxes / r 0.5 spheres, spacing 1.2, density 1000), SDF 64",
            "state": "after a 30-step pre-roll; 3 steps per arm from the same state and warm-start cache",
            "max_iterations": cap, "tolerance": args.tolerance, "arms": out}


def config_c4(dev, steps=500, cap=100, tol=1e-6):
    """32-high box tower, masses alternating 1 and 1000, mu 0.6, dt 0.005, `steps` steps in FP64, FP32 + FP64
    refinement and FP32: complementarity residual per step and position drift against the FP64 run."""
    import torch
    from rainbow_b200 import engine_io, scenes, world as W
    arrays = engine_io.scene_arrays(scenes.box_tower(32, device=dev))
    params = W.params_from_vector(arrays["params"])
    stream = torch.cuda.current_stream()
    runs = {}
    for mode in ("fp64", "fp32_refine", "fp32"):
        w = W.DeviceWorld(arrays, device=dev, max_iterations=max(cap, 100))
        rp = W.make_rb_params(params, precision=mode, termination="residual_fixed_r", residual_tolerance=tol,
                              residual_interval=4, warm_start=True)
        rp.max_iterations = cap
        x_init, u_init = w.state()
        w.step(rp)                        # sizes the work lists; the run starts from the initial state again
        w.set_state(x_init, u_init)
        w.reset_warm_start()
        xs, res, ms, sw = [], [], [], []
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            w.step(rp)
            e1.record(stream)
            xs.append(w.state()[0][:, :3].copy())
            s = w.stats()[0]
            res.append(s.residual)
            sw.append(s.fp32_sweeps)
            ms.append(e0.elapsed_time(e1))
        runs[mode] = (np.array(xs), np.array(res), np.array(ms), np.array(sw))
    x64 = runs["fp64"][0]
    every = max(1, steps // 20)
    rep = {}
    for mode, (xs, res, ms, sw) in runs.items():
        drift = np.abs(xs - x64).max(axis=(1, 2))
        rep[mode] = {"ms_per_step": float(ms[1:].mean()), "residual_median": float(np.median(res)),
                     "residual_max": float(res.max()), "steps_meeting_tolerance": int((res <= tol).sum()),
                     "fp32_sweeps_mean": float(sw[sw >= 0].mean()) if (sw >= 0).any() else 0.0,
                     "drift_m_max_first_50_steps": float(drift[:50].max()), "drift_m_max": float(drift.max()),
                     "per_step": [{"step": k + 1, "residual": float(res[k]), "drift_m": float(drift[k])}
                                  for k in range(every - 1, steps, every)]}
    return {"workload": "box_tower_32_mass_ratio_1e3", "bodies": 33, "dt": 0.005, "mu": 0.6, "steps": steps,
            "termination": "residual_fixed_r", "tolerance": tol, "max_iterations": cap, "precision": rep}


# --------------------------------------------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cpu_pool_workers = os.cpu_count() or 1   # the CPU baseline's pool is spawned, never forked
    torch.cuda.set_device(local)
    dev = "cuda:%d" % local
    if world_size > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device(dev))
    from rainbow_b200 import world as W
    from rainbow_b200.sharding import max_over_ranks, partition_scenes, sum_over_ranks
    if world_size > 1 and args.workload == "batch1024":
        # weak scaling: world_size x --scenes scenes, split by body count so every GPU holds --scenes of them;
        # each rank builds only its own share (the body counts come from the seeded draws alone)
        from rainbow_b200 import scenes as SC
        n_all = args.scenes * world_size
        if args.shapes == "per-body":
            counts = SC.per_body_counts(n_all, 0)
        else:
            counts = [len(a["body_mass"]) for a in SC.batch_arrays(n_scenes=n_all, seed=0, pool=64, resolution=32,
                                                                   device=dev)[0]]
        parts = partition_scenes(counts, world_size)
        arrays, params, cfg, engine = build_workload(args.workload, dev, n_all, args.shapes, select=parts[rank])
        cfg.update({"scenes_per_gpu": len(arrays), "scenes": n_all})
    else:
        arrays, params, cfg, engine = build_workload(args.workload, dev, args.scenes, args.shapes)
    pre_cap = int(params.max_iterations)      # the configuration's own iteration limit (100)
    cap = int(args.max_iterations)
    world = W.DeviceWorld(arrays, device=dev, max_iterations=max(cap, pre_cap))
    kw = dict(scheme=args.scheme, termination=args.termination, residual_tolerance=args.tolerance,
              residual_interval=args.residual_interval if args.termination == "residual_fixed_r" else 1,
              ordering=args.ordering)
    warm = not args.no_warm_start
    prec = args.precision if args.termination == "residual_fixed_r" else "fp64"

    def mk(precision, it, profiling=False):
        rp = W.make_rb_params(params, warm_start=warm, precision=precision, profiling=profiling, **kw)
        rp.max_iterations = it
        return rp
    rp_pre = mk(prec, pre_cap)
    for _ in range(args.pre_roll):
        world.step(rp_pre)
    # launch shapes tuned on this batch (speed only: results are the same bits for every shape), once at the
    # 100-sweep limit and once at the equal-residual cap: the slabs of the FP32 warp teams decide how many
    # scenes share an SM, which a short solve wants high and a long one (bound by its longest scene) lower
    tuning = None
    if not args.no_autotune and args.workload == "batch1024":
        from rainbow_b200 import autotune
        t0 = time.perf_counter()
        best100, info100 = autotune.tune(world, rp_pre)
        t1 = time.perf_counter()
        if cap != pre_cap:   # at the cap only the FP32 slabs matter: tuned over the timed horizon
            best, info = autotune.tune(world, mk(prec, cap), steps=args.steps, repeats=1, rounds=1,
                                       start=best100, knobs=("fp32_small_slab", "fp32_mid_slab"))
        else:
            best, info = best100, info100
        tuning = dict(best, seconds=time.perf_counter() - t1, **info)
        tuning["at_100_sweeps"] = dict(best100, seconds=t1 - t0, **info100)
    rps = {"mode": mk(prec, cap), "fp64": mk("fp64", cap), "prof": mk(prec, cap, True), "check": mk(prec, cap, 3),
           "mode100": mk(prec, pre_cap), "fp64_100": mk("fp64", pre_cap)}
    if tuning:
        from rainbow_b200 import autotune
        for name, rp in rps.items():
            autotune.apply(rp, best100 if name in ("mode100", "fp64_100") else best)
    x0, u0 = world.state()                 # state the timed region (and every baseline) starts from
    cache = (world.t_cache_key.clone(), world.t_cache_sol.clone(), world.t_cache_count.clone())

    def restore():
        world.set_state(x0, u0)
        world.t_cache_key.copy_(cache[0]); world.t_cache_sol.copy_(cache[1]); world.t_cache_count.copy_(cache[2])

    # the first step from the saved state in this precision mode (profiled: phase times, byte counts) and in
    # FP64: every scene's convergence in both, and the mode's error against FP64
    restore()
    world.step(rps["prof"])
    phases = world.profile_times()
    stats = world.stats()
    u_m = world.state()[1]
    restore()
    world.step(rps["check"])               # the FP32 contact search checked against the FP64 search
    stats_check = world.stats()
    restore()
    world.step(rps["fp64"])
    stats64 = world.stats()
    u_64 = world.state()[1]
    um, u6 = u_m.reshape(-1, 6), u_64.reshape(-1, 6)
    active = [i for i in range(world.n_scenes) if stats64[i].n_contacts > 0]
    rel = []
    for i in active:
        b0, b1 = world.scene_start[i], world.scene_start[i + 1]
        rel.append(np.abs(um[b0:b1] - u6[b0:b1]).max() / max(1e-30, np.abs(u6[b0:b1]).max()))
    rel = np.array(rel)
    both = [i for i in active if stats[i].exitcode == 3 and stats64[i].exitcode == 3]
    rel_conv = np.array([rel[active.index(i)] for i in both])
    pct = lambda v: [float(np.percentile(v, 50)), float(np.percentile(v, 99)), float(v.max())] if len(v) else None  # noqa: E731
    equal = {"first_step_from_saved_state": {"mode": solve_summary(stats, cap), "fp64": solve_summary(stats64, cap)},
             "mode_vs_fp64_per_scene_max_rel_velocity_error_p50_p99_max": pct(rel),
             "same_on_scenes_both_met_tolerance": pct(rel_conv),
             "fp32_sweeps_mean": float(np.mean([s.fp32_sweeps for s in stats if s.n_contacts > 0 and s.fp32_sweeps >= 0]
                                               or [0]))}

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    times, launches, clocks, status, after = batched_arm(world, rps["mode"], args.steps, args.warmup, restore, flush,
                                                        local, dist if world_size > 1 else None)
    total_ms = max_over_ranks(float(times.sum()), dev)       # the slowest rank's device time
    all_scenes = int(sum_over_ranks(world.n_scenes, dev))
    value = all_scenes * args.steps / (total_ms / 1000.0)

    sample = stratified_sample(np.diff(world.scene_start), args.plain_scenes) if world.n_scenes > 1 else []
    plain = None
    if sample and args.plain_scenes > 0 and rank == 0:
        plain = plain_arm(world, arrays, sample, x0, u0, cache, rps["fp64"], args.plain_steps, flush, cap)

    at100 = None
    if not args.no_100 and world.n_scenes > 1 and rank == 0:
        t100, _, c100, _, after100 = batched_arm(world, rps["mode100"], args.steps, args.warmup, restore, flush, local)
        v100 = world.n_scenes * args.steps / (t100.sum() / 1000.0)
        p100 = plain_arm(world, arrays, sample, x0, u0, cache, rps["fp64_100"], args.plain_steps, flush, pre_cap)
        rp100p = mk(prec, pre_cap, True)      # one profiled step from the saved state: the phase times
        if tuning:
            from rainbow_b200 import autotune
            autotune.apply(rp100p, best100)
        restore()
        world.step(rp100p)
        ph100 = world.profile_times()
        at100 = {"max_iterations": pre_cap, "value": v100, "unit": "scene-steps/s",
                 "phases_ms_first_step": {k: v * 1000.0 for k, v in zip(PHASE_NAMES, ph100)},
                 "ms_per_step": float(t100.mean()), "p50_ms": float(np.percentile(t100, 50)),
                 "p99_ms": float(np.percentile(t100, 99)), "solve_last_step": solve_summary(after100, pre_cap),
                 "plain": p100, "speedup_vs_plain": v100 / p100["value"],
                 "note": "the configuration's own 100-sweep limit: both arms stop at the same sweep count, most "
                         "scenes before the 1e-6 tolerance"}

    # end to end through the public API, host buffers in and out every step
    e2e = None
    if not args.no_e2e:
        if engine is not None:
            from rainbow_b200 import engine_io
            from rainbow_b200.stepper import GpuStepper
            engine_io.write_back(engine, x0.reshape(-1, 7), u0.reshape(-1, 6))
            engine.stepper = GpuStepper(device=dev, termination=args.termination,
                                        residual_tolerance=args.tolerance)
            engine.params.proximal_solver = None if args.scheme == "rigid_gauss_seidel" else args.scheme
            engine.params.warm_start = warm
            engine.params.solver_precision = prec
            engine.params.max_iterations = cap
            engine.stepper.step(engine.params.time_step, engine, False)
            engine_io.write_back(engine, x0.reshape(-1, 7), u0.reshape(-1, 6))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                engine.stepper.step(engine.params.time_step, engine, False)
            torch.cuda.synchronize()
            el = time.perf_counter() - t0
            K = len(engine.contact_points)
            d2h = 13 * 8 * world.n_bodies + K * 64 + 8
            api = "GpuStepper.step via engine"
        else:
            # the step as one CUDA graph replay; the state goes host -> device and back every step through the
            # pinned staging buffers, which the caller reads and passes back without host copies
            restore()
            g_e2e = world.capture(rps["mode"])
            restore()
            hx, hu = x0, u0
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                world.set_state(hx, hu)               # pinned host -> device
                g_e2e.replay()
                hx, hu = world.state(copy=False)      # device -> pinned host (synchronises)
                st = world.t_stats.cpu()
            el = time.perf_counter() - t0
            del g_e2e
            d2h = 13 * 8 * world.n_bodies + st.numel()
            api = "DeviceWorld set_state / graph replay / state(copy=False)"
        el = max_over_ranks(el, dev)
        e2e = {"value": all_scenes * args.steps / el, "unit": "scene-steps/s",
               "h2d_bytes_per_step": 13 * 8 * world.n_bodies, "d2h_bytes_per_step": int(d2h), "api": api}
        if engine is None and world_size == 1 and not args.no_plugin:
            try:
                e2e["plugin"] = plugin_arm(arrays, x0, u0, args, dev, flush, prec, warm, cap,
                                           best if tuning else None)
            except Exception as ex:   # recorded, not fatal: the headline line must still be printed
                e2e["plugin"] = {"error": repr(ex)[:400]}

    # rooflines of the profiled step's phases (event times on the launching stream)
    K = sum(s.n_contacts for s in stats)
    sweeps = sum(s.n_contacts * ((s.iterations + 1) if 0 <= s.iterations < cap else cap) for s in stats)
    sweeps32 = sum(s.n_contacts * min(max(s.fp32_sweeps, 0), cap) for s in stats)   # of those, in FP32
    sweeps64 = max(0, sweeps - sweeps32)
    cand = sum(s.n_candidates for s in stats)
    lookups = sum(s.n_grid_lookups for s in stats)
    lookups32 = sum(s.n_grid_lookups32 for s in stats)
    equal["contact_search_decision_flips"] = {
        "candidates": int(cand), "search_flips": int(sum(s.n_search_flips for s in stats_check)),
        "accept_flips": int(sum(s.n_accept_flips for s in stats_check)),
        "fp32_lookups": int(lookups32), "fp64_lookups": int(lookups),
        "note": "first step from the saved state: candidates whose FP32 search (seed, Frank-Wolfe choices, "
                "iterations) or acceptance differs from the plain FP64 search on the same candidate; FP64 lookups "
                "are the acceptance tests, the contact data and the near-ties decided in FP64"}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        peaks = {}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    src = "of measured (MEASURED_PEAKS.json hbm_gbs)" if peaks else "of fallback 6650 GB/s"

    def roof(name, dt_s, nbytes, model, kernel, bound_note):
        achieved = nbytes / dt_s / 1e9 if dt_s > 0 else 0.0
        prof = PROFILED_DRAM_BYTES.get(kernel)
        traffic = prof[0] if prof and prof[1] == (cfg["workload"], prec, cap) else None
        return {"bound": "hbm", "kernel_phase": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "algorithmic_bytes": int(nbytes), "bytes_model": model,
                "phase_ms": dt_s * 1000.0, "peak_source": src, "note": bound_note}
    solve_roof = roof("solve", phases[4], sweeps64 * 137 * 8 + sweeps32 * 137 * 4,
                      "per contact per sweep: J 48 + WJT 48 + b 4 + r 4 + mu 1 + x 8 + body w 24 values, 8 B each in "
                      "FP64 sweeps (1096 B) and 4 B in FP32 sweeps (548 B)", "k_solve_fp32",
                      "latency-bound: each scene is one chain of (levels x sweeps) dependent contact updates whose "
                      "rows sit in shared memory (FP32) or L2 (FP64); neither HBM nor the SMs are near their limit")
    narrow_roof = roof("contact_search", phases[2], cand * (72 + 64) + lookups * 64 + lookups32 * 32,
                       "per candidate triangle: 3 world vertices (72 B) + result record (64 B); 8 grid values per "
                       "signed distance lookup, 64 B on the FP64 grid and 32 B on the FP32 copy, lookups counted on "
                       "the device", "k_narrow",
                       "gathers of 8 grid nodes per lookup; " + ("a grid per body: the gathers go to HBM"
                                                                 if args.shapes == "per-body" and
                                                                 args.workload == "batch1024"
                                                                 else "with a shape pool the grids are L2-resident"))
    doms = {"solve": solve_roof, "contact_search": narrow_roof}
    dom = max(doms, key=lambda k: doms[k]["phase_ms"])

    cpu = None
    if rank == 0 and args.cpu_seconds > 0:
        x0r, u0r = x0.reshape(-1, 7), u0.reshape(-1, 6)
        states = {i: (x0r[world.scene_start[i]:world.scene_start[i + 1]], u0r[world.scene_start[i]:world.scene_start[i + 1]])
                  for i in range(world.n_scenes)}
        cv, info = cpu_baseline(arrays, args, cpu_pool_workers if world.n_scenes > 1 else 1, states=states,
                                pre_cap=pre_cap)
        cpu = dict(value=cv, unit="scene-steps/s", **info)

    # the batch's device memory (with a grid per body ~48 GB) is released before the serving run admits scenes
    # by its own memory budget
    n_bodies_world = world.n_bodies
    del world, arrays
    import gc
    gc.collect()
    torch.cuda.empty_cache()

    serving_rep = None
    if args.serve_seconds > 0 and args.workload == "batch1024" and world_size == 1:
        serving_rep = run_serving(args, dev, dict(warm_start=warm, precision=prec, **kw), cap, flush,
                                  tuning=best if tuning else None)

    configs = None
    if not args.no_configs and args.workload == "batch1024" and world_size == 1:
        configs = {"C1": config_c1(dev, cpu=args.cpu_seconds > 0), "C2": config_c2(dev, args, flush),
                   "C4": config_c4(dev, steps=500, cap=pre_cap, tol=args.tolerance)}


    cfg.update({"scheme": args.scheme, "ordering": args.ordering, "termination": args.termination,
                "tolerance": args.tolerance, "max_iterations": cap,
                "precision": prec, "warm_start": warm, "residual_interval": kw["residual_interval"],
                "pre_roll_steps": args.pre_roll, "pre_roll_max_iterations": pre_cap, "contacts_per_step": int(K),
                "sweeps_per_step_contacts": int(sweeps), "l2": "256 MB buffer written between timed steps",
                "launch": "each timed step replays one CUDA graph of the whole rb_step",
                "launch_shapes": tuning,
                "parallelism": ("scenes partitioned over %d GPUs, no collective on the step" % world_size
                                if world_size > 1 and args.workload == "batch1024"
                                else "replicas" if world_size > 1 else "single")})
    line = {
        "metric": "scene-steps/s", "value": value, "unit": "scene-steps/s", "n_gpus": world_size,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps,
        "p50_ms": float(np.percentile(times, 50)), "p99_ms": float(np.percentile(times, 99)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if prec != "fp64" else "f64", "data": "synthetic",
        "config": cfg,
        "plain": plain,
        "speedup_vs_plain": (value / world_size) / plain["value"] if plain else None,
        "served_vs_plain": serving_rep.get("served_vs_plain") if serving_rep else None,
        "residual": dict(solve_summary(after, cap) or {}, tolerance=args.tolerance, max_iterations=cap,
                         unconverged_scenes=(solve_summary(after, cap) or {}).get("unconverged"),
                         note="last timed step; every arm runs the same solver with the same tolerance and cap"),
        "equal_residual": equal,
        "at_100_sweeps": at100,
        "roofline": doms[dom], "roofline_phases": doms,
        "phases_ms": {k: v * 1000.0 for k, v in zip(PHASE_NAMES, phases)},
        "serving": serving_rep,
        "configs": configs,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": clocks,
        "status": status,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world_size > 1:
        dist.destroy_process_group()


def run_tower(args):
    import torch
    torch.cuda.set_device(0)
    c4 = config_c4("cuda:0", steps=args.steps if args.steps > 20 else 500, cap=args.max_iterations,
                   tol=args.tolerance)   # the tower alone: at the cap given (the default bench line uses 100)
    ms = c4["precision"]["fp32_refine"]["ms_per_step"]
    line = {"metric": "scene-steps/s", "value": 1000.0 / ms, "unit": "scene-steps/s", "n_gpus": 1,
            "steps": c4["steps"], "warmup": 1, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {k: v for k, v in c4.items() if k != "precision"}, "precision": c4["precision"]}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload == "tower32" and args.impl == "ours":
        if int(os.environ.get("RANK", "0")) == 0:
            run_tower(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
