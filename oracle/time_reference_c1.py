"""Times the reference's own NumPy step (api.py:676 simulate) on the 64-box lattice (4^3 unit boxes, spacing
1.05, jitter 0.02, SDF resolution 32, the reference's parameters) beside the oracle's restatement of the same
step on the same core, from the same scene, for a few steps.

MEASUREMENT INFRASTRUCTURE, run where the reference checkout is present (it is not on GPU hosts):

    python oracle/time_reference_c1.py [steps]

The scene is built by the reference's own API calls (tests/golden/make_golden.py, with its two import
stand-ins); the oracle steps the arrays read from that engine.  Prints one JSON line: seconds per step of each,
their ratio, and whether the two agree bit for bit after the timed steps.
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if sys.path and os.path.abspath(sys.path[0]) == HERE:   # run as a script: import the package, not oracle.py
    sys.path.pop(0)
sys.path[:0] = [ROOT, os.path.join(ROOT, "tests", "golden")]


def main():
    import numpy as np
    import make_golden as MG
    from oracle import oracle as O
    from rainbow_b200 import engine_io
    steps = int(sys.argv[1]) if len(sys.argv) > 1 else 3
    engine = MG.scene_box_lattice(4, 1.05, 0.02, 32, seed=0, params={"max_iterations": 100,
                                                                      "relative_tolerance": 1e-6})
    arrays = engine_io.scene_arrays(engine)
    sc = O.OracleScene(arrays)
    t0 = time.perf_counter()
    for _ in range(steps):
        o = sc.step()
    t_oracle = (time.perf_counter() - t0) / steps
    dt = engine.params.time_step
    t0 = time.perf_counter()
    for _ in range(steps):
        MG.API.simulate(engine, dt)
    t_ref = (time.perf_counter() - t0) / steps
    x, u = engine_io.body_state(engine)
    same = bool(np.array_equal(x.ravel(), o["x"]) and np.array_equal(u.ravel(), o["u"]))
    print(json.dumps({"scene": "box_lattice_64 (reference API), SDF 32, reference parameters", "steps": steps,
                      "reference_numpy_s_per_step": t_ref, "oracle_s_per_step": t_oracle,
                      "oracle_speedup_over_reference": t_ref / t_oracle, "bit_identical": same,
                      "cores": 1, "host": os.uname().machine}))


if __name__ == "__main__":
    main()
