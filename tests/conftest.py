import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
FIXTURES = ["boxes8", "tower6", "spheres", "flags", "c1_boxes64", "hinges", "hinges_stab"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


def load_fixture(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as d:
        return {k: d[k] for k in d.files}


def step_slice(d, key, s):
    """Per-step ragged array ``key`` of step s from a golden fixture."""
    lens = d["step_%s_len" % key]
    off = np.concatenate([[0], np.cumsum(lens)])
    return d["step_" + key][off[s]:off[s + 1]]


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O
    O.build()
    return O
