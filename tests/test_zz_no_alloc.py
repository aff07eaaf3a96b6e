"""rb_step_noalloc, the entry point for callers that cannot allocate device memory themselves.

Such a caller (an application that owns all device memory through its own pool, a real-time loop that must
not allocate once running) has no way to hand rb_step a workspace, so this variant keeps the step's
temporaries in a fixed scratch array inside the library.  The test first steps a larger, different scene
through the scratch (so it holds another scene's lists and counters), then steps one scene through the C ABI
with both entry points, twice in a row, and demands identical results (the FP64 step is bit-exact, so the
tolerance is zero): whatever a call leaves in the shared scratch must not leak into the next step.  This file
is collected last so that a failure here stops a run only after every other test has run.
"""
import ctypes

import numpy as np
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu


def test_noalloc_step_matches_workspace_step_twice():
    import torch
    from rainbow_b200 import _native as N
    from rainbow_b200 import world as W

    d = load_fixture("boxes8")
    params = W.make_rb_params(W.params_from_vector(d["params"]))
    with_ws = W.DeviceWorld(d)       # caller-provided workspace (rb_step)
    no_ws = W.DeviceWorld(d)         # same scene; its workspace tensor is never passed
    lib = N.load()

    need = ctypes.c_size_t(0)
    N.check(lib.rb_workspace_bytes(ctypes.byref(no_ws.rb_bodies), ctypes.byref(no_ws.caps), ctypes.byref(need)),
            "rb_workspace_bytes")
    assert need.value <= (16 << 20), "fixture scene must fit the 16 MiB scratch"

    # dirty the scratch: a few steps of the 64-box lattice (more bodies, pairs and contacts) through it
    big = load_fixture("c1_boxes64")
    big_params = W.make_rb_params(W.params_from_vector(big["params"]))
    other = W.DeviceWorld(big)
    other.step(big_params)   # with a workspace: grows the work lists to this scene's needs
    N.check(lib.rb_workspace_bytes(ctypes.byref(other.rb_bodies), ctypes.byref(other.caps), ctypes.byref(need)),
            "rb_workspace_bytes")
    assert need.value <= (16 << 20)
    for _ in range(3):
        other.t_status.zero_()
        N.check(lib.rb_step_noalloc(ctypes.byref(other.rb_shapes), ctypes.byref(other.rb_bodies),
                                    ctypes.byref(other.caps), ctypes.byref(big_params), ctypes.byref(other.rb_outputs),
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
                "rb_step_noalloc")
        torch.cuda.synchronize()
        assert int(other.t_status[0].item()) == 0 and other.n_contacts_total() > 0

    for _ in range(2):
        with_ws.t_status.zero_()
        with_ws.launch(params)
        no_ws.t_status.zero_()
        stream = torch.cuda.current_stream()
        rc = lib.rb_step_noalloc(ctypes.byref(no_ws.rb_shapes), ctypes.byref(no_ws.rb_bodies),
                                 ctypes.byref(no_ws.caps), ctypes.byref(params), ctypes.byref(no_ws.rb_outputs),
                                 ctypes.c_void_p(stream.cuda_stream))
        N.check(rc, "rb_step_noalloc")
        torch.cuda.synchronize()
        assert int(with_ws.t_status[0].item()) == 0 and int(no_ws.t_status[0].item()) == 0
        xa, ua = with_ws.state()
        xb, ub = no_ws.state()
        np.testing.assert_array_equal(xb, xa)
        np.testing.assert_array_equal(ub, ua)
        ca, cb = with_ws.contacts(), no_ws.contacts()
        for key in ("ids", "p", "n", "g", "sol"):
            np.testing.assert_array_equal(cb[key], ca[key], err_msg=key)
        sa, sb = with_ws.stats()[0], no_ws.stats()[0]
        assert (sb.n_contacts, sb.iterations, sb.exitcode) == (sa.n_contacts, sa.iterations, sa.exitcode)


def test_noalloc_rejects_batches_beyond_the_scratch():
    from rainbow_b200 import _native as N
    from rainbow_b200 import world as W

    d = load_fixture("boxes8")
    world = W.DeviceWorld(d, caps={"pairs": 1 << 16, "items": 1 << 18, "contacts": 1 << 16})
    lib = N.load()
    rc = lib.rb_step_noalloc(ctypes.byref(world.rb_shapes), ctypes.byref(world.rb_bodies),
                             ctypes.byref(world.caps), ctypes.byref(W.make_rb_params(W.params_from_vector(d["params"]))),
                             ctypes.byref(world.rb_outputs), None)
    assert rc == N.RB_ERR_WORKSPACE
    assert b"scratch" in lib.rb_last_error()
