"""The C ABI library: it loads without a GPU, exports every entry point declared in include/rainbow_b200.h, and
the ctypes mirrors of the header's structs have the C layout (field offsets compared with a compiled probe)."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "rainbow_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(rb_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("rb_step", "rb_workspace_bytes", "rb_signed_distance_grid", "rb_abi_version", "rb_last_error"):
        assert required in names


def test_library_loads_and_exports_every_declared_symbol():
    from rainbow_b200 import _native as N
    from rainbow_b200 import build
    build.build()
    lib = N.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
        assert name in N.SIGNATURES, "no ctypes signature for %s" % name
    assert lib.rb_abi_version() == 2


STRUCTS = {
    "rb_shapes": "RbShapes", "rb_bodies": "RbBodies", "rb_caps": "RbCaps", "rb_params": "RbParams",
    "rb_scene_stats": "RbSceneStats", "rb_outputs": "RbOutputs",
}


def test_struct_layouts_match_header(tmp_path):
    from rainbow_b200 import _native as N
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "rainbow_b200.h"', "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        cls = getattr(N, pyname)
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (cname, cname))
        for field, _ in cls._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (cname, field, cname, field))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = dict(line.split() for line in subprocess.check_output([str(exe)]).decode().splitlines())
    for cname, pyname in STRUCTS.items():
        cls = getattr(N, pyname)
        assert int(got[cname]) == ctypes.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert int(got["%s.%s" % (cname, field)]) == getattr(cls, field).offset, (cname, field)


def test_argument_errors_without_gpu():
    """Host-side validation answers before any device work (null descriptors, bad sizes)."""
    from rainbow_b200 import _native as N
    lib = N.load()
    size = ctypes.c_size_t(0)
    assert lib.rb_workspace_bytes(None, None, ctypes.byref(size)) == N.RB_ERR_ARG
    assert b"null" in lib.rb_last_error()
    assert lib.rb_step(None, None, None, None, None, None, 0, None) == N.RB_ERR_ARG
    out = (ctypes.c_float * 7)()
    assert lib.rb_profile_times(out, 3) == N.RB_ERR_ARG


def test_no_cpu_fallback():
    """Without a CUDA device the product path refuses to run instead of computing on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from rainbow_b200 import world as W
    from rainbow_b200._native import NativeError
    from conftest import load_fixture
    with pytest.raises(NativeError):
        W.DeviceWorld(load_fixture("boxes8"))


def test_launch_counter_is_exported_and_starts_without_device_work():
    from rainbow_b200 import _native as N
    lib = N.load()
    assert lib.rb_launch_count() >= 0
