"""Build recipe of the CUDA library (sm_100a) into ``rainbow_b200/lib/librainbow_b200.so``."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SOURCES = ["csrc/rb_step.cu", "csrc/rb_sdf.cu", "csrc/rb_batch.cu"]
HEADERS = ["csrc/rb_device.cuh", "csrc/rb_layout.h", "csrc/rb_internal.h", "../include/rainbow_b200.h"]
OUT = os.path.join(HERE, "lib", "librainbow_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    # FP64 parity: fuse nothing implicitly; the kernels spell out the fused multiply-adds NumPy performs
    "-fmad=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(os.path.join(HERE, f)) > t for f in SOURCES + HEADERS)


def build(force=False, verbose=False):
    """Compile the library if a source changed (or force).  Returns the library path."""
    if not force and not _stale():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-I", os.path.join(ROOT, "include")]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += ["-o", OUT] + [os.path.join(HERE, s) for s in SOURCES]
    subprocess.check_call(cmd, cwd=HERE)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
