"""Build recipe of the native library libgodunov2d.so (sm_100a).

The translation units get different floating-point flags: the
reference-exact FP64 kernels (kernels_f64.cu, kernels_tf_f64.cu,
gd2d_noalloc.cu) are built with -fmad=false, the mixed-precision kernels
(kernels_mixed.cu, kernels_tf_mixed.cu) with -use_fast_math, the host code with the defaults.  The library is
written in-tree next to this file so that it travels with the repository.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libgodunov2d.so")
BUILD_DIR = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + CSRC, "-I" + INCLUDE]

# (source, extra flags)
UNITS = [
    ("kernels_f64.cu", ["-fmad=false"]),
    ("kernels_tf_f64.cu", ["-fmad=false"]),
    ("kernels_mixed.cu", ["-use_fast_math"]),
    ("kernels_tf_mixed.cu", ["-use_fast_math"]),
    ("gd2d_api.cu", []),
    ("gd2d_noalloc.cu", ["-fmad=false"]),
]


def _sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cuh", ".h", ".cpp")):
            out.append(os.path.join(CSRC, name))
    out.append(os.path.join(INCLUDE, "godunov2d.h"))
    return out


def _digest() -> str:
    h = hashlib.sha256()
    for p in _sources():
        with open(p, "rb") as f:
            h.update(os.path.basename(p).encode())
            h.update(f.read())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile (if sources changed) and return the path of the library."""
    stamp = os.path.join(BUILD_DIR, "stamp")
    dig = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == dig:
                return LIB
    os.makedirs(BUILD_DIR, exist_ok=True)
    # a failed rebuild must not leave the previous library to be loaded
    for stale in (LIB, stamp):
        if os.path.exists(stale):
            os.remove(stale)
    objs, procs = [], []
    for src, extra in UNITS:  # translation units compile in parallel
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD_DIR, src + ".o")
        cmd = [NVCC] + ARCH + COMMON + extra + ["-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((cmd, subprocess.Popen(cmd)))
        objs.append(obj)
    for cmd, p in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, cmd)
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    with open(stamp, "w") as f:
        f.write(dig)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
