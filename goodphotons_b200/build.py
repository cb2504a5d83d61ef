"""Build the native library libftb200.so in-tree (sm_100a only).

    python -m goodphotons_b200.build [-v]

The kernels are compiled with -fmad=false: the path's fp64 arithmetic must round every
product separately, like the reference's x86-64 CPU build, so that photon paths match it
operation for operation.  The fp32 traversal uses explicit fmaf, which that flag leaves
alone.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
OUT_DIR = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libftb200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, flush=True)
    return r


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(verbose=False, force=False):
    nvcc = _nvcc()
    os.makedirs(OUT_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith(".h")]
    headers.append(os.path.join(PKG, "..", "include", "ftb200.h"))
    objs = []
    units = [
        ("ftb_kernels.cu", [*ARCH, "-O3", "-lineinfo", "-fmad=false", "-std=c++17",
                            "-Xcompiler", "-fPIC", "-Xptxas", "-v" if verbose else "-O3"]),
        ("ftb_noalloc.cu", [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]),
        ("ftb_api.cpp", ["-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off"]),
        ("bvh_build.cpp", ["-O2", "-std=c++17", "-Xcompiler", "-fPIC"]),
        ("bvh_device.cu", [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]),
        ("ftb_server.cpp", ["-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-pthread"]),
    ]
    for src, flags in units:
        s = os.path.join(CSRC, src)
        o = os.path.join(OUT_DIR, src + ".o")
        if force or _stale(o, [s, *headers]):
            _run([nvcc, "-c", s, "-o", o, *flags], verbose)
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([nvcc, "-shared", *ARCH, "-o", LIB, *objs, "-lpthread"], verbose)
    return LIB


def build_oracle(verbose=False, reference=None):
    """The CPU checkers under oracle/ (test infrastructure).  `reference` (or the
    FTB_REFERENCE environment variable) names a checkout of the reference, whose headers
    the reference-built checkers under oracle/_ref are compiled from; without one only the
    plain-C restatement is built."""
    root = os.path.dirname(PKG)
    ref = reference or os.environ.get("FTB_REFERENCE", "")
    cmd = ["make", "-s", "-C", os.path.join(root, "oracle")]
    if ref:
        cmd.append(f"REF={ref}")
    _run(cmd, verbose)


if __name__ == "__main__":
    v = "-v" in sys.argv
    print(build(verbose=v, force="-f" in sys.argv))
