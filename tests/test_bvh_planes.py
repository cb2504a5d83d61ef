"""The wide BVH's float planes are conservative: compiles tests/bvh_planes_check.cpp against
the host builder (goodphotons_b200/csrc/bvh_build.cpp) and runs it.  Every primitive's box,
grown by the scene margin, must lie inside the planes of every child slot on its path from
the root -- for the builder's own outward-rounded planes, for the planes decoded from the
8-bit form, and after a refit -- on unit-cube, far-from-origin, repeated and flat, and
mixed-scale box sets; a plane moved inward by one float step must be caught."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "goodphotons_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_float_planes_enclose_every_primitive(tmp_path):
    exe = str(tmp_path / "bvh_planes_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, os.path.join(ROOT, "tests", "bvh_planes_check.cpp"),
                    os.path.join(CSRC, "bvh_build.cpp"), "-o", exe], check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    lines = r.stdout.strip().splitlines()
    assert r.returncode == 0, r.stdout + r.stderr
    assert len(lines) == 17 and all(l.endswith(": ok") for l in lines[:16]), r.stdout
    assert lines[16].endswith("caught"), r.stdout
