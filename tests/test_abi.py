"""The C ABI library loads, exports every entry point the header declares, and its
structures match the ctypes mirror byte for byte.  No GPU calls here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from goodphotons_b200 import abi, build, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ftb200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ftb_[a-z0-9_]+)\s*\(", src)))


def test_exports_every_declared_symbol():
    lib = C.CDLL(build.LIB)
    names = declared_functions()
    assert set(names) == set(abi.EXPORTS)
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", build.LIB], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (ftb_\w+)", out))
    assert set(names) <= exported


def test_struct_layout_matches_header(tmp_path):
    """Compile a probe against the header and compare sizes and offsets with ctypes."""
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, py in abi.STRUCTS.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    c = tmp_path / "probe.c"
    c.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c11", str(c), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for cname, py in abi.STRUCTS.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, f"{cname}.{fname}"


def test_version_and_no_device_behaviour(L):
    assert L.L.ftb_abi_version() == abi_version_from_header()
    if not L.available():
        d = scenes.make_cornell(L)
        h = C.c_void_p()
        st = L.L.ftb_scene_create(d.ref(), 0, C.byref(h))
        assert st == 2  # FTB_ERR_NO_DEVICE
        assert "device" in L.L.ftb_last_error().decode()


def abi_version_from_header():
    return int(re.search(r"#define FTB_ABI_VERSION (\d+)", open(HEADER).read()).group(1))


def test_supported_gate(L):
    d = scenes.make_cornell(L)
    assert L.supported(d)[0] == 1
    sb = scenes.SceneBuilder()
    scenes.cornell_box(sb, boxes=False)
    sb.quad((0.5, 0.5, 0.5), (0.3, 0, 0), (0, 0.3, 0), sb.material(abi.MAT_MIRROR, reflect=sb.const(0.9)))
    assert L.supported(sb.build(L))[0] == 1            # planar mirrors: the plane connector
    sb.sphere((1, 1, 1), 0.2, sb.material(abi.MAT_MIRROR, reflect=sb.const(0.9)))
    r, why = L.supported(sb.build(L))
    assert r == 0 and "mirror sphere" in why           # the spherical mirror connector is not on the path
    sb = scenes.SceneBuilder()
    scenes.cornell_box(sb, boxes=False)
    tile = sb.material(abi.MAT_GLOSSY, reflect=sb.const(0.9), roughness=0.0)
    for k in range(65):                                 # 65 distinct planes
        sb.quad((0.1, 0.1 + 0.01 * k, 0.3), (0.2, 0, 0), (0, 0, 0.2), tile)
    r, why = L.supported(sb.build(L))
    assert r == 0 and "64 mirror planes" in why
    sb = scenes.SceneBuilder()
    scenes.cornell_box(sb, boxes=False)
    sb.sphere((1, 1, 1), 0.2, sb.material(abi.MAT_DIELECTRIC, ior=sb.cauchy(1.5, 0.004)))
    r, why = L.supported(sb.build(L))
    assert r == 0 and "sphere" in why
    sb = scenes.SceneBuilder()
    scenes.cornell_box(sb, boxes=False)
    sb.quad((0.5, 0.5, 0.5), (0.3, 0, 0), (0, 0.3, 0), 99)
    assert L.supported(sb.build(L))[0] == -1


def test_invalid_arguments_are_reported_not_fatal(L):
    assert L.L.ftb_camera_look_at(None, None, None, 40.0, 0, 0, None) == 1
    assert "camera" in L.L.ftb_last_error().decode()
    cdf = np.zeros(4)
    n = C.c_int32()
    integ = C.c_double()
    s = abi.Spectrum(abi.SPEC_CONST, 0, 0)
    st = L.L.ftb_emission_cdf(C.byref(s), None, None, 1.0, cdf.ctypes.data_as(C.POINTER(C.c_double)), 4,
                              C.byref(n), C.byref(integ))
    assert st == 1 and "small" in L.L.ftb_last_error().decode()


def test_header_constants_match_binding():
    """The no-allocation limits the header states are the binding's (the library itself
    checks its scratch array against the header's size at compile time)."""
    src = open(HEADER).read()
    get = lambda name: int(re.search(rf"#define {name} (\d+)", src).group(1))
    assert get("FTB_NOALLOC_MAX_PHOTONS") == abi.NOALLOC_MAX_PHOTONS
    assert get("FTB_NOALLOC_SCRATCH_BYTES") == abi.NOALLOC_SCRATCH_BYTES
