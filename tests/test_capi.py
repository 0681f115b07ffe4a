"""The C ABI library loads and exports every entry point include/snow_gpu.h declares (CPU only)."""
import ctypes
import os
import re
import subprocess

from oracle_lib import ROOT

HEADER = os.path.join(ROOT, "include", "snow_gpu.h")
LIB = os.path.join(ROOT, "stomakhin-style-snow-simulator_b200", "libsnow_b200.so")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(snow_gpu_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    for n in ("snow_gpu_setup", "snow_gpu_step", "snow_gpu_make_plane", "snow_gpu_batch_step",
              "snow_gpu_stage_p2g", "snow_gpu_stage_g2p"):
        assert n in names


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build libsnow_b200.so first (make in the package directory)"
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (snow_gpu_\w+)", out))
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing


def test_library_loads_and_reports_abi_without_gpu():
    L = ctypes.CDLL(LIB)
    L.snow_gpu_abi_version.restype = ctypes.c_int
    assert L.snow_gpu_abi_version() == 2  # 2: snow_collider gained the box fields (axis, extent)
    import snow_b200

    assert ctypes.sizeof(snow_b200.Collider) == 152
    # make_plane is pure host logic: unit normal, zero velocity (src/collision.cpp:5-27)
    import snow_b200

    c = snow_b200.make_plane((0, 0.05, 0), (0, 2, 0), 0.2)
    assert list(c.normal) == [0.0, 1.0, 0.0] and list(c.velocity) == [0.0, 0.0, 0.0]
    assert c.friction == 0.2 and c.point[1] == 0.05
    z = snow_b200.make_plane((0, 0, 0), (0, 0, 0), 1.0)  # a zero normal is kept as is
    assert list(z.normal) == [0.0, 0.0, 0.0]


def test_binding_covers_header():
    import snow_b200

    L = snow_b200.lib()
    for n in declared():
        assert getattr(L, n).argtypes is not None, f"no ctypes signature for {n}"
