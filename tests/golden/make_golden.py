"""Generates the golden fixtures under tests/golden/ from the REFERENCE itself.

Runs the reference solver's own code -- src/import.cpp, src/grid.cpp and
src/collision.cpp compiled unmodified against the project's Eigen-subset shim
into oracle/_ref/libsnow_ref.so by oracle/Makefile -- and stores its outputs:

  sample_scene.npz   the reference's sample input (input/groups.csv +
                     input/particles.csv, 957 particles; the two files' bytes
                     are kept as groups_csv / particles_csv so the importer
                     can be tested on them) imported by the reference's
                     import_particles, setup() at dx = 0.05, then 1 and 10
                     step() calls with the parameters of src/main.cpp
  cube_scene.npz     an 8^3 jittered lattice cube (seed 0) with the small-case
                     material, setup() at dx = 0.02, then 1 and 10 steps with a
                     ground plane the lower particles already touch

Run from the repository root, with the reference tree's location given as
the argument or in the environment variable SNOW_REFERENCE_DIR:
    python tests/golden/make_golden.py [/path/to/reference]
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "stomakhin-style-snow-simulator_b200"))
sys.path.insert(0, os.path.dirname(HERE))

from oracle_lib import REF_SO, Reference  # noqa: E402
from snow_b200 import scenes  # noqa: E402


def main_params() -> np.ndarray:
    """step() arguments of the reference's src/main.cpp:14-29,37."""
    E, nu = 2.5e5, 0.2
    mu0 = E / (2 * (1 + nu))
    lam0 = E * nu / ((1 + nu) * (1 - 2 * nu))
    return np.array([0, -10, 0, 0.0005, 0.05, mu0, lam0, 10.0, 0.015, 0.0075, 0.95])


def import_sample(ref_root: str) -> np.ndarray:
    L = ctypes.CDLL(REF_SO)
    L.ref_import.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int64]
    L.ref_import.restype = ctypes.c_int64
    g = os.path.join(ref_root, "input", "groups.csv").encode()
    p = os.path.join(ref_root, "input", "particles.csv").encode()
    n = L.ref_import(g, p, None, 0)
    assert n > 0, n
    out = np.zeros((n, 26))
    assert L.ref_import(g, p, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n) == n
    return out


def file_bytes(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        return np.frombuffer(f.read(), dtype=np.uint8)


def main(ref_root: str | None = None) -> None:
    ref_root = ref_root or os.environ.get("SNOW_REFERENCE_DIR")
    if not ref_root:
        sys.exit("give the reference tree as the argument or in SNOW_REFERENCE_DIR")
    ref = Reference()
    # sample scene, exactly as src/main.cpp drives it
    rec = import_sample(ref_root)
    prm = main_params()
    planes = np.array([[0, 0, 0, 0, 1, 0, 1.0]])  # make_plane({0,0,0},{0,1,0}, 1)
    s0 = ref.setup(rec, 0.05)
    s1, _ = ref.step(s0, prm, planes, 1)
    s10, _ = ref.step(s0, prm, planes, 10)
    np.savez_compressed(os.path.join(HERE, "sample_scene.npz"), imported=rec, setup=s0, step1=s1,
                        step10=s10, params=prm, planes=planes, dx=0.05,
                        groups_csv=file_bytes(os.path.join(ref_root, "input", "groups.csv")),
                        particles_csv=file_bytes(os.path.join(ref_root, "input", "particles.csv")))
    # small cube resting on the ground plane (contact from the first step)
    cube = scenes.cube(8, lo=(0.46, 0.045, 0.46), velocity=(0.5, -1.5, 0.25), seed=0)
    sc = scenes.Scene(cube, dx=0.02, dt=1e-4, steps=10, material=scenes.Material(),
                      planes=[scenes.GROUND])
    c0 = ref.setup(cube, sc.dx)
    c1, _ = ref.step(c0, sc.params(), sc.plane_array(), 1)
    c10, _ = ref.step(c0, sc.params(), sc.plane_array(), 10)
    np.savez_compressed(os.path.join(HERE, "cube_scene.npz"), setup_in=cube, setup=c0, step1=c1,
                        step10=c10, params=sc.params(), planes=sc.plane_array(), dx=sc.dx)
    print("wrote", os.path.join(HERE, "sample_scene.npz"), os.path.join(HERE, "cube_scene.npz"))


if __name__ == "__main__":
    main(*sys.argv[1:])
