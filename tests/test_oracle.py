"""The oracle pinned against the reference: known answers and golden outputs (CPU only)."""
import os
import subprocess

import numpy as np
import pytest

from oracle_lib import ROOT, Reference, errors, reference_available

GOLDEN = os.path.join(ROOT, "tests", "golden")


def test_known_answers_of_reference_unit_tests(oracle):
    """oracle/oracle_tests restates tests/snow_tests.cpp:30-407 of the reference (24 cases)."""
    exe = os.path.join(ROOT, "oracle", "oracle_tests")
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "24 reference cases + svd checks: all passed" in r.stdout


def test_bspline_known_values(oracle):
    # tests/snow_tests.cpp:30-60
    assert abs(oracle.N(1, 1) - 2 / 3) < 1e-10 and abs(oracle.N(1, 2) - 1 / 6) < 1e-10
    assert oracle.N(1, 3) == 0 and oracle.N(1, 10) == 0
    assert abs(oracle.N_dash(0, 0.5) + 0.625) < 1e-10 and abs(oracle.N_dash(0, 1) + 0.5) < 1e-10


@pytest.mark.parametrize("name", ["sample_scene", "cube_scene"])
def test_oracle_matches_reference_golden(oracle, name):
    """Golden outputs written by tests/golden/make_golden.py from the reference's own code."""
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    start = g["imported"] if name == "sample_scene" else g["setup_in"]
    s0 = oracle.setup(start, float(g["dx"]))
    assert np.max(np.abs(s0[:, 7] - g["setup"][:, 7]) / np.abs(g["setup"][:, 7])) < 1e-12
    s1, _ = oracle.step(g["setup"], g["params"], g["planes"], 1)
    s10, _ = oracle.step(g["setup"], g["params"], g["planes"], 10)
    for got, want in ((s1, g["step1"]), (s10, g["step10"])):
        e = errors(got, want)
        assert max(e.values()) < 1e-12, e


@pytest.mark.skipif(not reference_available(), reason="reference build (oracle/_ref) not present")
def test_reference_own_unit_tests_pass_with_shim():
    exe = os.path.join(ROOT, "oracle", "_ref", "snow_tests")
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0 and "all tests passed" in r.stdout, r.stdout + r.stderr


@pytest.mark.skipif(not reference_available(), reason="reference build (oracle/_ref) not present")
def test_oracle_matches_reference_trajectory(oracle):
    from snow_b200 import scenes

    sc = scenes.cube_scene(12, steps=20)
    ref = Reference()
    a = oracle.setup(sc.particles, sc.dx)
    b = ref.setup(sc.particles, sc.dx)
    assert np.array_equal(a[:, 7], b[:, 7]) or np.max(np.abs(a[:, 7] / b[:, 7] - 1)) < 1e-13
    a, _ = oracle.step(a, sc.params(), sc.plane_array(), 20)
    b, _ = ref.step(b, sc.params(), sc.plane_array(), 20)
    e = errors(a, b)
    assert max(e.values()) < 1e-12, e
