"""The particle input and frame output of the drop-in library (CPU only).

* The importer (snow_io_import, the C face of import_particles) reads the
  reference's own sample input -- its input/groups.csv and input/particles.csv,
  kept byte for byte in tests/golden/sample_scene.npz by make_golden.py -- and
  returns exactly the records the reference's import_particles made from them.
* A frame written by snow_io_export is byte-identical to the one the
  reference's export_particles writes for the same records (oracle/_ref).
* A missing file fails with the reference's error text.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle_lib import REF_SO, ROOT

LIBSNOW = os.path.join(ROOT, "stomakhin-style-snow-simulator_b200", "libsnow.so")
GOLDEN = os.path.join(ROOT, "tests", "golden", "sample_scene.npz")
_dp = ctypes.POINTER(ctypes.c_double)


def _io():
    L = ctypes.CDLL(LIBSNOW)
    L.snow_io_import.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _dp, ctypes.c_int64]
    L.snow_io_import.restype = ctypes.c_int64
    L.snow_io_export.argtypes = [_dp, ctypes.c_int64, ctypes.c_int]
    L.snow_io_export.restype = ctypes.c_int
    L.snow_io_last_error.restype = ctypes.c_char_p
    return L


def _import(L, groups, particles):
    n = L.snow_io_import(groups.encode(), particles.encode(), None, 0)
    if n < 0:
        return n, None
    out = np.zeros((n, 26))
    assert L.snow_io_import(groups.encode(), particles.encode(), out.ctypes.data_as(_dp), n) == n
    return n, out


def test_import_reproduces_reference_import_of_its_sample_input(tmp_path):
    g = np.load(GOLDEN)
    (tmp_path / "groups.csv").write_bytes(g["groups_csv"].tobytes())
    (tmp_path / "particles.csv").write_bytes(g["particles_csv"].tobytes())
    n, got = _import(_io(), str(tmp_path / "groups.csv"), str(tmp_path / "particles.csv"))
    assert n == g["imported"].shape[0] == 957
    assert np.array_equal(got, g["imported"])


def test_import_capacity_and_missing_file(tmp_path):
    L = _io()
    g = np.load(GOLDEN)
    (tmp_path / "groups.csv").write_bytes(g["groups_csv"].tobytes())
    (tmp_path / "particles.csv").write_bytes(g["particles_csv"].tobytes())
    small = np.zeros((10, 26))
    assert L.snow_io_import(str(tmp_path / "groups.csv").encode(), str(tmp_path / "particles.csv").encode(),
                            small.ctypes.data_as(_dp), 10) == -2
    missing = str(tmp_path / "nope.csv")
    assert L.snow_io_import(missing.encode(), str(tmp_path / "particles.csv").encode(), None, 0) == -1
    assert L.snow_io_last_error().decode() == "File not open: " + missing


def _reference():
    R = ctypes.CDLL(REF_SO)
    R.ref_import.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _dp, ctypes.c_int64]
    R.ref_import.restype = ctypes.c_int64
    R.ref_last_error.restype = ctypes.c_char_p
    return R


def _large_input(tmp_path, n=200_000, edits=None, seed=11):
    """groups.csv with 5 groups and a particles.csv of n lines (about 12 MB, so
    the importer parses it in several parts), some lines ending in CRLF and
    some blank lines between them; `edits` replaces particle lines by index."""
    rng = np.random.default_rng(seed)
    g = tmp_path / "groups.csv"
    g.write_text("group_id,vx,vy,vz,mass\n" + "".join(
        f"{i},{float(rng.normal())!r},{float(rng.normal())!r},{float(rng.normal())!r},"
        f"{float(rng.uniform(1e-4, 1e-3))!r}\n" for i in range(5)))
    gid = rng.integers(0, 5, n).tolist()
    x = rng.uniform(-1, 1, (n, 3)).tolist()
    lines = [f"{gid[i]},{x[i][0]!r},{x[i][1]!r},{x[i][2]!r}" for i in range(n)]
    for i, text in (edits or {}).items():
        lines[i] = text
    body = []
    for i, line in enumerate(lines):
        body.append(line + ("\r\n" if i % 997 == 0 else "\n"))
        if i % 1231 == 0:
            body.append("\n")
    p = tmp_path / "particles.csv"
    p.write_text("group_id,x,y,z\n" + "".join(body))
    return str(g), str(p)


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference build (oracle/_ref) not present")
def test_import_of_a_large_input_matches_the_reference(tmp_path):
    """The importer parses large files in parallel parts: the records are the
    reference's, in file order, CRLF lines and blank lines included."""
    g, p = _large_input(tmp_path)
    n, got = _import(_io(), g, p)
    R = _reference()
    want = np.zeros((n, 26))
    assert R.ref_import(g.encode(), p.encode(), want.ctypes.data_as(_dp), n) == n == 200_000
    assert np.array_equal(got, want)


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("edits", [
    {10: "9,0.1,0.2,0.3", 180_000: "1,0.1,0.2"},      # undefined group early, missing field late
    {10: "9,0.1,0.2,0.3", 150_000: "8,0.1,0.2,0.3"},  # two undefined groups
    {5_000: "1,,0.2,0.3", 190_000: "1,0.1,0.2"},      # empty field early, missing field late
    {190_000: "1,abc,0.2,0.3"},                       # not a number
], ids=["parse-error-wins", "first-undefined-group", "first-parse-error", "not-a-number"])
def test_import_errors_of_a_large_input_match_the_reference(tmp_path, edits):
    """Errors of a file parsed in parallel parts are the reference's sequential
    ones: a malformed line anywhere before an undefined group, and of each kind
    the first in file order, with the reference's message."""
    g, p = _large_input(tmp_path, edits=edits)
    L, R = _io(), _reference()
    assert R.ref_import(g.encode(), p.encode(), None, 0) == -1
    assert L.snow_io_import(g.encode(), p.encode(), None, 0) == -1
    assert L.snow_io_last_error() == R.ref_last_error()


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference build (oracle/_ref) not present")
def test_export_matches_reference_export_byte_for_byte(tmp_path):
    g = np.load(GOLDEN)
    rec = np.ascontiguousarray(g["step10"])
    # formatting corner cases, then numbers of every magnitude and sign
    rec[:12, 0] = [0.0, -0.0, 1e-300, 12345.678901234, -7.5e-7, 4e-320, 999999.5, 123456.5, 1e21,
                   0.000123456789, np.inf, -np.inf]
    rng = np.random.default_rng(5)
    mags = 10.0 ** rng.uniform(-12, 12, (rec.shape[0] - 12, 3))
    rec[12:, 0:3] = mags * rng.choice([-1.0, 1.0], mags.shape)
    L = _io()
    R = ctypes.CDLL(REF_SO)
    R.ref_export.argtypes = [_dp, ctypes.c_int64, ctypes.c_int]
    cwd = os.getcwd()
    try:
        for who, d in (("ours", tmp_path / "a"), ("ref", tmp_path / "b")):
            (d / "output").mkdir(parents=True)
            os.chdir(d)
            if who == "ours":
                assert L.snow_io_export(rec.ctypes.data_as(_dp), rec.shape[0], 7) == 0
            else:
                R.ref_export(rec.ctypes.data_as(_dp), rec.shape[0], 7)
    finally:
        os.chdir(cwd)
    a = (tmp_path / "a" / "output" / "frame_000007.csv").read_bytes()
    b = (tmp_path / "b" / "output" / "frame_000007.csv").read_bytes()
    assert a == b and a.startswith(b"x,y,z\n") and a.count(b"\n") == rec.shape[0] + 1


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference build (oracle/_ref) not present")
def test_large_export_is_formatted_in_parts_and_matches_reference(tmp_path):
    """A frame of 100,003 particles is formatted by several threads (16,384
    rows or more each) and written in order: still byte for byte the
    reference's export of the same records."""
    rng = np.random.default_rng(9)
    n = 100_003
    rec = np.zeros((n, 26))
    mags = 10.0 ** rng.uniform(-8, 8, (n, 3))
    rec[:, 0:3] = mags * rng.choice([-1.0, 1.0], mags.shape)
    L = _io()
    R = ctypes.CDLL(REF_SO)
    R.ref_export.argtypes = [_dp, ctypes.c_int64, ctypes.c_int]
    cwd = os.getcwd()
    try:
        for who, d in (("ours", tmp_path / "a"), ("ref", tmp_path / "b")):
            (d / "output").mkdir(parents=True)
            os.chdir(d)
            if who == "ours":
                assert L.snow_io_export(rec.ctypes.data_as(_dp), n, 3) == 0
            else:
                R.ref_export(rec.ctypes.data_as(_dp), n, 3)
    finally:
        os.chdir(cwd)
    a = (tmp_path / "a" / "output" / "frame_000003.csv").read_bytes()
    b = (tmp_path / "b" / "output" / "frame_000003.csv").read_bytes()
    assert a.count(b"\n") == n + 1 and a == b
