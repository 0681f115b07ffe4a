"""Parity of the FP64 CUDA step with the oracle and the reference's golden outputs.

Tolerance: 1e-10 relative per quantity (x, v, F_E, F_P), the bound the plain
FP64 path is held to; V_p0 from setup() to 1e-12.
"""
import os

import numpy as np
import pytest

from oracle_lib import ROOT, errors

pytestmark = pytest.mark.gpu

TOL = 1e-10
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _run_batch(snow, rec, params, planes, steps, graphs=True, dense=True):
    b = snow.Batch(snow.SNOW_FP64)
    b.set_graphs(graphs)
    b.set_dense(dense)
    sid = b.add_scene(rec, params, planes)
    b.step(steps)
    out = b.download(sid)
    b.close()
    return out


@pytest.mark.parametrize("name", ["sample_scene", "cube_scene"])
def test_setup_volume_matches_reference_golden(snow, name):
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    start = g["imported"] if name == "sample_scene" else g["setup_in"]
    out = snow.setup(start.copy(), float(g["dx"]))
    want = g["setup"]
    assert np.max(np.abs(out[:, 7] / want[:, 7] - 1)) < 1e-12
    assert np.array_equal(np.delete(out, 7, axis=1), np.delete(want, 7, axis=1))


@pytest.mark.parametrize("name", ["sample_scene", "cube_scene"])
@pytest.mark.parametrize("steps", [1, 10])
def test_step_matches_reference_golden(snow, name, steps):
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    out = _run_batch(snow, g["setup"], g["params"], g["planes"], steps)
    e = errors(out, g[f"step{steps}"])
    assert max(e.values()) < TOL, e


@pytest.mark.parametrize("steps", [1, 10])
@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("dense", [True, False])
def test_cube_32_matches_oracle(snow, oracle, steps, graphs, dense):
    """The small-case cube (32^3 = 32,768 particles) against the oracle, with
    the counting sort over dense key bins and with the radix-sort fallback."""
    from snow_b200 import scenes

    sc = scenes.cube_scene(32)
    rec = oracle.setup(sc.particles, sc.dx)
    want, _ = oracle.step(rec, sc.params(), sc.plane_array(), steps)
    got = _run_batch(snow, rec, sc.params(), sc.planes, steps, graphs, dense)
    e = errors(got, want)
    assert max(e.values()) < TOL, e


def test_literal_step_entry_point(snow, oracle):
    """snow_gpu_step: upload, step, download on every call (the drop-in step())."""
    from snow_b200 import scenes

    sc = scenes.cube_scene(10)
    rec = snow.setup(sc.particles.copy(), sc.dx)
    want, _ = oracle.step(rec, sc.params(), sc.plane_array(), 3)
    got = rec.copy()
    for _ in range(3):
        t = snow.step(got, sc.params(), sc.planes, 1, timings=True)
        assert t["p2g"] > 0 and t["stress_update"] > 0
    e = errors(got, want)
    assert max(e.values()) < TOL, e


def test_step_calls_in_sorted_order(snow, oracle):
    """Consecutive snow_gpu_step calls on as many records place them in the
    order the last step left (block-sorted).  Results follow the caller's
    records: chained calls equal the oracle's steps, and a call on the same
    records shuffled equals the oracle on the shuffled records, row for row."""
    from snow_b200 import scenes

    sc = scenes.tori_scene(n_per_torus=6000, steps=4)
    sc.particles[:, 0] += np.where(sc.particles[:, 3] > 0, 0.12, -0.12)  # start in contact
    rec = oracle.setup(sc.particles, sc.dx)
    want, _ = oracle.step(rec, sc.params(), sc.plane_array(), 3)
    got = rec.copy()
    snow.step(got, sc.params(), sc.planes, 1)
    snow.step(got, sc.params(), sc.planes, 2)
    e = errors(got, want)
    assert max(e.values()) < TOL, e
    perm = np.random.default_rng(5).permutation(got.shape[0])
    mixed = got[perm].copy()
    want2, _ = oracle.step(mixed, sc.params(), sc.plane_array(), 1)
    snow.step(mixed, sc.params(), sc.planes, 1)
    e = errors(mixed, want2)
    assert max(e.values()) < TOL, e


def test_colliding_tori_small(snow, oracle):
    """Two small tori at +-8 m/s meeting over a few steps, against the oracle."""
    from snow_b200 import scenes

    sc = scenes.tori_scene(n_per_torus=6000, steps=10)
    sc.particles[:, 0] += np.where(sc.particles[:, 3] > 0, 0.12, -0.12)  # start in contact
    rec = oracle.setup(sc.particles, sc.dx)
    want, _ = oracle.step(rec, sc.params(), sc.plane_array(), 10)
    got = _run_batch(snow, rec, sc.params(), sc.planes, 10)
    e = errors(got, want)
    assert max(e.values()) < TOL, e


def test_negative_coordinates(snow, oracle):
    """Signed block keys: a cube straddling the origin (the sample input has x, z < 0)."""
    from snow_b200 import scenes

    rec = scenes.cube(8, lo=(-0.05, -0.03, -0.07), velocity=(0.3, -1.0, 0.2), seed=4)
    sc = scenes.Scene(rec, dx=0.02, dt=1e-4, steps=5, material=scenes.Material(),
                      planes=[((0, -0.2, 0), (0, 1, 0), 0.3)])
    r0 = oracle.setup(rec, sc.dx)
    want, _ = oracle.step(r0, sc.params(), sc.plane_array(), 5)
    got = _run_batch(snow, r0, sc.params(), sc.planes, 5)
    e = errors(got, want)
    assert max(e.values()) < TOL, e


def test_device_stencil_weights_match_reference_spline(snow, oracle):
    """The kernels' own branch-free weights and slopes (axis_weights, run on
    the device in double) against the reference's N and N_dash (grid.cpp:24-58,
    through the oracle) at random positions, on the grid knots and one ulp to
    either side: the same stencil base, weights within 2e-15 and slopes within
    2e-15 / dx; the weights sum to 1 and the slopes to 0.  The float form
    (the mixed path) against the same functions at |x / dx| <= 5, away from
    the knots: its single-precision grid position x / dx may differ from the
    double one by two ulp, so within 4e-6."""
    rng = np.random.default_rng(17)
    dx = 0.02
    knots = np.arange(-50, 50) * dx
    xs = np.concatenate([rng.uniform(-1.0, 1.0, 2000), knots, np.nextafter(knots, 10), np.nextafter(knots, -10)])
    base, w, dw = snow.stage_weights(xs, dx, 0)
    tol = 2e-15
    for i, x in enumerate(xs):
        gp = x / dx
        b = int(np.floor(gp)) - 1
        assert base[i] == b, (x, base[i], b)
        for k in range(4):
            assert abs(w[i, k] - oracle.N(b + k, gp)) <= tol, (x, k)
            assert abs(dw[i, k] - oracle.N_dash(b + k, gp) / dx) <= tol / dx, (x, k)
    assert np.abs(w.sum(axis=1) - 1).max() <= 4 * tol
    assert np.abs(dw.sum(axis=1)).max() <= 8 * tol / dx
    xf = rng.uniform(-0.1, 0.1, 2000)
    fr = xf / dx - np.floor(xf / dx)
    xf = xf[(fr > 1e-4) & (fr < 1 - 1e-4)]
    base, w, dw = snow.stage_weights(xf, dx, 1)
    for i, x in enumerate(xf):
        gp = x / dx
        b = int(np.floor(gp)) - 1
        assert base[i] == b, (x, base[i], b)
        for k in range(4):
            assert abs(w[i, k] - oracle.N(b + k, gp)) <= 4e-6, (x, k)
            assert abs(dw[i, k] - oracle.N_dash(b + k, gp) / dx) <= 4e-6 / dx, (x, k)
