"""Host-side arithmetic of bench.py (CPU): the roofline line, the algorithmic
bytes it divides, the per-quantity errors and the served tick summary.

The roofline's `bound` must be the measured roof the kernel comes closest to,
not a fixed choice; achieved = algorithmic bytes (or executed FLOPs) per
launch over the launch time; the served summary must separate the typical gap
between ticks (median) from the few long ones.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

PEAKS = {"fp64_tflops": 37.2, "fp32_tflops": 72.6, "fp32x2_tflops": 73.9}


def test_alg_bytes_per_kernel():
    n, nodes = 1000, 300
    ab = bench.alg_bytes(n, nodes, 8)
    assert ab["p2g"] == n * 13 * 8 + nodes * 7 * 8
    # g2p: 17 reals + F_P and id read, 23 reals + F_P, id, key and position written, 6 reals per node
    assert ab["g2p"] == n * (17 * 8 + 76) + nodes * 6 * 8 + n * (23 * 8 + 84)
    assert bench.alg_bytes(n, nodes, 4)["p2g"] < ab["p2g"]


def test_kernel_roofline_arithmetic_and_bound():
    n = 650_000
    ms = 0.1555
    alg = 315_563_520
    r = bench.kernel_roofline("g2p", ms, alg, n, "tori", "fp64", PEAKS)
    hbm = r["roofs"]["hbm"]
    assert hbm["achieved"] == pytest.approx(alg / (ms * 1e-3) / 1e9)
    assert hbm["frac"] == pytest.approx(hbm["achieved"] / hbm["peak"])
    # executed FP64 FLOPs from the committed ncu counts, against the measured FMA peak
    assert "fp64" in r["roofs"]
    fp = r["roofs"]["fp64"]
    assert fp["frac"] == pytest.approx(fp["achieved"] / PEAKS["fp64_tflops"])
    assert r["bound"] == max(r["roofs"], key=lambda k: r["roofs"][k]["frac"])
    assert r["frac"] == r["roofs"][r["bound"]]["frac"]
    # ten times the bytes in the same time: the HBM roof is then the closest one
    slow = bench.kernel_roofline("g2p", ms, alg * 10, n, "tori", "fp64", PEAKS)
    assert slow["bound"] == "hbm"


def test_roofline_line_takes_the_longest_kernel():
    per = {"p2g": 0.12, "stress_update": 0.16}
    ab = bench.alg_bytes(650_000, 60_000, 8)
    line = bench.roofline_line(per, ab, 650_000, "tori", "fp64", PEAKS)
    assert line["kernel"] == "g2p" and line["launch_ms"] == 0.16
    assert set(line["kernels"]) == {"p2g", "g2p"}
    assert line["hbm_frac"] == pytest.approx(line["kernels"]["g2p"]["roofs"]["hbm"]["frac"])


def test_errors_per_quantity():
    rng = np.random.default_rng(3)
    a = rng.normal(size=(50, 26))
    assert all(v == 0.0 for v in bench.errors(a, a).values())
    b = a.copy()
    b[7, 17:26] *= 1 + 1e-6  # F_E of one particle
    e = bench.errors(b, a)
    assert e["F_E"] == pytest.approx(1e-6, rel=1e-3) and e["x"] == e["v"] == e["F_P"] == 0.0


def test_tick_summary_separates_typical_and_long_gaps():
    ticks, t = [], 0.0
    for k in range(10):
        gap = 0.02 if k == 5 else 3e-6  # one long stall
        t += gap
        ticks.append({"device_start_s": t, "device_end_s": t + 0.01, "steps": 8})
        t += 0.01
    s = bench.tick_summary(ticks, wall_s=t)
    assert s["median_gap_ms"] == pytest.approx(3e-3)
    assert s["gaps_over_1ms"] == 1 and s["gap_ms_in_those"] == pytest.approx(20.0)
    assert s["device_busy_frac"] == pytest.approx(0.1 / t)
    assert s["mean_steps_per_tick"] == 8
    assert bench.tick_summary([], 1.0) == {}
