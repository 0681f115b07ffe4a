#!/usr/bin/env python
"""Benchmark of the B200 explicit-MPM snow step (one JSON line on rank 0).

Default workload: two colliding snow tori, 650,000 particles, dx = 0.01,
dt = 2e-5, plain FP64 path -- the configuration the headline metric is quoted
on.  A "step" is one explicit MPM timestep over the whole scene.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload tori|cube|snowball|batch] [--precision fp64|mixed]

* value        particle-steps/s with the scene resident in HBM, device time of
               K CUDA-graph-replayed steps (CUDA events on the launching stream),
               max over ranks; ranks run independent replicas (weak scaling)
* e2e          the same metric through the drop-in entry point snow_gpu_step on
               pinned host records: every step uploads the 208-byte records,
               steps and downloads them
* roofline     the dominant kernel's algorithmic bytes per launch over its mean
               launch time (CUDA events around each kernel over K steps of the
               same workload), against the measured HBM copy bandwidth
* cpu_baseline the reference's own CPU step (oracle/_ref: reference sources with
               the Eigen-subset shim, OpenMP on all host cores) on a bounded
               number of full-scene steps of the same workload
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "stomakhin-style-snow-simulator_b200")
sys.path.insert(0, PKG)

import numpy as np  # noqa: E402

REF_SAMPLE_S = 20.0    # target seconds of reference CPU work per bounded sample


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tori", choices=["tori", "touching", "cube", "snowball", "batch", "served"],
                    help="batch: the 256 independent scenes, split across ranks by work (strong scaling); "
                         "touching: the two tori placed in contact (plastic flow from the first steps); "
                         "served: the request stream through the server (single GPU)")
    ap.add_argument("--particles", type=int, default=0,
                    help="tori/touching with this many particles instead of 650,000 (small cases for ncu)")
    ap.add_argument("--requests", type=int, default=512, help="served: number of requests in the stream")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the mixed / batched / served forms")
    return ap.parse_args()


def workload(name: str, particles: int = 0):
    from snow_b200 import scenes

    per = particles // 2 if particles else 325_000
    if name == "tori":
        return scenes.tori_scene(n_per_torus=per)
    if name == "touching":
        return scenes.tori_scene(n_per_torus=per, gap=0.0)
    if name == "cube":
        return scenes.cube_scene(32)
    return scenes.snowball_scene()


def describe(sc) -> dict:
    return {"workload": sc.name, "particles": sc.n, "dx": sc.dx, "dt": sc.dt,
            "colliders": len(sc.planes), "theta_c": sc.material.theta_c, "E": sc.material.E}


# ------------------------------------------------------------------ ranks
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# --------------------------------------------------------------- reference
def reference_lib():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import REF_SO, Oracle, Reference

    if os.path.exists(REF_SO):
        return Reference(), "reference", "reference sources (src/grid.cpp et al.) + Eigen-subset shim, OpenMP"
    return Oracle(), "port", "oracle restatement of src/grid.cpp, OpenMP"


def cpu_rate(sc, max_steps: int, budget_s: float = REF_SAMPLE_S):
    """Reference CPU particle-steps/s over a bounded number of full-scene steps."""
    lib, kind, what = reference_lib()
    rec = lib.setup(sc.particles, sc.dx)
    # one step to size the sample, then the timed sample
    rec, ms = lib.step(rec, sc.params(), sc.plane_array(), 1)
    per_step = ms[10] / 1e3
    steps = int(max(1, min(max_steps, budget_s // max(per_step, 1e-3))))
    rec, ms = lib.step(rec, sc.params(), sc.plane_array(), steps)
    wall = ms[10] / 1e3
    return sc.n * steps / wall, steps, wall, kind, what


def cpu_rate_batch(scs, budget_s: float = REF_SAMPLE_S):
    """Reference CPU particle-steps/s over the batch scenes: each scene in turn
    (a few steps each, as one process would step them) until the budget is spent."""
    lib, kind, what = reference_lib()
    done_ps, wall, used, steps_each = 0.0, 0.0, 0, 5
    for sc in scs:
        rec = lib.setup(sc.particles, sc.dx)
        rec, ms = lib.step(rec, sc.params(), sc.plane_array(), steps_each)
        done_ps += sc.n * steps_each
        wall += ms[10] / 1e3
        used += 1
        if wall > budget_s:
            break
    return done_ps / wall, steps_each, wall, kind, f"{what}; {used} of {len(scs)} scenes, {steps_each} steps each"


def run_reference(args, ws, rank):
    if rank != 0:
        return
    if args.workload == "batch":
        from snow_b200 import scenes

        scs = scenes.batch_scenes(count=256)
        rate, steps, wall, kind, what = cpu_rate_batch(scs)
        line = {
            "impl": "reference", "metric": "particle-steps/s", "value": rate, "unit": "particle-steps/s",
            "n_gpus": args.gpus, "steps": steps, "warmup": 0, "ms_per_step": None,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": {"workload": "batch-256-scenes", "scenes": len(scs),
                                                      "particles": sum(x.n for x in scs)},
            "cpu_baseline": {"value": rate, "unit": "particle-steps/s", "cores": os.cpu_count(), "kind": kind,
                             "sample": what},
            "e2e": {"value": rate, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    sc = workload(args.workload, args.particles)
    rate, steps, wall, kind, what = cpu_rate(sc, max(1, args.steps))
    cores = os.cpu_count()
    line = {
        "impl": "reference", "metric": "particle-steps/s", "value": rate, "unit": "particle-steps/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": 1, "ms_per_step": 1e3 * wall / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": describe(sc),
        "cpu_baseline": {"value": rate, "unit": "particle-steps/s", "cores": cores, "kind": kind,
                         "sample": f"{steps} full-scene steps after setup() and 1 untimed step; {what}; "
                                   f"bounded to ~{REF_SAMPLE_S:.0f} s of CPU work"},
        "e2e": {"value": rate, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------- clocks
class Clocks:
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id: str):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", device_id, f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in out.strip().splitlines():
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def device_selector(torch, dev: int) -> str:
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return str(dev)


# -------------------------------------------------------------------- ours
def alg_bytes(n_p: int, nodes: int, real: int) -> dict:
    """Algorithmic DRAM bytes per launch of the two particle kernels.

    p2g reads x, v, m and the 6-entry force matrix (13 `real` values) per
        particle and writes the 7 accumulated channels of every grid node;
    g2p reads x, v, m, V_p0, F_E (17 `real`), F_P (9 doubles) and the particle id
        per particle and the 6 velocity channels per node, and writes the new
        state: x, v, m, V_p0, F_E, the next force matrix (23 `real`), F_P and the id,
        and the next step's sort key and position (8 B; in the steady state G2P
        emits them and the keys kernel reads nothing).
    """
    return {"p2g": n_p * 13 * real + nodes * 7 * real,
            "g2p": n_p * (17 * real + 72 + 4) + nodes * 6 * real + n_p * (23 * real + 72 + 4 + 8)}


def errors(a, b) -> dict:
    """Per-quantity max relative error of records a against b: ||a_i - b_i|| / max(||b_i||, 1e-6)."""
    out = {}
    for k, s in (("x", slice(0, 3)), ("v", slice(3, 6)), ("F_P", slice(8, 17)), ("F_E", slice(17, 26))):
        num = np.linalg.norm(a[:, s] - b[:, s], axis=1)
        den = np.maximum(np.linalg.norm(b[:, s], axis=1), 1e-6)
        out[k] = float(np.max(num / den))
    return out


def timed_steps(batch, steps, sp, torch) -> float:
    """Device milliseconds of `steps` graph-replayed steps on stream sp."""
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    batch.step(steps, stream=sp)
    e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def copy_bound(torch, host, n: int, rate: float) -> dict:
    """The host-link bound of one drop-in call: the same record bytes copied
    host -> device and back from the same page-locked buffer, with no step
    between (best of three, CUDA events), the share of the measured call time
    it takes, and the link rate of the two copies (bytes moved / their time)."""
    dev = torch.empty(host.shape, dtype=torch.float64, device="cuda")
    src = torch.from_numpy(host)
    best = float("inf")
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        dev.copy_(src, non_blocking=True)
        src.copy_(dev, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    call_ms = 1e3 * n / rate
    return {"copy_only_ms": best, "call_ms": call_ms, "copy_share_of_call": best / call_ms,
            "link_gbs": 2 * host.nbytes / (best * 1e-3) / 1e9}


def plain_fp64_rate(snow_b200, torch, sp, items, settle: int = 0) -> float:
    """Particle-steps/s of the plain FP64 path on the given scenes: each scene
    alone in its own one-scene batch (the drop-in step on resident state, with
    its captured step graph), one scene after another.  items: (scene, steps,
    timed steps); a scene's time is its timed steps' time scaled to `steps`;
    `settle` untimed steps first (as the batch it is compared with had)."""
    particle_steps, ms = 0.0, 0.0
    for sc, n_steps, k in items:
        b = snow_b200.Batch(snow_b200.SNOW_FP64)
        i = b.add(sc, stream=sp)
        b.setup(i, sc.dx, stream=sp)
        b.step(max(3, settle), stream=sp)
        ms += timed_steps(b, k, sp, torch) * n_steps / k
        particle_steps += sc.n * n_steps
        b.close()
    return particle_steps / (ms * 1e-3)


def serve_stream(snow_b200, sp, reqs, precision, streaming: bool = True) -> dict:
    """One served run.  Streaming: run() loops on a thread while this thread
    submits each request at its arrival time (a Poisson stream in real time,
    each request stamped on arrival), then closes the stream; otherwise every
    request is queued with its arrival time before run()."""
    import threading

    srv = snow_b200.Server(precision, budget_bytes=150 * 10**9, max_steps_per_tick=16)
    if not streaming:
        for sc, n, t in reqs:
            srv.submit(sc, n, t)
        srv.run(stream=sp)
    else:
        srv.set_streaming(True)
        failure = []

        def serve():
            try:
                srv.run(stream=sp)
            except Exception as e:  # re-raised below
                failure.append(e)

        th = threading.Thread(target=serve)
        t0 = time.perf_counter()
        th.start()
        for sc, n, t in reqs:
            wait = t - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            srv.submit(sc, n)
        srv.end_of_stream()
        th.join()
        if failure:
            raise failure[0]
    st = srv.stats()
    st.update(tick_summary(srv.ticks(), st["wall_s"]))
    srv.close()
    return st


def tick_summary(ticks, wall_s: float) -> dict:
    """Where a served run's time went, from its per-tick trace: the device's
    busy share of the wall time, the mean steps and device milliseconds per
    tick, and the mean device gap between two ticks (admission, retirement and
    the host's launch of the next tick)."""
    if not ticks:
        return {}
    busy = sum(t["device_end_s"] - t["device_start_s"] for t in ticks)
    gaps = [b["device_start_s"] - a["device_end_s"] for a, b in zip(ticks, ticks[1:])]
    big = [g for g in gaps if g > 1e-3]
    return {"device_busy_frac": busy / wall_s if wall_s > 0 else None,
            "mean_steps_per_tick": sum(t["steps"] for t in ticks) / len(ticks),
            "mean_tick_device_ms": 1e3 * busy / len(ticks),
            "mean_gap_ms": 1e3 * sum(gaps) / len(gaps) if gaps else 0.0,
            "median_gap_ms": 1e3 * statistics.median(gaps) if gaps else 0.0,
            "gaps_over_1ms": len(big), "gap_ms_in_those": 1e3 * sum(big)}


def measure_served(snow_b200, torch, sp, count: int, fp64_rate: float | None = None, grounded: bool = False,
                   runs: int = 3) -> dict:
    """The served form on `count` requests (2k..500k particles, 100..2000 steps,
    Poisson 200/s): every run's throughput, the slowest run's ratio against
    the plain FP64 path stepping the same requests one at a time, and the
    median run's latencies."""
    from snow_b200 import scenes

    reqs = scenes.served_requests(count=count, rate=200.0, grounded=grounded)
    allruns = [serve_stream(snow_b200, sp, reqs, snow_b200.SNOW_MIXED) for _ in range(runs)]
    order = sorted(allruns, key=lambda r: r["particle_steps_per_s"])
    med = order[len(order) // 2]
    plain_s = plain_fp64_rate(snow_b200, torch, sp, [(sc, n, min(n, 40)) for sc, n, _ in reqs],
                              settle=40 if grounded else 0)
    out = {"requests": len(reqs), "arrival_rate_per_s": 200.0, "budget_bytes": 150 * 10**9,
           "submission": "streaming: submitted at their arrival times while run() loops",
           "grounded": grounded, "precision": "mixed",
           "plain_fp64_one_request_at_a_time": plain_s,
           "plain_fp64_sample": "each request's scene alone, min(steps, 40) timed steps scaled to its requested steps",
           "runs_particle_steps_per_s": [r["particle_steps_per_s"] for r in allruns],
           "served_vs_plain_fp64_same_requests_min_run": order[0]["particle_steps_per_s"] / plain_s,
           "served_vs_plain_fp64_same_requests_median_run": med["particle_steps_per_s"] / plain_s,
           "p50_latency_s": med["p50_s"], "p99_latency_s": med["p99_s"], "mean_latency_s": med["mean_s"],
           "particle_steps_per_s": med["particle_steps_per_s"], "completed": med["completed"],
           "rejected": med["rejected"], "peak_concurrent_scenes": med["peak_scenes"], "ticks": med["ticks"],
           "reservations": med["reservations"], "wall_s": med["wall_s"],
           "ticks_summary": {k: med.get(k) for k in ("device_busy_frac", "mean_steps_per_tick",
                                                     "mean_tick_device_ms", "mean_gap_ms", "median_gap_ms",
                                                     "gaps_over_1ms", "gap_ms_in_those")},
           "host_phases_s": {"admit": med["admit_s"], "step": med["step_s"], "retire": med["retire_s"]}}
    if fp64_rate:
        out["served_vs_plain_fp64_headline"] = med["particle_steps_per_s"] / fp64_rate
    return out


def measure_forms(snow_b200, torch, sp, tori, fp64_rate, steps, served_count: int = 512) -> dict:
    """The mixed-precision, batched and served forms (single GPU).

    mixed     the headline scene in the mixed form: particle-steps/s, ratio to the
              plain FP64 path, error vs the FP64 path after 1 and 10 steps
    batched   256 independent scenes (log-uniform 1k..64k particles), one launch per
              stage: FP64 and autotuned mixed particle-steps/s, mixed error after 10 steps
    served    a Poisson stream of scene requests admitted by memory budget and
              stepped together: p50/p99 latency and aggregate particle-steps/s
    snowball  4M-particle sphere, mixed vs FP64 error at steps 1, 10 and 200
    """
    from snow_b200 import scenes

    forms = {}
    # -- mixed form of the headline scene
    mixed = snow_b200.Batch(snow_b200.SNOW_MIXED)
    mid = mixed.add(tori, stream=sp)
    mixed.setup(mid, tori.dx, stream=sp)
    mixed.step(5, stream=sp)
    ms = timed_steps(mixed, steps, sp, torch)
    rate = tori.n * steps / (ms * 1e-3)
    mixed.close()
    ref = snow_b200.Batch(snow_b200.SNOW_FP64)
    rid = ref.add(tori, stream=sp)
    ref.setup(rid, tori.dx, stream=sp)
    start = ref.download(rid)
    errs = {}
    for n in (1, 10):
        a = snow_b200.Batch(snow_b200.SNOW_FP64)
        b = snow_b200.Batch(snow_b200.SNOW_MIXED)
        ia, ib = a.add_scene(start, tori.params(), tori.planes), b.add_scene(start, tori.params(), tori.planes)
        a.step(n)
        b.step(n)
        errs[f"step{n}"] = errors(b.download(ib), a.download(ia))
        errs[f"step{n}_fp64_projections"] = b.fp64_projections
        a.close()
        b.close()
    ref.close()
    forms["mixed"] = {"workload": tori.name, "value": rate, "unit": "particle-steps/s",
                      "ms_per_step": ms / steps, "vs_plain_fp64": rate / fp64_rate,
                      "error_vs_fp64": errs}
    # -- colliding: the same measurements where the snow deforms
    forms["colliding"] = measure_colliding(snow_b200, torch, sp, steps)
    # -- input / output and the frame loop
    forms["io"] = measure_io(tori)
    # -- batched: 256 scenes, FP64 and mixed
    bscenes = scenes.batch_scenes(count=256)
    nb = sum(s.n for s in bscenes)
    brates = {}
    for name, prec in (("fp64", snow_b200.SNOW_FP64), ("mixed", snow_b200.SNOW_MIXED)):
        b = snow_b200.Batch(prec)
        ids = [b.add(s, stream=sp) for s in bscenes]
        for i, s in zip(ids, bscenes):
            b.setup(i, s.dx, stream=sp)
        b.step(3, stream=sp)
        chunk, _ = b.autotune(trial_steps=5, stream=sp)
        b.step(3, stream=sp)  # re-measured boxes and the step graph after the tuner's restore
        bsteps = max(20, steps // 4)
        ms_b = timed_steps(b, bsteps, sp, torch)
        brates[name] = {"value": nb * bsteps / (ms_b * 1e-3), "ms_per_step": ms_b / bsteps,
                        "work_item": chunk, "sort": b.sort_mode()}
        b.close()
    berr = {}
    a = snow_b200.Batch(snow_b200.SNOW_FP64)
    b = snow_b200.Batch(snow_b200.SNOW_MIXED)
    sample = bscenes[:16]
    pa = [a.add(s) for s in sample]
    pb = [b.add(s) for s in sample]
    for i, j, s in zip(pa, pb, sample):
        a.setup(i, s.dx)
        b.setup(j, s.dx)
    a.step(10)
    b.step(10)
    worst = {}
    for i, j in zip(pa, pb):
        e = errors(b.download(j), a.download(i))
        for k, v in e.items():
            worst[k] = max(worst.get(k, 0.0), v)
    a.close()
    b.close()
    bsteps = max(20, steps // 4)
    plain_b = plain_fp64_rate(snow_b200, torch, sp, [(sc, bsteps, bsteps) for sc in bscenes])
    forms["batched"] = {"scenes": len(bscenes), "particles": nb, "unit": "particle-steps/s",
                        "fp64": brates["fp64"], "mixed": brates["mixed"],
                        "plain_fp64_one_scene_at_a_time": plain_b,
                        "mixed_vs_plain_fp64_same_scenes": brates["mixed"]["value"] / plain_b,
                        "fp64_batched_vs_plain_fp64_same_scenes": brates["fp64"]["value"] / plain_b,
                        "mixed_vs_fp64": brates["mixed"]["value"] / brates["fp64"]["value"],
                        "mixed_vs_plain_fp64_headline": brates["mixed"]["value"] / fp64_rate,
                        "mixed_error_vs_fp64_step10_first16": worst,
                        "graph": "CUDA graph per step", "autotuned": "work-item size and particle ordering"}
    # -- served: a Poisson stream submitted while the server runs, mixed form
    forms["served"] = measure_served(snow_b200, torch, sp, count=served_count, fp64_rate=fp64_rate)
    # -- snowball: error of the mixed form at steps 1, 10, 200
    ball = scenes.snowball_scene()
    a = snow_b200.Batch(snow_b200.SNOW_FP64)
    ia = a.add(ball, stream=sp)
    a.setup(ia, ball.dx, stream=sp)
    start = a.download(ia)
    b = snow_b200.Batch(snow_b200.SNOW_MIXED)
    ib = b.add_scene(start, ball.params(), ball.planes)
    serr = {}
    done = 0
    for n in (1, 10, 200):
        a.step(n - done, stream=sp)
        b.step(n - done, stream=sp)
        done = n
        serr[f"step{n}"] = errors(b.download(ib), a.download(ia))
    # throughput: 50 steps after the 200, graphs captured, boxes settled
    a.step(3, stream=sp)
    b.step(3, stream=sp)
    t_fp64 = timed_steps(a, 50, sp, torch)
    t_mixed = timed_steps(b, 50, sp, torch)
    a.close()
    b.close()
    forms["snowball"] = {"workload": ball.name, "error_vs_fp64": serr,
                         "fp64_particle_steps_per_s": ball.n * 50 / (t_fp64 * 1e-3),
                         "mixed_particle_steps_per_s": ball.n * 50 / (t_mixed * 1e-3),
                         "throughput_window": "steps 204-253"}
    return forms


def plastic_fraction(rec) -> float:
    """Fraction of particles whose F_P differs from I (the clamp has acted on them)."""
    d = np.linalg.norm(rec[:, 8:17] - np.eye(3).reshape(-1), axis=1)
    return float((d > 1e-6).mean()) if len(d) else 0.0


def measure_colliding(snow_b200, torch, sp, steps, settle=40) -> dict:
    """The deforming regime: snow that strikes snow or the ground from its first
    steps, so the plastic clamp, the hardening and (in the mixed form) the
    double-precision fallback are all at work inside the timed window.

    tori      the headline tori placed in contact (gap 0, +-8 m/s): `settle` steps
              untimed, then `steps` timed, FP64 and mixed; the fallback fraction per
              step; the fraction of particles with F_P != I; the mixed error against
              the FP64 path 10 steps on from the settled FP64 state
    batched   the 256 scenes set on the ground moving down: batched FP64 and mixed
              against the plain FP64 path one scene at a time
    served    the request stream set on the ground: served mixed against the plain
              FP64 path one request at a time
    """
    from snow_b200 import scenes

    out = {}
    sc = scenes.tori_scene(gap=0.0)
    res, settled = {}, None
    for name, prec in (("fp64", snow_b200.SNOW_FP64), ("mixed", snow_b200.SNOW_MIXED)):
        b = snow_b200.Batch(prec)
        i = b.add(sc, stream=sp)
        b.setup(i, sc.dx, stream=sp)
        b.step(settle, stream=sp)
        if name == "fp64":
            settled = b.download(i)
        ms = timed_steps(b, steps, sp, torch)
        fb = []
        for _ in range(5):
            b.step(1, stream=sp)
            fb.append(b.fp64_projections)
        res[name] = {"value": sc.n * steps / (ms * 1e-3), "ms_per_step": ms / steps,
                     "plastic_fraction_after": plastic_fraction(b.download(i))}
        if name == "mixed":
            res[name]["fp64_fallback_per_step"] = float(np.mean(fb)) / sc.n
        b.close()
    a, b = snow_b200.Batch(snow_b200.SNOW_FP64), snow_b200.Batch(snow_b200.SNOW_MIXED)
    ia = a.add_scene(settled, sc.params(), sc.planes)
    ib = b.add_scene(settled, sc.params(), sc.planes)
    fb = 0
    for _ in range(10):
        a.step(1)
        b.step(1)
        fb += b.fp64_projections
    err = errors(b.download(ib), a.download(ia))
    a.close()
    b.close()
    out["tori"] = {"workload": sc.name, "settle_steps": settle, "timed_steps": steps, "fp64": res["fp64"],
                   "mixed": res["mixed"], "mixed_vs_fp64": res["mixed"]["value"] / res["fp64"]["value"],
                   "plastic_fraction_at_start": plastic_fraction(settled),
                   "mixed_error_vs_fp64_10_steps_from_settled": err,
                   "mixed_fp64_fallbacks_in_those_10_steps": fb}
    # -- batched scenes on the ground
    bscenes = scenes.batch_scenes(count=256, grounded=True)
    nb = sum(x.n for x in bscenes)
    brates = {}
    bsteps = max(20, steps // 4)
    for name, prec in (("fp64", snow_b200.SNOW_FP64), ("mixed", snow_b200.SNOW_MIXED)):
        b = snow_b200.Batch(prec)
        ids = [b.add(x, stream=sp) for x in bscenes]
        for i, x in zip(ids, bscenes):
            b.setup(i, x.dx, stream=sp)
        b.step(settle, stream=sp)
        chunk, _ = b.autotune(trial_steps=5, stream=sp)
        b.step(3, stream=sp)
        ms_b = timed_steps(b, bsteps, sp, torch)
        pf = float(np.mean([plastic_fraction(b.download(i)) for i in ids]))
        brates[name] = {"value": nb * bsteps / (ms_b * 1e-3), "ms_per_step": ms_b / bsteps, "work_item": chunk,
                        "mean_plastic_fraction_after": pf}
        b.close()
    plain_b = plain_fp64_rate(snow_b200, torch, sp, [(x, bsteps, bsteps) for x in bscenes], settle=settle)
    out["batched"] = {"scenes": len(bscenes), "particles": nb, "settle_steps": settle, "fp64": brates["fp64"],
                      "mixed": brates["mixed"], "plain_fp64_one_scene_at_a_time": plain_b,
                      "mixed_vs_plain_fp64_same_scenes": brates["mixed"]["value"] / plain_b,
                      "fp64_batched_vs_plain_fp64_same_scenes": brates["fp64"]["value"] / plain_b}
    # -- served stream on the ground
    out["served"] = measure_served(snow_b200, torch, sp, count=96, grounded=True, runs=2)
    return out


def write_scene_csv(sc, d: str) -> tuple[str, str]:
    """The scene as the reference's input files (one group per distinct
    velocity and mass)."""
    rec = sc.particles
    keys, inv = np.unique(np.concatenate([rec[:, 3:7]], axis=1), axis=0, return_inverse=True)
    g, p = os.path.join(d, "groups.csv"), os.path.join(d, "particles.csv")
    with open(g, "w") as f:
        f.write("group_id,vx,vy,vz,mass\n")
        for i, k in enumerate(keys):
            f.write(f"{i},{float(k[0])!r},{float(k[1])!r},{float(k[2])!r},{float(k[3])!r}\n")
    np.savetxt(p, np.column_stack([inv.reshape(-1), rec[:, 0:3]]), fmt=["%d", "%.17g", "%.17g", "%.17g"],
               delimiter=",", header="group_id,x,y,z", comments="")
    return g, p


def measure_io(sc) -> dict:
    """The drop-in's input and output against the reference's on the headline
    scene: import of its groups.csv/particles.csv, export of one frame, and the
    reference's frame loop (import, setup, frames of steps, a frame written
    after each) run by the snow_frames app with the state resident on the GPU,
    without export, with the reference's synchronous export and with the
    background export that overlaps the next frame's steps."""
    import ctypes
    import tempfile

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import REF_SO

    dp = ctypes.POINTER(ctypes.c_double)
    L = ctypes.CDLL(os.path.join(PKG, "libsnow.so"))
    L.snow_io_import.argtypes = [ctypes.c_char_p, ctypes.c_char_p, dp, ctypes.c_int64]
    L.snow_io_import.restype = ctypes.c_int64
    L.snow_io_export.argtypes = [dp, ctypes.c_int64, ctypes.c_int]
    R = ctypes.CDLL(REF_SO) if os.path.exists(REF_SO) else None
    if R is not None:
        R.ref_import.argtypes = [ctypes.c_char_p, ctypes.c_char_p, dp, ctypes.c_int64]
        R.ref_import.restype = ctypes.c_int64
        R.ref_export.argtypes = [dp, ctypes.c_int64, ctypes.c_int]
    out = {"workload": sc.name, "particles": sc.n}
    rec = np.ascontiguousarray(sc.particles)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as d:
        g, p = write_scene_csv(sc, d)
        out["particles_csv_bytes"] = os.path.getsize(p)

        def best(fn, reps=2):
            t = []
            for _ in range(reps):
                t0 = time.perf_counter()
                fn()
                t.append(time.perf_counter() - t0)
            return 1e3 * min(t)

        n_ours = L.snow_io_import(g.encode(), p.encode(), None, 0)
        if n_ours != sc.n:
            raise RuntimeError(f"snow_io_import read {n_ours} particles, expected {sc.n}")
        # both importers fill the caller's records (the reference's through its vector)
        dst = np.zeros((sc.n, 26))
        dptr = dst.ctypes.data_as(dp)
        out["import_ms"] = {"ours": best(lambda: L.snow_io_import(g.encode(), p.encode(), dptr, sc.n))}
        os.makedirs(os.path.join(d, "output"), exist_ok=True)
        os.chdir(d)
        try:
            out["export_ms"] = {"ours": best(lambda: L.snow_io_export(rec.ctypes.data_as(dp), sc.n, 1))}
            if R is not None:
                out["import_ms"]["reference"] = best(lambda: R.ref_import(g.encode(), p.encode(), dptr, sc.n))
                out["export_ms"]["reference"] = best(lambda: R.ref_export(rec.ctypes.data_as(dp), sc.n, 2))
        finally:
            os.chdir(cwd)
        for k in ("import_ms", "export_ms"):
            if "reference" in out[k]:
                out[k]["reference_over_ours"] = out[k]["reference"] / out[k]["ours"]
        m = sc.material
        args = [os.path.join(PKG, "snow_frames"), g, p, "--frames", "6", "--substeps", "25", "--dx", str(sc.dx),
                "--dt", str(sc.dt), "--E", str(m.E), "--nu", str(m.nu), "--xi", str(m.xi),
                "--theta-c", str(m.theta_c), "--theta-s", str(m.theta_s), "--alpha", str(m.alpha),
                "--gravity", str(m.gravity[1]), "--plane-y", "0.05", "--friction", "0.2"]
        loops = {}
        for mode in ("none", "async", "sync"):
            r = subprocess.run(args + ["--export", mode], cwd=d, capture_output=True, text=True, timeout=600)
            if r.returncode != 0:
                loops[mode] = {"error": (r.stderr or r.stdout)[-300:]}
                continue
            j = json.loads(r.stdout.strip().splitlines()[-1])
            loops[mode] = {k: j[k] for k in ("loop_ms", "steps_done_ms", "export_wait_ms", "particle_steps_per_s",
                                             "import_ms", "setup_ms")}
        out["frame_loop"] = {"frames": 6, "substeps": 25, "resident": True, "modes": loops}
        try:
            base, a, s = (loops[k]["loop_ms"] for k in ("none", "async", "sync"))
            out["frame_loop"]["export_cost_ms_per_frame"] = {"sync": (s - base) / 6, "async": (a - base) / 6}
        except (KeyError, TypeError):
            pass
    return out


def measured_peak() -> tuple[float, str]:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(workload: str, precision: str, kernel: str):
    """Per-launch DRAM bytes (read + write) of `kernel` from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)
        return t.get(f"{workload}/{precision}/{kernel}")
    except (OSError, ValueError):
        return None


def profile_flops(workload: str, precision: str, kernel: str):
    """Executed floating-point operations per particle of `kernel` ({"fp64": F, "fp32": F})
    from the committed ncu instruction counts (profiles/flops.json): 2 per FMA, 1 per add
    or multiply, twice that for the packed two-wide float forms."""
    try:
        with open(os.path.join(ROOT, "profiles", "flops.json")) as f:
            t = json.load(f)
        return t.get(f"{workload}/{precision}/{kernel}")
    except (OSError, ValueError):
        return None


def measure_peaks(snow_b200) -> dict:
    """FMA throughput of this GPU measured now (TFLOP/s; snow_gpu_measure_fma_peak)."""
    return {name: snow_b200.measure_fma_peak(kind) / 1e12
            for name, kind in (("fp64_tflops", snow_b200.SNOW_PEAK_FP64),
                               ("fp32_tflops", snow_b200.SNOW_PEAK_FP32),
                               ("fp32x2_tflops", snow_b200.SNOW_PEAK_FP32X2))}


def kernel_roofline(kernel: str, ms: float, alg_bytes: float, n_particles: int, workload: str,
                    precision: str, peaks: dict) -> dict:
    """One kernel against its roofs: HBM (algorithmic bytes / launch time against the
    measured copy bandwidth) and the FMA pipes (executed FLOPs / launch time against the
    measured FMA peaks).  `bound` is the roof with the largest fraction."""
    hbm_peak, hbm_src = measured_peak()
    gbs = alg_bytes / (ms * 1e-3) / 1e9
    roofs = {"hbm": {"achieved": gbs, "peak": hbm_peak, "unit": "GB/s", "frac": gbs / hbm_peak,
                     "peak_source": hbm_src}}
    fl = profile_flops(workload, precision, kernel) or {}
    for pipe, peak in (("fp64", peaks.get("fp64_tflops")),
                       ("fp32", max(peaks.get("fp32_tflops") or 0, peaks.get("fp32x2_tflops") or 0))):
        per = fl.get(pipe)
        if per and peak:
            tf = per * n_particles / (ms * 1e-3) / 1e12
            roofs[pipe] = {"achieved": tf, "peak": peak, "unit": "TFLOP/s", "frac": tf / peak,
                           "peak_source": "measured (snow_gpu_measure_fma_peak)",
                           "flops_per_launch": per * n_particles,
                           "pipe_active_pct_ncu": fl.get(f"{'fp64' if pipe == 'fp64' else 'fma'}_pipe_active_pct")}
    bound = max(roofs, key=lambda k: roofs[k]["frac"])
    return {"kernel": kernel, "launch_ms": ms, "alg_bytes_per_launch": alg_bytes, "bound": bound,
            "frac": roofs[bound]["frac"], "roofs": roofs,
            "traffic": profile_traffic(workload, precision, kernel)}


def roofline_line(per: dict, ab: dict, n_particles: int, workload: str, precision: str, peaks: dict) -> dict:
    """The bench line's roofline object: the dominant (longest) particle kernel's
    binding roof, with both particle kernels' roofs beside it."""
    ks = {"p2g": kernel_roofline("p2g", per["p2g"], ab["p2g"], n_particles, workload, precision, peaks),
          "g2p": kernel_roofline("g2p", per["stress_update"], ab["g2p"], n_particles, workload, precision,
                                 peaks)}
    dom = max(ks, key=lambda k: ks[k]["launch_ms"])
    d = ks[dom]
    r = d["roofs"][d["bound"]]
    return {"bound": d["bound"], "kernel": dom, "achieved": r["achieved"], "peak": r["peak"], "unit": r["unit"],
            "frac": r["frac"], "peak_source": r["peak_source"], "traffic": d["traffic"],
            "alg_bytes_per_launch": d["alg_bytes_per_launch"], "launch_ms": d["launch_ms"],
            "hbm_frac": d["roofs"]["hbm"]["frac"],
            "fp64_pipe_frac": d["roofs"].get("fp64", {}).get("frac"),
            "fp32_pipe_frac": d["roofs"].get("fp32", {}).get("frac"),
            "kernels": ks, "peaks": peaks}


def run_ours(args, ws, rank, local):
    import torch

    torch.cuda.set_device(local)
    import snow_b200

    snow_b200.init(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    prec = snow_b200.SNOW_FP64 if args.precision == "fp64" else snow_b200.SNOW_MIXED
    sc = workload(args.workload, args.particles)
    stream = torch.cuda.Stream()  # our kernels and the timing events share this stream
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream

    batch = snow_b200.Batch(prec)
    sid = batch.add(sc, stream=sp)
    batch.setup(sid, sc.dx, stream=sp)
    batch.step(max(3, args.warmup), stream=sp)
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    clocks = Clocks(device_selector(torch, local))
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.step(args.steps, stream=sp)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    status, blocks, cap = batch.status()
    launches = batch.graph_kernels() * args.steps  # kernel nodes of the replayed step graph

    # per-kernel times over K eagerly launched steps (events around each kernel)
    kt = batch.step(args.steps, timings=True, stream=sp)
    per = {k: v / args.steps for k, v in kt.items() if v > 0}
    real = 8 if args.precision == "fp64" else 4
    ab = alg_bytes(sc.n, blocks * 64, real)
    peaks = measure_peaks(snow_b200)
    roof = roofline_line(per, ab, sc.n, args.workload, args.precision, peaks)

    # end to end through the drop-in entry point on pinned host records
    e2e = None
    if not args.no_e2e:
        host = torch.empty((sc.n, 26), dtype=torch.float64, pin_memory=True).numpy()
        host[:] = batch.download(sid)
        ke = max(3, min(args.steps // 10, 40))
        snow_b200.step(host, sc.params(), sc.planes, 1)  # warm the one-scene context
        snow_b200.step(host, sc.params(), sc.planes, 1)
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for _ in range(ke):
            snow_b200.step(host, sc.params(), sc.planes, 1)
        dt_e = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([dt_e], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt_e = float(t.item())
        e2e = {"value": ws * sc.n * ke / dt_e, "unit": "particle-steps/s",
               "h2d_bytes_per_step": sc.n * 208, "d2h_bytes_per_step": sc.n * 208,
               "steps": ke, "api": "snow_gpu_step (upload, step, download per call)"}
        e2e.update(copy_bound(torch, host, sc.n, e2e["value"] / ws))

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        rate, steps, wall, kind, what = cpu_rate(sc, 50)
        cpu = {"value": rate, "unit": "particle-steps/s", "cores": os.cpu_count(), "kind": kind,
               "sample": f"{steps} full-scene steps ({wall:.1f} s) after setup(); {what}"}

    value = ws * sc.n * args.steps / (ms * 1e-3)
    forms = None
    if ws == 1 and not args.no_forms and args.workload == "tori" and args.precision == "fp64" and not args.particles:
        forms = measure_forms(snow_b200, torch, sp, sc, sc.n * args.steps / (ms * 1e-3), args.steps,
                              served_count=args.requests)
    line = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": ws,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic: seeded jittered-lattice scene (no dataset in the reference)",
        "config": dict(describe(sc), precision=args.precision,
                       parallelism=f"replicas x{ws}" if ws > 1 else "single GPU",
                       l2="particle state > 126 MB L2 (no flush needed)" if sc.n * 416 > 126e6
                       else "state fits L2; steps read the previous step's output",
                       graph="CUDA graph per step"),
        "roofline": roof,
        "stages_ms_per_step": per,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clk,
        "grid_blocks": {"used": blocks, "capacity": cap},
        "status": status,
        "forms": forms,
    }
    batch.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_batch(args, ws, rank, local):
    """The 256 independent scenes, split across ranks by work (snow_b200.shard):
    one batch per rank, one launch per stage, CUDA graph per step, autotuned
    work-item size; value = all scenes' particle-steps / max-over-ranks time."""
    import torch

    torch.cuda.set_device(local)
    import snow_b200
    from snow_b200 import scenes, shard

    snow_b200.init(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    prec = snow_b200.SNOW_FP64 if args.precision == "fp64" else snow_b200.SNOW_MIXED
    allsc = scenes.batch_scenes(count=256)
    total = sum(s.n for s in allsc)
    mine = [allsc[i] for i in shard.shard([s.n for s in allsc], ws, rank)]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    batch = snow_b200.Batch(prec)
    ids = [batch.add(s, stream=sp) for s in mine]
    for i, s in zip(ids, mine):
        batch.setup(i, s.dx, stream=sp)
    chunk, _ = batch.autotune(trial_steps=5, stream=sp)
    batch.step(max(3, args.warmup), stream=sp)
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    clocks = Clocks(device_selector(torch, local))
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.step(args.steps, stream=sp)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    clk = clocks.stop()
    status, blocks, cap = batch.status()
    launches = batch.graph_kernels() * args.steps
    kt = batch.step(args.steps, timings=True, stream=sp)
    per = {k: v / args.steps for k, v in kt.items() if v > 0}
    real = 8 if args.precision == "fp64" else 4
    nmine = sum(s.n for s in mine)
    ab = alg_bytes(nmine, blocks * 64, real)
    roof = roofline_line(per, ab, nmine, "batch", args.precision, measure_peaks(snow_b200))

    e2e = None
    if not args.no_e2e:
        # every step: this rank's scenes uploaded from pinned host records, one
        # batched step, every scene downloaded
        hosts = []
        for i, s in zip(ids, mine):
            h = torch.empty((s.n, 26), dtype=torch.float64, pin_memory=True).numpy()
            batch.download(i, h, stream=sp)
            hosts.append(h)
        ke = max(3, min(args.steps // 10, 20))
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for _ in range(ke):
            for i, h in zip(ids, hosts):
                batch.upload(i, h, stream=sp)
            batch.step(1, stream=sp)
            for i, h in zip(ids, hosts):
                batch.download(i, h, stream=sp)
        dt_e = max_over_ranks(time.perf_counter() - t0)
        nb = sum(s.n for s in mine)
        e2e = {"value": total * ke / dt_e, "unit": "particle-steps/s", "h2d_bytes_per_step": nb * 208,
               "d2h_bytes_per_step": nb * 208, "steps": ke,
               "api": "snow_gpu_batch_upload / _step / _download per step (this rank's bytes)"}
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        rate, steps_each, wall, kind, what = cpu_rate_batch(allsc)
        cpu = {"value": rate, "unit": "particle-steps/s", "cores": os.cpu_count(), "kind": kind, "sample": what}
    line = {
        "metric": "particle-steps/s", "value": total * args.steps / (ms * 1e-3), "unit": "particle-steps/s",
        "n_gpus": ws, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic: 256 seeded box/sphere scenes, log-uniform 1k..64k particles",
        "config": {"workload": "batch-256-scenes", "scenes": len(allsc), "particles": total,
                   "precision": args.precision, "parallelism": f"scene shards x{ws}" if ws > 1 else "single GPU",
                   "rank0_scenes": len(mine), "work_item": chunk, "sort": batch.sort_mode(),
                   "l2": "particle state > 126 MB L2 (no flush needed)", "graph": "CUDA graph per step"},
        "roofline": roof,
        "stages_ms_per_step": per, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk, "grid_blocks": {"used": blocks, "capacity": cap}, "status": status,
    }
    batch.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_served(args, ws, rank, local):
    """The served stream alone (--workload served): --requests requests (2k..500k
    particles, 100..2000 steps, Poisson 200/s) submitted at their arrival times
    while the server runs, mixed form.  With N ranks every rank serves its share
    of the stream (snow_b200.shard by particles x steps) on its own GPU; value =
    all requests' particle-steps / the slowest rank's wall time."""
    import torch

    torch.cuda.set_device(local)
    import snow_b200
    from snow_b200 import scenes, shard

    snow_b200.init(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    reqs = scenes.served_requests(count=args.requests, rate=200.0)
    mine = [reqs[i] for i in shard.shard([sc.n * n for sc, n, _ in reqs], ws, rank)]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    serve_stream(snow_b200, sp, mine[: min(4, len(mine))], snow_b200.SNOW_MIXED)  # warm-up
    clocks = Clocks(device_selector(torch, local))
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    st = serve_stream(snow_b200, sp, mine, snow_b200.SNOW_MIXED)
    torch.cuda.synchronize()
    wall = st["wall_s"]
    if dist is not None:
        t = torch.tensor([wall], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        wall = float(t.item())
    clk = clocks.stop()
    total = sum(sc.n * n for sc, n, _ in reqs)
    line = {"metric": "particle-steps/s", "value": total / wall, "unit": "particle-steps/s", "n_gpus": ws,
            "steps": None, "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic: seeded Poisson stream of scene requests",
            "config": {"workload": f"served-{len(reqs)}-requests", "precision": "mixed",
                       "parallelism": f"request shards x{ws}" if ws > 1 else "single GPU",
                       "submission": "streaming"},
            "rank0": {k: st.get(k) for k in ("p50_s", "p99_s", "mean_s", "completed", "ticks", "peak_scenes",
                                              "reservations", "particle_steps_per_s", "device_busy_frac",
                                              "mean_steps_per_tick", "mean_tick_device_ms", "mean_gap_ms",
                                              "median_gap_ms", "gaps_over_1ms", "gap_ms_in_those")},
            "clocks": clk}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, ws, rank)
    elif args.workload == "batch":
        run_batch(args, ws, rank, local)
    elif args.workload == "served":
        run_served(args, ws, rank, local)
    else:
        run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
