"""Continuous-batching server and the work-item autotuner on the GPU.

The server admits requests as they arrive while memory and slots allow and
advances all admitted scenes together; each scene's result must be the one it
gets alone (FP64: 1e-12 relative, only atomic order differs; mixed: 1e-5).
The autotuner must leave the simulation state as it found it.
"""
import numpy as np
import pytest

from oracle_lib import errors

pytestmark = pytest.mark.gpu


def _requests(n=6, seed=21):
    from snow_b200 import scenes

    reqs = scenes.served_requests(count=n, rate=2000.0, lo=300, hi=4000, steps_lo=5, steps_hi=37, seed=seed)
    return reqs


def _alone(snow, prec, sc, steps):
    b = snow.Batch(prec)
    sid = b.add(sc)
    b.setup(sid, sc.dx)
    b.step(steps)
    out = b.download(sid)
    b.close()
    return out


@pytest.mark.parametrize("prec,tol,item", [(0, 1e-12, 0), (1, 1e-5, 0), (0, 1e-12, 1024), (1, 1e-5, 64)])
def test_served_results_match_alone(snow, prec, tol, item):
    reqs = _requests()
    srv = snow.Server(prec, max_steps_per_tick=8, work_item=item)
    ids = [srv.submit(sc, steps, t) for sc, steps, t in reqs]
    srv.run()
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["rejected"] == 0
    assert st["particle_steps"] == sum(sc.n * steps for sc, steps, _ in reqs)
    assert 0 < st["p50_s"] <= st["p99_s"]
    assert st["peak_scenes"] >= 2, "requests should overlap on the device"
    for rid, (sc, steps, _) in zip(ids, reqs):
        got, lat = srv.result(rid)
        assert lat > 0
        e = errors(got, _alone(snow, prec, sc, steps))
        assert max(e.values()) < tol, (sc.name, e)
    # the tick trace accounts for every particle-step, in order on both clocks
    ticks = srv.ticks()
    assert len(ticks) == st["ticks"]
    assert sum(t["steps"] * t["particles"] for t in ticks) == st["particle_steps"]
    assert sum(t["admitted"] for t in ticks) == len(reqs)  # each joined before one tick
    assert sum(t["retired"] for t in ticks) == len(reqs)   # and finished with one
    for a, b in zip(ticks, ticks[1:]):
        assert a["device_end_s"] <= b["device_start_s"]
        assert a["host_start_s"] <= b["host_start_s"] and a["host_end_s"] <= b["host_end_s"]
    # each tick is queued behind the one in flight before the host waits for that one
    assert any(b["host_start_s"] < a["host_end_s"] for a, b in zip(ticks, ticks[1:]))
    assert all(0 <= t["device_start_s"] <= t["device_end_s"] for t in ticks)
    assert all(1 <= t["steps"] <= 8 and t["scenes"] >= 1 for t in ticks)
    srv.close()


def test_budget_defers_and_rejects(snow):
    from snow_b200 import scenes

    reqs = _requests(4, seed=5)
    small = max(r[0].n for r in reqs)
    # room for about two of these scenes at a time; one request far too large
    srv = snow.Server(0, budget_bytes=int(2.5 * 900 * small + 2 * 70000), max_scenes=2, max_steps_per_tick=4)
    ids = [srv.submit(sc, steps, t) for sc, steps, t in reqs]
    big = scenes.cube_scene(40)
    big_id = srv.submit(big, 3, 0.0)
    srv.run()
    st = srv.stats()
    assert st["rejected"] == 1 and st["completed"] == len(reqs)
    assert st["peak_scenes"] <= 2
    with pytest.raises(snow.SnowError):
        srv.result(big_id)
    for rid, (sc, steps, _) in zip(ids, reqs):
        got, _ = srv.result(rid)
        assert max(errors(got, _alone(snow, 0, sc, steps)).values()) < 1e-12
    srv.close()


def test_autotune_restores_state(snow):
    from snow_b200 import scenes

    scs = scenes.batch_scenes(count=4, lo=500, hi=5000, seed=8)
    recs = [snow.setup(s.particles.copy(), s.dx) for s in scs]
    ref = snow.Batch(snow.SNOW_FP64)
    tuned = snow.Batch(snow.SNOW_FP64)
    rid = [ref.add_scene(r, s.params(), s.planes) for r, s in zip(recs, scs)]
    tid = [tuned.add_scene(r, s.params(), s.planes) for r, s in zip(recs, scs)]
    ref.step(3)
    tuned.step(3)
    chunk, ms = tuned.autotune(trial_steps=3)
    assert chunk in (64, 128, 256, 512, 1024) and ms > 0
    ref.step(4)
    tuned.step(4)
    for a, b in zip(rid, tid):
        assert max(errors(tuned.download(b), ref.download(a)).values()) < 1e-12


def test_submit_rejects_nonfinite(snow):
    sc = _requests(1, seed=3)[0][0]
    sc.particles[7, 1] = float("nan")
    srv = snow.Server(0)
    with pytest.raises(snow.SnowError) as e:
        srv.submit(sc, 3, 0.0)
    assert e.value.code == -4
    srv.close()


def test_work_item_size_checked(snow):
    for bad in (100, 16, 2048, -1):
        with pytest.raises(snow.SnowError):
            snow.Server(0, work_item=bad)


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 1e-5)])
def test_requests_submitted_while_running(snow, prec, tol):
    """Streaming: run() loops on one thread while requests are submitted on
    another, each stamped with its arrival on the server clock; later requests
    are larger than anything queued when run() started, so the server grows its
    reservation between ticks.  Every result equals the scene alone."""
    import threading
    import time

    from snow_b200 import scenes

    small = _requests(n=3, seed=31)
    large = scenes.served_requests(count=5, rate=2000.0, lo=6000, hi=12000, steps_lo=20, steps_hi=40, seed=32)
    srv = snow.Server(prec, max_steps_per_tick=8)
    srv.set_streaming(True)
    ids = [(srv.submit(sc, steps, 0.0), sc, steps) for sc, steps, _ in small]
    failure = []

    def serve():
        try:
            srv.run()
        except Exception as e:  # reported by the main thread
            failure.append(e)

    th = threading.Thread(target=serve)
    th.start()
    # the first requests complete while the stream is still open
    deadline = time.time() + 60
    while not srv.done(ids[0][0]) and time.time() < deadline and not failure:
        time.sleep(0.005)
    assert srv.done(ids[0][0]), failure
    for sc, steps, _ in large:
        ids.append((srv.submit(sc, steps), sc, steps))
        time.sleep(0.003)
    srv.end_of_stream()
    th.join(timeout=120)
    assert not th.is_alive() and not failure, failure
    with pytest.raises(snow.SnowError):
        srv.submit(small[0][0], 5)  # closed to new requests
    st = srv.stats()
    assert st["completed"] == len(ids) and st["rejected"] == 0
    assert st["reservations"] >= 2, "later, larger requests should grow the reservation"
    for rid, sc, steps in ids:
        got, lat = srv.result(rid)
        assert lat > 0
        e = errors(got, _alone(snow, prec, sc, steps))
        assert max(e.values()) < tol, (sc.name, e)
    srv.close()


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 1e-5)])
def test_reservation_grows_under_a_live_scene(snow, prec, tol):
    """A long-running scene is live (its steps write the next step's sort keys
    as they go) when a much larger request arrives: the server grows the live
    batch's particle and sort buffers between two ticks, and the next tick must
    sort afresh instead of reading keys from the replaced buffers.  Both results
    equal their scenes alone."""
    import threading
    import time

    from snow_b200 import scenes

    (long_sc, _, _), = scenes.served_requests(count=1, rate=2000.0, lo=1500, hi=2500, seed=41)
    (big_sc, _, _), = scenes.served_requests(count=1, rate=2000.0, lo=40000, hi=60000, seed=42)
    srv = snow.Server(prec, max_steps_per_tick=4)
    srv.set_streaming(True)
    ids = [(srv.submit(long_sc, 400, 0.0), long_sc, 400)]
    failure = []

    def serve():
        try:
            srv.run()
        except Exception as e:  # reported by the main thread
            failure.append(e)

    th = threading.Thread(target=serve)
    th.start()
    time.sleep(0.02)
    ids.append((srv.submit(big_sc, 20), big_sc, 20))
    srv.end_of_stream()
    th.join(timeout=120)
    assert not th.is_alive() and not failure, failure
    assert srv.stats()["reservations"] >= 2
    for rid, sc, steps in ids:
        got, _ = srv.result(rid)
        e = errors(got, _alone(snow, prec, sc, steps))
        assert max(e.values()) < tol, (sc.name, e)
