"""Mixed-precision form and multi-scene batches on the GPU.

Mixed form (float bulk, double F_P / hardening / near-critical projections)
against the FP64 oracle: relative position error <= 1e-4 after 10 steps (the
bound the mixed form is held to), and stated bounds for v, F_E, F_P.
Batches: every scene advanced inside a batch of unequal scenes matches the
same scene advanced alone -- to 1e-12 relative in FP64 (only the order of the
grid's floating-point atomics differs) and to 1e-5 in the mixed form.
"""
import numpy as np
import pytest

from oracle_lib import errors

pytestmark = pytest.mark.gpu

MIXED_TOL = {"x": 1e-4, "v": 5e-3, "F_E": 1e-4, "F_P": 1e-4}


def _alone(snow, prec, rec, params, planes, steps):
    b = snow.Batch(prec)
    sid = b.add_scene(rec, params, planes)
    b.step(steps)
    out = b.download(sid)
    b.close()
    return out


@pytest.mark.parametrize("steps", [1, 10])
def test_mixed_cube_against_fp64_oracle(snow, oracle, steps):
    from snow_b200 import scenes

    sc = scenes.cube_scene(32)
    rec = oracle.setup(sc.particles, sc.dx)
    want, _ = oracle.step(rec, sc.params(), sc.plane_array(), steps)
    b = snow.Batch(snow.SNOW_MIXED)
    sid = b.add_scene(rec, sc.params(), sc.planes)
    b.step(steps)
    got = b.download(sid)
    e = errors(got, want)
    for k, tol in MIXED_TOL.items():
        assert e[k] < tol, (k, e)
    # The cube is in free fall, far from the ground and from the clamp bounds:
    # no projection is clamped or near-critical, so nothing goes to the
    # double-precision fallback and F_P stays I -- exactly on the GPU, which
    # leaves an unclamped F_P untouched, and to rounding (1e-15) in the
    # reference, which always recomputes F_P = F_E^-1 F* F_P.  (The
    # touching-tori test in test_parity_full.py covers the regime where both
    # happen.)
    assert b.fp64_projections == 0
    eye = np.tile(np.eye(3).reshape(-1), (want.shape[0], 1))
    assert np.array_equal(got[:, 8:17], eye)
    assert np.abs(want[:, 8:17] - eye).max() < 1e-14


def test_mixed_tori_in_contact(snow, oracle):
    """Colliding tori: plastic flow, clamped singular values, FP64 fallbacks."""
    from snow_b200 import scenes

    sc = scenes.tori_scene(n_per_torus=5000)
    sc.particles[:, 0] += np.where(sc.particles[:, 3] > 0, 0.12, -0.12)
    rec = oracle.setup(sc.particles, sc.dx)
    want, _ = oracle.step(rec, sc.params(), sc.plane_array(), 10)
    b = snow.Batch(snow.SNOW_MIXED)
    sid = b.add_scene(rec, sc.params(), sc.planes)
    b.step(10)
    e = errors(b.download(sid), want)
    for k, tol in MIXED_TOL.items():
        assert e[k] < tol, (k, e)


def _mixed_batch_scenes():
    from snow_b200 import scenes

    out = scenes.batch_scenes(count=5, lo=300, hi=6000, seed=11, dt=5e-5)
    # different material / colliders per scene
    out[1].planes = [scenes.GROUND, ((0.62, 0, 0), (-1, 0, 0), 0.3)]
    out[2].dx = 0.015
    return out


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 1e-5)])
def test_batch_matches_each_scene_alone(snow, prec, tol):
    scs = _mixed_batch_scenes()
    recs = [snow.setup(s.particles.copy(), s.dx) for s in scs]
    b = snow.Batch(prec)
    ids = [b.add_scene(r, s.params(), s.planes) for r, s in zip(recs, scs)]
    b.step(8)
    for sid, r, s in zip(ids, recs, scs):
        alone = _alone(snow, prec, r, s.params(), s.planes, 8)
        e = errors(b.download(sid), alone)
        assert max(e.values()) < tol, (s.name, e)


def test_batch_scene_removed_and_added_mid_run(snow):
    scs = _mixed_batch_scenes()
    recs = [snow.setup(s.particles.copy(), s.dx) for s in scs]
    b = snow.Batch(snow.SNOW_FP64)
    ids = [b.add_scene(r, s.params(), s.planes) for r, s in zip(recs[:3], scs[:3])]
    b.step(4)
    b.remove_scene(ids[1])
    new_id = b.add_scene(recs[3], scs[3].params(), scs[3].planes)
    b.step(4)
    for sid, r, s, n in ((ids[0], recs[0], scs[0], 8), (ids[2], recs[2], scs[2], 8),
                         (new_id, recs[3], scs[3], 4)):
        alone = _alone(snow, 0, r, s.params(), s.planes, n)
        e = errors(b.download(sid), alone)
        assert max(e.values()) < 1e-12, (s.name, e)
    assert b.particles == sum(recs[i].shape[0] for i in (0, 2, 3))


def test_setup_in_batch_leaves_other_scenes_alone(snow):
    scs = _mixed_batch_scenes()[:2]
    b = snow.Batch(snow.SNOW_FP64)
    ids = [b.add_scene(s.particles, s.params(), s.planes) for s in scs]
    b.setup(ids[0], scs[0].dx)
    b.setup(ids[1], scs[1].dx)
    for sid, s in zip(ids, scs):
        want = snow.setup(s.particles.copy(), s.dx)
        got = b.download(sid)
        assert np.max(np.abs(got[:, 7] / want[:, 7] - 1)) < 1e-12


def test_automatic_work_item_size(snow):
    """A batch that has not been given a work-item size takes one from its
    particle count (about four items per resident CTA, 2 per SM in FP64,
    256..1024); the result equals the same steps at a fixed 256 up to the
    order of atomic sums."""
    import torch
    from snow_b200 import scenes

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    sc = scenes.snowball_scene(n=2_000_000)
    want = 256
    while want < 1024 and 2 * want <= sc.n // (8 * sms):
        want *= 2
    auto, fixed = snow.Batch(snow.SNOW_FP64), snow.Batch(snow.SNOW_FP64)
    fixed.set_chunk(256)
    ia, ib = auto.add(sc), fixed.add(sc)
    auto.setup(ia, sc.dx)
    fixed.setup(ib, sc.dx)
    auto.step(3)
    fixed.step(3)
    assert auto.chunk() == want and fixed.chunk() == 256
    assert max(errors(auto.download(ia), fixed.download(ib)).values()) < 1e-12
    auto.close()
    fixed.close()
