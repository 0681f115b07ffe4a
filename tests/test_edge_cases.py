"""Edge cases of the GPU step: empty and single-particle scenes, a particle
whose position is not finite, and scenes too far apart for the block keys.

An empty scene next to a normal one leaves the normal one exactly as alone
(FP64, 1e-12: only the order of atomic sums differs); a one-particle scene
matches the oracle to the FP64 parity bound (1e-10); the error cases end the
call with the matching status code instead of a wrong result.
"""
import numpy as np
import pytest

from oracle_lib import errors

pytestmark = pytest.mark.gpu


def _cube(seed=2, n_side=6, lo=(0.3, 0.3, 0.3)):
    from snow_b200 import scenes

    rec = scenes.cube(n_side, lo=lo, velocity=(0.2, -1.0, 0.1), seed=seed)
    return scenes.Scene(rec, dx=0.02, dt=1e-4, steps=5, material=scenes.Material(),
                        planes=[((0, 0.05, 0), (0, 1, 0), 0.2)])


def test_empty_scene_beside_a_normal_one(snow):
    sc = _cube()
    rec = snow.setup(sc.particles.copy(), sc.dx)
    alone = snow.Batch(snow.SNOW_FP64)
    a = alone.add_scene(rec, sc.params(), sc.planes)
    alone.step(5)
    want = alone.download(a)
    alone.close()

    b = snow.Batch(snow.SNOW_FP64)
    e0 = b.add_scene(np.zeros((0, 26)), sc.params(), sc.planes)
    s1 = b.add_scene(rec, sc.params(), sc.planes)
    e2 = b.add_scene(np.zeros((0, 26)), sc.params(), sc.planes)
    b.step(5)
    got = b.download(s1)
    assert b.download(e0).shape == (0, 26) and b.download(e2).shape == (0, 26)
    b.close()
    assert max(errors(got, want).values()) < 1e-12


@pytest.mark.parametrize("prec", [0, 1])
def test_single_particle(snow, oracle, prec):
    sc = _cube(n_side=1)
    rec = oracle.setup(sc.particles, sc.dx)
    want, _ = oracle.step(rec, sc.params(), sc.plane_array(), 10)
    b = snow.Batch(prec)
    sid = b.add_scene(rec, sc.params(), sc.planes)
    b.step(10)
    got = b.download(sid)
    b.close()
    e = errors(got, want)
    tol = 1e-10 if prec == 0 else 1e-4
    assert max(e["x"], e["F_E"]) < tol, e


@pytest.mark.parametrize("graphs", [True, False])
def test_particle_outrunning_its_key_box(snow, oracle, graphs):
    """G2P writes the next step's sort keys against the particles' block box
    grown by one block; a particle that moves more than a block in one step
    (here 0.12 m per step, 1.5 blocks at dx = 0.02) falls outside it, and that
    step's keys come from the keys kernel instead, after the counts G2P wrote
    are cleared.  The result matches the oracle to the FP64 parity bound over
    steps that take that path and steps that do not."""
    sc = _cube()
    fast = sc.particles[:1].copy()
    fast[0, 0:3] = (0.1, 0.6, 0.5)
    fast[0, 3:6] = (1200.0, 0.0, 0.0)
    rec0 = np.concatenate([sc.particles, fast])
    rec = oracle.setup(rec0, sc.dx)
    want, _ = oracle.step(rec, sc.params(), sc.plane_array(), 6)
    b = snow.Batch(snow.SNOW_FP64)
    b.set_graphs(graphs)
    sid = b.add_scene(rec, sc.params(), sc.planes)
    b.step(3)
    b.step(3)
    got = b.download(sid)
    b.close()
    e = errors(got, want)
    assert max(e.values()) < 1e-10, e


def test_nonfinite_position_is_reported(snow):
    sc = _cube()
    rec = snow.setup(sc.particles.copy(), sc.dx)
    rec[7, 1] = np.nan
    b = snow.Batch(snow.SNOW_FP64)
    b.add_scene(rec, sc.params(), sc.planes)
    with pytest.raises(snow.SnowError) as err:
        b.step(2)
    assert err.value.code == -4  # SNOW_E_NONFINITE
    b.close()


def test_long_thin_scene_is_stepped(snow, oracle):
    """A particle 100 m away along x only: a long box (~1.3e4 blocks), still within the keys."""
    sc = _cube(n_side=2)
    rec = oracle.setup(sc.particles, sc.dx)
    rec[-1, 0] += 100.0
    want, _ = oracle.step(rec, sc.params(), sc.plane_array(), 3)
    b = snow.Batch(snow.SNOW_FP64)
    sid = b.add_scene(rec, sc.params(), sc.planes)
    b.step(3)
    got = b.download(sid)
    b.close()
    assert max(errors(got, want).values()) < 1e-10


def test_scene_beyond_key_range_is_reported(snow):
    sc = _cube(n_side=2)
    rec = snow.setup(sc.particles.copy(), sc.dx)
    rec[-1, 0:3] += 100.0  # one particle 100 m away on every axis: ~2e9 blocks in the scene's box
    b = snow.Batch(snow.SNOW_FP64)
    b.add_scene(rec, sc.params(), sc.planes)
    with pytest.raises(snow.SnowError) as err:
        b.step(1)
    assert err.value.code == -5  # SNOW_E_KEYRANGE
    b.close()


def test_zero_steps_leave_state_alone(snow):
    sc = _cube()
    rec = snow.setup(sc.particles.copy(), sc.dx)
    b = snow.Batch(snow.SNOW_FP64)
    sid = b.add_scene(rec, sc.params(), sc.planes)
    b.step(0)
    got = b.download(sid)
    b.close()
    assert np.array_equal(got, rec)


def test_snapshot_and_restore(snow):
    """A scene put back to its snapshot continues exactly as it did from there."""
    sc = _cube()
    rec = snow.setup(sc.particles.copy(), sc.dx)
    b = snow.Batch(snow.SNOW_FP64)
    other = b.add_scene(_cube(seed=5, lo=(0.6, 0.3, 0.6)).particles, sc.params(), sc.planes)
    sid = b.add_scene(rec, sc.params(), sc.planes)
    b.step(2)
    before = b.download(sid)
    b.snapshot(sid)
    b.step(5)
    first = b.download(sid)
    b.restore(sid)
    assert np.array_equal(b.download(sid), before)
    b.step(5)
    again = b.download(sid)
    b.close()
    assert max(errors(again, first).values()) < 1e-12
    with pytest.raises(snow.SnowError):
        b2 = snow.Batch(snow.SNOW_FP64)
        try:
            s2 = b2.add_scene(rec, sc.params(), sc.planes)
            b2.restore(s2)
        finally:
            b2.close()
    assert other >= 0


def test_fresh_start_after_emitted_keys(snow, oracle):
    """G2P writes the next step's sort keys and counts as it goes; a change of
    scenes between two steps makes the next step sort afresh and must clear
    every count the finished step left behind, also when the scene's block box
    shrank in between (a fast-moving scene loses a block column at one end
    while it gains one at the other).  A tiny scene added and removed after
    every step forces the fresh start; the result equals the oracle's."""
    from snow_b200 import scenes

    sc = scenes.cube_scene(10)
    rec = oracle.setup(sc.particles, sc.dx)
    rec[:, 3] = -300.0  # 3 cm per step: a block column every few steps
    want, _ = oracle.step(rec, sc.params(), sc.plane_array(), 12)
    tiny = scenes.cube_scene(2)
    b = snow.Batch(snow.SNOW_FP64)
    sid = b.add_scene(rec, sc.params(), sc.planes)
    for _ in range(12):
        b.step(1)
        t = b.add_scene(tiny.particles, tiny.params(), tiny.planes)
        b.remove_scene(t)
    got = b.download(sid)
    b.close()
    e = errors(got, want)
    assert max(e.values()) < 1e-10, e


@pytest.mark.parametrize("prec", [0, 1])
def test_download_positions_match_records(snow, prec):
    """The positions-only read-back (what a frame export reads) equals the
    position columns of the full records, in the particles' original order."""
    from snow_b200 import scenes

    sc = scenes.cube_scene(8)
    b = snow.Batch(prec)
    sid = b.add_scene(snow.setup(sc.particles.copy(), sc.dx), sc.params(), sc.planes)
    b.step(3)
    pos = b.download_positions(sid)
    rec = b.download(sid)
    b.close()
    assert pos.shape == (rec.shape[0], 3)
    assert np.array_equal(pos, rec[:, 0:3])
