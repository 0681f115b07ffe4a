"""Colliders beyond make_plane: a solid sphere, a plane moving with a
constant velocity and a solid oriented box (the reference accepts any
CollisionBody; these are the analytic bodies the GPU step runs).

Pinned on the CPU against the reference's own collision code (its
collision_helper with CollisionBody functions for the sphere and the moving
plane, oracle/_ref) and the oracle; on the GPU the FP64 path matches the
reference to the parity bound (1e-10 after 10 steps) and the mixed form stays
within the mixed bound.
"""
import os

import numpy as np
import pytest

from oracle_lib import REF_SO, Reference, errors


def _scene():
    from snow_b200 import scenes

    rec = scenes.cube(8, lo=(0.45, 0.35, 0.45), velocity=(0.3, -1.5, 0.2), seed=9)
    sc = scenes.Scene(rec, dx=0.02, dt=1e-4, steps=10, material=scenes.Material(), planes=[])
    # kind, point, normal, velocity, friction, radius.  Off the grid's lattice: a
    # node exactly on a collider surface (phi = 0) is in contact or not by one
    # rounding, which the float form need not reproduce.
    z6 = [0.0] * 6
    bodies = np.array([
        [1, 0.503, 0.297, 0.501, 0, 0, 0, 0.0, 0.0, 0.0, 0.3, 0.0813] + z6,    # resting sphere under the cube
        [0, 0.0, 0.3613, 0.0, 0.01, 2, 0, 0.0, 0.5, 0.1, 0.2, 0.0] + z6,       # rising plane (normal not unit)
        [1, 0.4017, 0.4009, 0.5003, 0, 0, 0, -0.2, 0.0, 0.0, 0.0, 0.0307] + z6,  # small moving sphere, no friction
    ], dtype=np.float64)
    # a tilted box whose top face the cube's corner falls onto, sliding slowly in z
    u = np.array([1.0, 0.27, 0.11])
    u /= np.linalg.norm(u)
    w = np.array([-0.25, 1.0, 0.13])
    w -= u.dot(w) * u
    w /= np.linalg.norm(w)
    box = [2, 0.5407, 0.3311, 0.4893, *u, 0.0, 0.0, 0.07, 0.25, 0.0, *w, 0.0413, 0.0237, 0.0519]
    bodies = np.vstack([bodies, np.array(box)])
    return sc, bodies


def _gpu_colliders(snow, bodies):
    out = []
    for r in bodies:
        if r[0] == 2:
            out.append(snow.box(r[1:4], r[15:18], r[4:7], r[12:15], r[10], velocity=r[7:10]))
        elif r[0] == 1:
            out.append(snow.sphere(r[1:4], r[11], r[10], velocity=r[7:10]))
        else:
            out.append(snow.moving_plane(r[1:4], r[4:7], r[10], r[7:10]))
    return out


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference build (oracle/_ref) not present")
def test_oracle_bodies_match_reference(oracle):
    sc, bodies = _scene()
    rec = oracle.setup(sc.particles, sc.dx)
    want, _ = Reference().step_bodies(rec, sc.params(), bodies, 10)
    got, _ = oracle.step_bodies(rec, sc.params(), bodies, 10)
    moved = np.abs(got[:, 3:6] - rec[:, 3:6]).max()
    assert moved > 0.01, "the bodies should act on the particles"
    assert max(errors(got, want).values()) < 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_gpu_bodies_match_reference(snow, oracle, prec):
    sc, bodies = _scene()
    rec = oracle.setup(sc.particles, sc.dx)
    if os.path.exists(REF_SO):
        want, _ = Reference().step_bodies(rec, sc.params(), bodies, 10)
    else:
        want, _ = oracle.step_bodies(rec, sc.params(), bodies, 10)
    cols = _gpu_colliders(snow, bodies)
    keep = [0, 1, 2, 3, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17]
    np.testing.assert_allclose(snow.body_rows(cols)[:, keep], bodies[:, keep], rtol=0, atol=1e-15)
    b = snow.Batch(prec)
    sid = b.add_scene(rec, sc.params(), cols)
    b.step(10)
    got = b.download(sid)
    b.close()
    e = errors(got, want)
    if prec == 0:
        assert max(e.values()) < 1e-10, e
    else:
        assert e["x"] < 1e-4 and e["v"] < 5e-3 and e["F_E"] < 1e-4 and e["F_P"] < 1e-4, e


@pytest.mark.gpu
def test_sphere_needs_a_radius(snow):
    sc, _ = _scene()
    b = snow.Batch(0)
    with pytest.raises(snow.SnowError):
        b.add_scene(sc.particles, sc.params(), [snow.sphere((0.5, 0.3, 0.5), 0.0, 0.2)])
    b.close()


def test_oracle_box_touches_the_cube(oracle):
    """CPU only: the box in the scene acts on the particles (its removal changes
    the result), so the GPU comparison above exercises box contacts."""
    sc, bodies = _scene()
    rec = oracle.setup(sc.particles, sc.dx)
    with_box, _ = oracle.step_bodies(rec, sc.params(), bodies, 10)
    without, _ = oracle.step_bodies(rec, sc.params(), bodies[:3], 10)
    assert np.abs(with_box[:, 3:6] - without[:, 3:6]).max() > 1e-3


@pytest.mark.gpu
def test_box_needs_unit_orthogonal_axes(snow):
    sc, _ = _scene()
    b = snow.Batch(0)
    bad = snow.box((0.5, 0.3, 0.5), (0.1, 0.1, 0.1), (1, 0, 0), (0, 1, 0), 0.2)
    bad.axis[0] = 0.5  # no longer orthogonal to the first axis
    with pytest.raises(snow.SnowError):
        b.add_scene(sc.particles, sc.params(), [bad])
    b.close()
