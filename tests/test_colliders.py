"""Colliders beyond make_plane: a solid sphere and a plane moving with a
constant velocity (the reference accepts any CollisionBody; these are the
analytic bodies the GPU step runs).

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
    bodies = np.array([
        [1, 0.503, 0.297, 0.501, 0, 0, 0, 0.0, 0.0, 0.0, 0.3, 0.0813],    # resting sphere under the cube
        [0, 0.0, 0.3613, 0.0, 0.01, 2, 0, 0.0, 0.5, 0.1, 0.2, 0.0],       # rising plane (normal not unit)
        [1, 0.4017, 0.4009, 0.5003, 0, 0, 0, -0.2, 0.0, 0.0, 0.0, 0.0307],  # small moving sphere, no friction
    ], dtype=np.float64)
    return sc, bodies


def _gpu_colliders(snow, bodies):
    out = []
    for r in bodies:
        if r[0] == 1:
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
    np.testing.assert_allclose(snow.body_rows(cols)[:, [0, 1, 2, 3, 7, 8, 9, 10, 11]],
                               bodies[:, [0, 1, 2, 3, 7, 8, 9, 10, 11]])
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
