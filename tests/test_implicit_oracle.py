"""The oracle's semi-implicit update (CPU only): the restatement of Stomakhin
et al. 2013's implicit velocity solve that the GPU implicit mode is checked
against.  The reference declares these functions and defines none, so the
oracle is pinned by the mathematics instead:

* constitutive_differential is the derivative of force_constitutive (central
  differences agree to 1e-6 relative) and a symmetric bilinear form
  (dP(a) : b = dP(b) : a to 1e-10), so the solve's operator is self-adjoint;
* apply_A is linear, and A q = q at beta = 0;
* a step at beta = 0 is the explicit step, and conjugate residuals reach the
  requested tolerance at beta = 1.
"""
import numpy as np

from snow_b200 import scenes


def _particle(rng, stretch=0.03):
    """A particle record whose F_E is a random rotation times a random stretch."""
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    s = 1 + rng.uniform(-stretch, stretch, 3)
    v, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    fe = q @ np.diag(s) @ v.T
    fp = np.eye(3) + rng.uniform(-0.01, 0.01, (3, 3))
    r = np.zeros(26)
    r[6], r[7] = 1e-3, 1e-6
    r[8:17] = fp.T.reshape(9)
    r[17:26] = fe.T.reshape(9)
    return r


def test_constitutive_differential_is_the_derivative_of_p(oracle):
    rng = np.random.default_rng(3)
    m = scenes.Material()
    for _ in range(20):
        r = _particle(rng)
        fe = r[17:26].reshape(3, 3).T
        d = rng.normal(size=(3, 3))
        eps = 1e-6
        rp, rm = r.copy(), r.copy()
        rp[17:26] = (fe + eps * d).T.reshape(9)
        rm[17:26] = (fe - eps * d).T.reshape(9)
        fd = (oracle.force_constitutive(rp, m.mu0, m.lambda0, m.xi) -
              oracle.force_constitutive(rm, m.mu0, m.lambda0, m.xi)) / (2 * eps)
        dp = oracle.constitutive_differential(r, d, m.mu0, m.lambda0, m.xi)
        assert np.linalg.norm(dp - fd) <= 1e-6 * np.linalg.norm(fd)


def test_constitutive_differential_is_symmetric(oracle):
    rng = np.random.default_rng(4)
    m = scenes.Material()
    for _ in range(20):
        r = _particle(rng)
        a, b = rng.normal(size=(3, 3)), rng.normal(size=(3, 3))
        ab = np.sum(oracle.constitutive_differential(r, a, m.mu0, m.lambda0, m.xi) * b)
        ba = np.sum(oracle.constitutive_differential(r, b, m.mu0, m.lambda0, m.xi) * a)
        assert abs(ab - ba) <= 1e-10 * max(abs(ab), 1.0)


def _deformed_cube(oracle, n_side=6):
    sc = scenes.cube_scene(n_side)
    sc.particles[:, 1] -= 0.448  # on the ground plane
    rec = oracle.setup(sc.particles, sc.dx)
    rec, _ = oracle.step(rec, sc.params(), sc.plane_array(), 5)  # F_E away from I
    return sc, rec


def test_apply_a_is_linear_and_the_identity_at_beta_zero(oracle):
    sc, rec = _deformed_cube(oracle)
    p, pl = sc.params(), sc.plane_array()
    rng = np.random.default_rng(5)
    ijk, _, _, _ = oracle.implicit_grid(rec, p, pl, 1.0, q=np.zeros((1, 3)))
    n = ijk.shape[0]
    u, v = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    au = oracle.implicit_grid(rec, p, pl, 1.0, q=u)[2]
    av = oracle.implicit_grid(rec, p, pl, 1.0, q=v)[2]
    auv = oracle.implicit_grid(rec, p, pl, 1.0, q=2 * u - 3 * v)[2]
    assert np.allclose(auv, 2 * au - 3 * av, rtol=1e-10, atol=1e-12)
    assert not np.allclose(au, u)
    a0 = oracle.implicit_grid(rec, p, pl, 0.0, q=u)[2]
    assert np.array_equal(a0, u)


def test_implicit_step_converges_and_beta_zero_is_explicit(oracle):
    sc, rec = _deformed_cube(oracle)
    explicit, _ = oracle.step(rec, sc.params(), sc.plane_array(), 3)
    zero, its0, _ = oracle.step_implicit(rec, sc.params(), sc.plane_array(), 3, 0.0)
    assert np.array_equal(zero, explicit) and not its0.any()
    imp, its, res = oracle.step_implicit(rec, sc.params(), sc.plane_array(), 3, 1.0, squared_tolerance=1e-20,
                                         max_iterations=200)
    assert (its > 0).all() and (res <= 1e-10).all(), (its, res)
    d = np.abs(imp[:, 3:6] - explicit[:, 3:6]).max()
    assert 0 < d < 0.1, d
