"""Seeded synthetic snow scenes.

The reference solver reads its particles from ``groups.csv``/``particles.csv``
(src/import.cpp:131) written by a Blender add-on; there is no public dataset.
These generators build the scenes the benchmark and the parity tests use:
a jittered lattice cube, two tori, a sphere ("snowball") and the mixed batch,
with particle mass = rho0 * spacing^3 and the material constants in
:class:`Material`.  Everything is seeded and deterministic.

A particle set is returned as an ``(n, 26)`` float64 array of particle records in
the reference's ``struct Particle`` order (include/snow/particle.hpp:5-28):
``x_p[3], v_p[3], m_p, V_p0, F_P[9], F_E[9]`` (matrices column-major), with
V_p0 = 0 and F_P = F_E = I as ``assemble_particles`` leaves them
(src/import.cpp:126).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

RECORD = 26  # doubles per particle record (208 bytes)
X, V, M, VOL, FP, FE = slice(0, 3), slice(3, 6), 6, 7, slice(8, 17), slice(17, 26)
_EYE = np.eye(3).reshape(-1, order="F")


@dataclasses.dataclass
class Material:
    """Material and integration constants passed to ``step`` (src/grid.cpp:359)."""

    E: float = 1.4e5
    nu: float = 0.2
    xi: float = 10.0
    theta_c: float = 2.5e-2
    theta_s: float = 7.5e-3
    alpha: float = 0.95
    gravity: tuple = (0.0, -9.81, 0.0)

    @property
    def mu0(self) -> float:  # src/main.cpp:28
        return self.E / (2 * (1 + self.nu))

    @property
    def lambda0(self) -> float:  # src/main.cpp:29
        return self.E * self.nu / ((1 + self.nu) * (1 - 2 * self.nu))


@dataclasses.dataclass
class Scene:
    particles: np.ndarray          # (n, 26) records
    dx: float
    dt: float
    steps: int
    material: Material
    planes: list                   # [(point3, normal3, friction)]
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.particles.shape[0])

    def params(self) -> np.ndarray:
        """The 11 step parameters: gravity[3], dt, dx, mu0, lambda0, xi, theta_c, theta_s, alpha."""
        m = self.material
        return np.array([*m.gravity, self.dt, self.dx, m.mu0, m.lambda0, m.xi, m.theta_c,
                         m.theta_s, m.alpha], dtype=np.float64)

    def plane_array(self) -> np.ndarray:
        """Colliders as (k, 7): point[3], normal[3] (as given to make_plane), friction."""
        a = np.zeros((len(self.planes), 7))
        for i, (p, nrm, mu) in enumerate(self.planes):
            a[i, :3], a[i, 3:6], a[i, 6] = p, nrm, mu
        return a


def records(x: np.ndarray, v: np.ndarray, m: np.ndarray | float) -> np.ndarray:
    n = x.shape[0]
    r = np.zeros((n, RECORD))
    r[:, X] = x
    r[:, V] = v
    r[:, M] = m
    r[:, FP] = _EYE
    r[:, FE] = _EYE
    return r


GROUND = ((0.0, 0.05, 0.0), (0.0, 1.0, 0.0), 0.2)


def cube(n_side: int = 32, spacing: float = 0.01, lo=(0.34, 0.5, 0.34), jitter: float = 0.001,
         velocity=(0.0, -2.0, 0.0), rho0: float = 400.0, seed: int = 0) -> np.ndarray:
    """Jittered n_side^3 lattice cube (the 32,768-particle cube of the small case)."""
    rng = np.random.default_rng(seed)
    g = np.arange(n_side) * spacing
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) + np.asarray(lo)
    x = x + rng.uniform(-jitter, jitter, x.shape)
    return records(x, np.broadcast_to(velocity, x.shape), rho0 * spacing ** 3)


def cube_scene(n_side: int = 32, steps: int = 100, seed: int = 0) -> Scene:
    """One snow cube, 32^3 particles at 0.01 m, dx = 0.02, dt = 1e-4, ground plane y = 0.05."""
    return Scene(cube(n_side, seed=seed), dx=0.02, dt=1e-4, steps=steps, material=Material(),
                 planes=[GROUND], name=f"cube{n_side}^3")


def _lattice_in(pred, lo, hi, h, jitter_frac, rng):
    axes = [np.arange(lo[a] + 0.5 * h, hi[a], h) for a in range(3)]
    x = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    x = x[pred(x)]
    return x + rng.uniform(-jitter_frac * h, jitter_frac * h, x.shape)


def torus(center, R: float, r: float, n_target: int, rng, axis: int = 0, exact: bool = False):
    """Jittered lattice torus of about n_target particles (exactly n_target with
    `exact`: a slightly finer lattice, then a seeded subset in lattice order);
    symmetry axis along `axis`."""
    h = (2 * math.pi ** 2 * R * r * r / n_target) ** (1 / 3)
    if exact:
        x, _ = torus(center, R, r, int(n_target * 1.03) + 64, rng, axis)
        keep = np.sort(rng.choice(x.shape[0], n_target, replace=False))
        return x[keep], h
    c = np.asarray(center)
    ext = R + r
    lo, hi = c - ext, c + ext
    ax = axis
    o1, o2 = [a for a in range(3) if a != ax]

    def inside(x):
        d = x - c
        rad = np.sqrt(d[:, o1] ** 2 + d[:, o2] ** 2)
        return (rad - R) ** 2 + d[:, ax] ** 2 <= r * r

    x = _lattice_in(inside, lo, hi, h, 0.1, rng)
    return x, h


def tori_scene(n_per_torus: int = 325_000, steps: int = 500, seed: int = 1, gap: float | None = None) -> Scene:
    """Two colliding tori, R = 0.15, r = 0.06, +-8 m/s along x.

    The symmetry axis is x (the direction of motion), so the tori do not
    overlap at t = 0; spacing h = (2 pi^2 R r^2 / n)^(1/3) gives n per torus.
    By default the centres are (0.3, 0.5, 0.5) and (0.7, 0.5, 0.5), 0.286 m
    apart along x, which the tori do not close within 500 steps.  With `gap`
    the centres are placed symmetrically about x = 0.5 with `gap` metres
    between the tori (0: touching), so the snow deforms from the first steps:
    the same particles, moved rigidly along x.
    """
    rng = np.random.default_rng(seed)
    xa, h = torus((0.3, 0.5, 0.5), 0.15, 0.06, n_per_torus, rng, exact=True)
    xb, _ = torus((0.7, 0.5, 0.5), 0.15, 0.06, n_per_torus, rng, exact=True)
    if gap is not None:
        shift = 0.2 - 0.06 - 0.5 * gap  # centre at 0.5 -+ (r + gap / 2)
        xa[:, 0] += shift
        xb[:, 0] -= shift
    m = 400.0 * h ** 3
    ra = records(xa, np.broadcast_to((8.0, 0.0, 0.0), xa.shape), m)
    rb = records(xb, np.broadcast_to((-8.0, 0.0, 0.0), xb.shape), m)
    name = f"two-tori-{ra.shape[0] + rb.shape[0]}" + ("" if gap is None else f"-gap{gap:g}")
    return Scene(np.concatenate([ra, rb]), dx=0.01, dt=2e-5, steps=steps, material=Material(),
                 planes=[GROUND], name=name)


def sphere(center, radius: float, n_target: int, rng, jitter_frac: float = 0.1):
    h = (4 / 3 * math.pi * radius ** 3 / n_target) ** (1 / 3)
    c = np.asarray(center)
    x = _lattice_in(lambda p: ((p - c) ** 2).sum(1) <= radius * radius, c - radius, c + radius,
                    h, jitter_frac, rng)
    return x, h


def snowball_scene(n: int = 4_000_000, steps: int = 200, seed: int = 2) -> Scene:
    """Snowball r = 0.2 at (0.3,0.5,0.5), 12 m/s toward a wall at x = 0.9."""
    rng = np.random.default_rng(seed)
    x, h = sphere((0.3, 0.5, 0.5), 0.2, n, rng)
    mat = Material(theta_c=1.9e-2)
    wall = ((0.9, 0.0, 0.0), (-1.0, 0.0, 0.0), 0.2)
    return Scene(records(x, np.broadcast_to((12.0, 0.0, 0.0), x.shape), 400.0 * h ** 3),
                 dx=0.005, dt=1e-5, steps=steps, material=mat, planes=[GROUND, wall],
                 name=f"snowball-{x.shape[0]}")


def _ground(x: np.ndarray, vel: np.ndarray, h: float):
    """Rests a particle set on the ground plane (lowest particle half a lattice
    spacing above y = 0.05) and turns its velocity downward, so it strikes the
    ground in its first steps."""
    x = x.copy()
    x[:, 1] += 0.05 + 0.5 * h - x[:, 1].min()
    v = np.array(vel, dtype=np.float64)
    v[1] = -abs(v[1]) - 1.0
    return x, v


def batch_scenes(count: int = 256, lo: int = 1000, hi: int = 64000, seed: int = 3,
                 dt: float = 5e-5, steps: int = 200, grounded: bool = False) -> list[Scene]:
    """Independent scenes with log-uniform particle counts, box or sphere, random
    velocity in [-5,5]^3 and material drawn per scene; dx = 0.02, spacing 0.01.
    By default every scene starts 0.25 m or more above the ground plane (free
    flight for 200 steps); `grounded` sets each scene on the ground moving
    down (vy = -|vy| - 1 m/s), so it deforms plastically from its first steps."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(count):
        n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        mat = Material(E=float(rng.uniform(4.8e4, 1.4e5)), theta_c=float(rng.uniform(1.9e-2, 2.5e-2)),
                       theta_s=float(rng.uniform(5e-3, 7.5e-3)), xi=float(rng.uniform(5, 10)))
        vel = rng.uniform(-5, 5, 3)
        h = 0.01
        if rng.uniform() < 0.5:
            side = n ** (1 / 3)
            k = max(1, int(round(side)))
            ext = k * h
            lo_c = np.array([0.5 - ext / 2, 0.3, 0.5 - ext / 2])
            g = np.arange(k) * h
            x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) + lo_c
            x = x + rng.uniform(-0.1 * h, 0.1 * h, x.shape)
        else:
            rad = (3 * n / (4 * math.pi)) ** (1 / 3) * h
            x, _ = sphere((0.5, 0.3 + rad, 0.5), rad, n, rng)
        if grounded:
            x, vel = _ground(x, vel, h)
        out.append(Scene(records(x, np.broadcast_to(vel, x.shape), 400.0 * h ** 3), dx=0.02,
                         dt=dt, steps=steps, material=mat, planes=[GROUND], name=f"batch{s}"))
    return out


def served_requests(count: int = 64, rate: float = 200.0, lo: int = 2000, hi: int = 500_000,
                    steps_lo: int = 100, steps_hi: int = 2000, seed: int = 4, dt: float = 5e-5,
                    grounded: bool = False):
    """A Poisson stream of scene requests: (scene, steps, arrival seconds).

    Particle counts are log-uniform in [lo, hi], shapes box / sphere / torus at
    lattice spacing 0.01 (so the count sets the size), velocity in [-5, 5]^3,
    material drawn as for the batch scenes, steps uniform in [steps_lo,
    steps_hi], grid dx = 0.02, ground plane.  `grounded` as for batch_scenes."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for r in range(count):
        t += rng.exponential(1.0 / rate)
        n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        mat = Material(E=float(rng.uniform(4.8e4, 1.4e5)), theta_c=float(rng.uniform(1.9e-2, 2.5e-2)),
                       theta_s=float(rng.uniform(5e-3, 7.5e-3)), xi=float(rng.uniform(5, 10)))
        vel = rng.uniform(-5, 5, 3)
        h = 0.01
        shape = int(rng.integers(3))
        if shape == 0:
            k = max(1, int(round(n ** (1 / 3))))
            g = np.arange(k) * h
            x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
            x = x + np.array([0.5 - k * h / 2, 0.3, 0.5 - k * h / 2]) + rng.uniform(-0.1 * h, 0.1 * h, x.shape)
        elif shape == 1:
            rad = (3 * n / (4 * math.pi)) ** (1 / 3) * h
            x, _ = sphere((0.5, 0.3 + rad, 0.5), rad, n, rng)
        else:
            r_minor = (n * h ** 3 / (2 * math.pi ** 2 * 2.5)) ** (1 / 3)  # R = 2.5 r
            x, _ = torus((0.5, 0.3 + r_minor, 0.5), 2.5 * r_minor, r_minor, n, rng, axis=1)
        if grounded:
            x, vel = _ground(x, vel, h)
        steps = int(rng.integers(steps_lo, steps_hi + 1))
        sc = Scene(records(x, np.broadcast_to(vel, x.shape), 400.0 * h ** 3), dx=0.02, dt=dt, steps=steps,
                   material=mat, planes=[GROUND], name=f"request{r}")
        out.append((sc, steps, t))
    return out
