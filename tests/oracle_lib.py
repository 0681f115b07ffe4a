"""ctypes access to the ORACLE (test infrastructure only).

* ``oracle/liboracle.so``      the CPU restatement of the MPM step
* ``oracle/_ref/libsnow_ref.so`` the reference's own sources compiled against
  the project's Eigen-subset shim (present where it was built)

Both take (n, 26) float64 particle records and the 11 step parameters of
:meth:`snow_b200.scenes.Scene.params`.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libsnow_ref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


class _StepLib:
    prefix = ""

    def __init__(self, path: str):
        self.L = ctypes.CDLL(path)
        f = getattr(self.L, self.prefix + "_setup")
        f.argtypes, f.restype = [_dp, ctypes.c_int64, ctypes.c_double], None
        for name in ("_step", "_step_bodies"):
            f = getattr(self.L, self.prefix + name)
            f.argtypes = [_dp, ctypes.c_int64, _dp, _dp, ctypes.c_int, ctypes.c_int, _dp]
            f.restype = None

    def setup(self, rec: np.ndarray, dx: float) -> np.ndarray:
        out = np.ascontiguousarray(rec, dtype=np.float64).copy()
        getattr(self.L, self.prefix + "_setup")(_p(out), out.shape[0], float(dx))
        return out

    def step_bodies(self, rec: np.ndarray, params, bodies, steps: int = 1):
        """Like step() with general colliders: (k, 18) rows of kind (0 plane, 1 sphere,
        2 oriented box), point[3], normal[3], velocity[3], friction, radius, axis[3],
        extent[3] (the box's centre, first axis, second axis and half extents)."""
        out = np.ascontiguousarray(rec, dtype=np.float64).copy()
        prm = np.ascontiguousarray(params, dtype=np.float64)
        b = np.asarray(bodies, dtype=np.float64)
        b = b.reshape(-1, b.shape[-1]) if b.size else np.zeros((0, 18))
        if b.shape[1] < 18:
            b = np.concatenate([b, np.zeros((b.shape[0], 18 - b.shape[1]))], axis=1)
        b = np.ascontiguousarray(b)
        ms = np.zeros(11)
        getattr(self.L, self.prefix + "_step_bodies")(_p(out), out.shape[0], _p(prm), _p(b), b.shape[0],
                                                      int(steps), _p(ms))
        return out, ms

    def step(self, rec: np.ndarray, params, planes, steps: int = 1):
        """Returns (new records, milliseconds[11]: ten stages, then the step loop's wall time)."""
        out = np.ascontiguousarray(rec, dtype=np.float64).copy()
        prm = np.ascontiguousarray(params, dtype=np.float64)
        pl = np.ascontiguousarray(np.asarray(planes, dtype=np.float64).reshape(-1, 7))
        ms = np.zeros(11)
        getattr(self.L, self.prefix + "_step")(_p(out), out.shape[0], _p(prm), _p(pl), pl.shape[0],
                                               int(steps), _p(ms))
        return out, ms


class Oracle(_StepLib):
    prefix = "oracle"

    def __init__(self, path: str = ORACLE_SO):
        super().__init__(path)
        L = self.L
        L.oracle_N.argtypes = [ctypes.c_double, ctypes.c_double]
        L.oracle_N.restype = ctypes.c_double
        L.oracle_N_dash.argtypes = [ctypes.c_double, ctypes.c_double]
        L.oracle_N_dash.restype = ctypes.c_double
        L.oracle_grid_new.restype = ctypes.c_void_p
        L.oracle_grid_free.argtypes = [ctypes.c_void_p]
        L.oracle_grid_size.argtypes = [ctypes.c_void_p]
        L.oracle_grid_size.restype = ctypes.c_int64
        L.oracle_grid_export.argtypes = [ctypes.c_void_p, _ip, _dp]
        L.oracle_grid_set.argtypes = [ctypes.c_void_p, _ip, _dp, ctypes.c_int64]
        L.oracle_p2g.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int64, ctypes.c_double]
        L.oracle_calculate_volume.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int64, ctypes.c_double]
        L.oracle_force_calculation.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int64] + [ctypes.c_double] * 4
        L.oracle_grid_velocity.argtypes = [ctypes.c_void_p, _dp, ctypes.c_double]
        L.oracle_grid_collisions.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_double]
        L.oracle_stress_update.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int64] + [ctypes.c_double] * 4
        L.oracle_g2p.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int64, ctypes.c_double, ctypes.c_double]
        L.oracle_particle_collisions.argtypes = [_dp, ctypes.c_int64, _dp, ctypes.c_int]
        L.oracle_position_update.argtypes = [_dp, ctypes.c_int64, ctypes.c_double]
        L.oracle_svd3.argtypes = [_dp, _dp, _dp, _dp]

    def step_implicit(self, rec: np.ndarray, params, planes, steps: int, beta: float,
                      squared_tolerance: float = 1e-12, max_iterations: int = 50):
        """Steps with the semi-implicit update; returns (records, iterations[steps], residual[steps])."""
        L = self.L
        L.oracle_step_implicit.argtypes = [_dp, ctypes.c_int64, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_int, _ip, _dp]
        out = np.ascontiguousarray(rec, dtype=np.float64).copy()
        prm = np.ascontiguousarray(params, dtype=np.float64)
        pl = np.ascontiguousarray(np.asarray(planes, dtype=np.float64).reshape(-1, 7))
        its = np.zeros(steps, np.int32)
        res = np.zeros(steps)
        L.oracle_step_implicit(_p(out), out.shape[0], _p(prm), _p(pl), pl.shape[0], int(steps), float(beta),
                               float(squared_tolerance), int(max_iterations), _p(its, _ip), _p(res))
        return out, its, res

    def constitutive_differential(self, rec1: np.ndarray, dF: np.ndarray, mu0, lambda0, xi) -> np.ndarray:
        """dP (3x3) of one particle record for the 3x3 dF (both as numpy 3x3 arrays)."""
        self.L.oracle_constitutive_differential.argtypes = [_dp, _dp] + [ctypes.c_double] * 3 + [_dp]
        r = np.ascontiguousarray(rec1, dtype=np.float64).reshape(26)
        d = np.ascontiguousarray(np.asarray(dF, dtype=np.float64).T.reshape(9))  # column-major
        out = np.zeros(9)
        self.L.oracle_constitutive_differential(_p(r), _p(d), mu0, lambda0, xi, _p(out))
        return out.reshape(3, 3).T

    def force_constitutive(self, rec1: np.ndarray, mu0, lambda0, xi) -> np.ndarray:
        self.L.oracle_force_constitutive.argtypes = [_dp] + [ctypes.c_double] * 3 + [_dp]
        r = np.ascontiguousarray(rec1, dtype=np.float64).reshape(26)
        out = np.zeros(9)
        self.L.oracle_force_constitutive(_p(r), mu0, lambda0, xi, _p(out))
        return out.reshape(3, 3).T

    def implicit_grid(self, rec: np.ndarray, params, planes, beta: float, q: np.ndarray | None = None,
                      squared_tolerance: float = 1e-24, max_iterations: int = 300):
        """The grid one step of the records builds (its nodes with mass): returns
        (ijk, fields[m][10] before the solve, A q -- or the solved velocities
        when q is None --, iterations).  q is taken over the first m rows."""
        L = self.L
        L.oracle_implicit_grid.argtypes = [_dp, ctypes.c_int64, _dp, _dp, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_int, _dp, _dp, _ip, _dp, ctypes.c_int64, _ip]
        L.oracle_implicit_grid.restype = ctypes.c_int64
        r = np.ascontiguousarray(rec, dtype=np.float64)
        prm = np.ascontiguousarray(params, dtype=np.float64)
        pl = np.ascontiguousarray(np.asarray(planes, dtype=np.float64).reshape(-1, 7))
        m = L.oracle_implicit_grid(_p(r), r.shape[0], _p(prm), _p(pl), pl.shape[0], beta, squared_tolerance,
                                   max_iterations, None, None, None, None, 0, None)
        out = np.zeros((m, 3))
        ijk = np.zeros((m, 3), np.int32)
        fields = np.zeros((m, 10))
        it = np.zeros(1, np.int32)
        qq = None
        if q is not None:
            qq = np.zeros((m, 3))
            qn = np.asarray(q, dtype=np.float64).reshape(-1, 3)
            qq[: min(m, qn.shape[0])] = qn[:m]
        L.oracle_implicit_grid(_p(r), r.shape[0], _p(prm), _p(pl), pl.shape[0], beta, squared_tolerance,
                               max_iterations, None if qq is None else _p(qq), _p(out), _p(ijk, _ip), _p(fields), m,
                               _p(it, _ip))
        return ijk, fields, out, int(it[0])

    def N(self, a, b):
        return self.L.oracle_N(float(a), float(b))

    def N_dash(self, a, b):
        return self.L.oracle_N_dash(float(a), float(b))


class OracleGrid:
    """The oracle's std::unordered_map grid, as node lists (ijk, fields[10])."""

    def __init__(self, oracle: Oracle):
        self.o = oracle
        self.h = ctypes.c_void_p(oracle.L.oracle_grid_new())

    def __del__(self):
        try:
            self.o.L.oracle_grid_free(self.h)
        except Exception:
            pass

    def set(self, ijk, fields):
        ijk = np.ascontiguousarray(ijk, dtype=np.int32).reshape(-1, 3)
        f = np.ascontiguousarray(fields, dtype=np.float64).reshape(-1, 10)
        self.o.L.oracle_grid_set(self.h, _p(ijk, _ip), _p(f), ijk.shape[0])
        return self

    def nodes(self):
        n = self.o.L.oracle_grid_size(self.h)
        ijk = np.zeros((n, 3), np.int32)
        f = np.zeros((n, 10))
        if n:
            self.o.L.oracle_grid_export(self.h, _p(ijk, _ip), _p(f))
        return ijk, f

    def as_dict(self):
        ijk, f = self.nodes()
        return {tuple(int(v) for v in k): row for k, row in zip(ijk, f)}


class Reference(_StepLib):
    prefix = "ref"

    def __init__(self, path: str = REF_SO):
        super().__init__(path)


def reference_available() -> bool:
    return os.path.exists(REF_SO)


def rel_err(a: np.ndarray, b: np.ndarray, floor: float = 1e-6) -> float:
    """max_i ||a_i - b_i|| / max(||b_i||, floor) over rows."""
    a = np.asarray(a).reshape(a.shape[0], -1)
    b = np.asarray(b).reshape(b.shape[0], -1)
    num = np.linalg.norm(a - b, axis=1)
    den = np.maximum(np.linalg.norm(b, axis=1), floor)
    return float(np.max(num / den)) if len(num) else 0.0


QUANTITIES = {"x": slice(0, 3), "v": slice(3, 6), "F_P": slice(8, 17), "F_E": slice(17, 26)}


def errors(a: np.ndarray, b: np.ndarray) -> dict:
    """Per-quantity relative error of records a against reference records b."""
    return {k: rel_err(a[:, s], b[:, s]) for k, s in QUANTITIES.items()}
