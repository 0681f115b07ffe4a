"""Python access to the B200 snow step through its C ABI (include/snow_gpu.h).

This module is a thin ctypes binding: every computation runs in the CUDA
library ``libsnow_b200.so`` built beside this package (``make`` in the package
directory).  If that library is missing, importing :func:`lib` raises; there is
no CPU fallback.

Particle sets are ``(n, 26)`` float64 arrays of particle records in the order
of the reference's ``struct Particle``: x_p[3], v_p[3], m_p, V_p0, F_P[9],
F_E[9] (matrices column-major), see :mod:`snow_b200.scenes`.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("SNOW_B200_LIB") or os.path.join(PKG_DIR, "libsnow_b200.so")

SNOW_FP64, SNOW_MIXED = 0, 1
SNOW_COLLIDER_PLANE, SNOW_COLLIDER_SPHERE, SNOW_COLLIDER_BOX = 0, 1, 2
SNOW_PEAK_FP64, SNOW_PEAK_FP32, SNOW_PEAK_FP32X2 = 0, 1, 2
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "grid capacity exceeded",
          -4: "non-finite particle state", -5: "key range exceeded", -6: "invalid state"}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)


class Collider(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("point", ctypes.c_double * 3), ("normal", ctypes.c_double * 3),
                ("velocity", ctypes.c_double * 3), ("friction", ctypes.c_double),
                ("param", ctypes.c_double * 2), ("axis", ctypes.c_double * 3), ("extent", ctypes.c_double * 3)]


class StepParams(ctypes.Structure):
    _fields_ = [("gravity", ctypes.c_double * 3), ("time_step", ctypes.c_double),
                ("grid_spacing", ctypes.c_double), ("mu_0", ctypes.c_double),
                ("lambda_0", ctypes.c_double), ("hardening_coefficient", ctypes.c_double),
                ("max_compression", ctypes.c_double), ("max_stretch", ctypes.c_double),
                ("alpha", ctypes.c_double)]

    @classmethod
    def from_array(cls, a) -> "StepParams":
        """From the 11-value layout gravity[3], dt, dx, mu0, lambda0, xi, theta_c, theta_s, alpha."""
        a = [float(x) for x in a]
        p = cls()
        p.gravity[:] = a[0:3]
        (p.time_step, p.grid_spacing, p.mu_0, p.lambda_0, p.hardening_coefficient,
         p.max_compression, p.max_stretch, p.alpha) = a[3:11]
        return p


class StepTimings(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "stencil", "p2g", "forces_constitutive", "forces_accumulative", "grid_velocity",
        "grid_collisions", "stress_update", "g2p", "particle_collisions", "position_update")]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class ServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("completed", "rejected", "peak_scenes", "peak_bytes", "ticks",
                                               "particle_steps")] + \
               [(n, ctypes.c_double) for n in ("wall_s", "p50_s", "p99_s", "mean_s", "particle_steps_per_s",
                                                "admit_s", "step_s", "retire_s")] + \
               [("reservations", ctypes.c_int64)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class ServerTick(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("host_start_s", "host_end_s", "device_start_s", "device_end_s")] + \
               [(n, ctypes.c_int64) for n in ("steps", "scenes", "particles", "admitted", "retired")]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class SnowError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_LIB = None


def lib() -> ctypes.CDLL:
    """Loads libsnow_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make` in {PKG_DIR}")
    L = ctypes.CDLL(LIB_PATH)
    vp, i32, i64, d = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    sig = {
        "snow_gpu_init": (ctypes.c_int, [ctypes.c_int]),
        "snow_gpu_last_error": (ctypes.c_char_p, []),
        "snow_gpu_abi_version": (ctypes.c_int, []),
        "snow_gpu_make_plane": (ctypes.c_int, [_dp, _dp, d, ctypes.POINTER(Collider)]),
        "snow_gpu_batch_create": (ctypes.c_int, [ctypes.POINTER(vp), ctypes.c_int]),
        "snow_gpu_batch_destroy": (ctypes.c_int, [vp]),
        "snow_gpu_batch_add_scene": (ctypes.c_int, [vp, _dp, i64, ctypes.POINTER(StepParams),
                                                    ctypes.POINTER(Collider), ctypes.c_int, _ip, vp]),
        "snow_gpu_batch_remove_scene": (ctypes.c_int, [vp, i32]),
        "snow_gpu_batch_set_params": (ctypes.c_int, [vp, i32, ctypes.POINTER(StepParams),
                                                     ctypes.POINTER(Collider), ctypes.c_int]),
        "snow_gpu_batch_upload": (ctypes.c_int, [vp, i32, _dp, i64, vp]),
        "snow_gpu_batch_download": (ctypes.c_int, [vp, i32, _dp, i64, vp]),
        "snow_gpu_batch_download_positions": (ctypes.c_int, [vp, i32, _dp, i64, vp]),
        "snow_gpu_stage_weights": (ctypes.c_int, [_dp, i64, ctypes.c_double, ctypes.c_int, _ip, _dp, _dp]),
        "snow_gpu_batch_setup": (ctypes.c_int, [vp, i32, d, vp]),
        "snow_gpu_batch_step": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(StepTimings), vp]),
        "snow_gpu_batch_scene_count": (ctypes.c_int, [vp]),
        "snow_gpu_batch_particles": (i64, [vp]),
        "snow_gpu_batch_device_bytes": (i64, [vp]),
        "snow_gpu_batch_status": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_uint32), _i64p, _i64p]),
        "snow_gpu_batch_set_graphs": (ctypes.c_int, [vp, ctypes.c_int]),
        "snow_gpu_batch_fp64_projections": (i64, [vp]),
        "snow_gpu_batch_autotune": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                   _dp, vp]),
        "snow_gpu_server_create": (ctypes.c_int, [ctypes.POINTER(vp), ctypes.c_int, i64, ctypes.c_int,
                                                  ctypes.c_int]),
        "snow_gpu_server_destroy": (ctypes.c_int, [vp]),
        "snow_gpu_server_submit": (ctypes.c_int, [vp, _dp, i64, ctypes.POINTER(StepParams),
                                                  ctypes.POINTER(Collider), ctypes.c_int, i64, d, _i64p]),
        "snow_gpu_server_run": (ctypes.c_int, [vp, vp]),
        "snow_gpu_server_result": (ctypes.c_int, [vp, i64, _dp, i64, _dp]),
        "snow_gpu_server_stats": (ctypes.c_int, [vp, ctypes.POINTER(ServerStats)]),
        "snow_gpu_server_ticks": (ctypes.c_int, [vp, ctypes.POINTER(ServerTick), i64, _i64p]),
        "snow_gpu_server_set_work_item": (ctypes.c_int, [vp, ctypes.c_int]),
        "snow_gpu_server_set_streaming": (ctypes.c_int, [vp, ctypes.c_int]),
        "snow_gpu_server_close": (ctypes.c_int, [vp]),
        "snow_gpu_batch_set_chunk": (ctypes.c_int, [vp, ctypes.c_int]),
        "snow_gpu_batch_set_dense": (ctypes.c_int, [vp, ctypes.c_int]),
        "snow_gpu_batch_chunk": (ctypes.c_int, [vp]),
        "snow_gpu_batch_graph_kernels": (ctypes.c_int, [vp]),
        "snow_gpu_batch_sort_mode": (ctypes.c_int, [vp]),
        "snow_gpu_measure_fma_peak": (ctypes.c_int, [ctypes.c_int, _dp, _dp, vp]),
        "snow_gpu_batch_set_implicit": (ctypes.c_int, [vp, d, d, ctypes.c_int]),
        "snow_gpu_batch_implicit_stats": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int), _dp]),
        "snow_gpu_stage_constitutive_differential": (ctypes.c_int, [_dp, i64, _dp, d, d, d, _dp]),
        "snow_gpu_stage_deformation_differential": (ctypes.c_int, [_dp, i64, d, _dp, _dp, _dp]),
        "snow_gpu_stage_implicit": (ctypes.c_int, [_ip, _dp, i64, _dp, i64, d, d, d, d, d, d, d, ctypes.c_int,
                                                   _dp, _dp, ctypes.POINTER(ctypes.c_int)]),
        "snow_gpu_batch_snapshot": (ctypes.c_int, [vp, ctypes.c_int32, vp]),
        "snow_gpu_batch_restore": (ctypes.c_int, [vp, ctypes.c_int32, vp]),
        "snow_gpu_setup": (ctypes.c_int, [_dp, i64, d]),
        "snow_gpu_step": (ctypes.c_int, [_dp, i64, ctypes.POINTER(StepParams), ctypes.POINTER(Collider),
                                         ctypes.c_int, ctypes.c_int, ctypes.POINTER(StepTimings)]),
        "snow_gpu_step_noalloc": (ctypes.c_int, [_dp, i64, ctypes.POINTER(StepParams), ctypes.POINTER(Collider),
                                                 ctypes.c_int, ctypes.c_int, vp]),
        "snow_gpu_stage_p2g": (ctypes.c_int, [_dp, i64, d, _ip, _dp, i64, _i64p]),
        "snow_gpu_stage_force": (ctypes.c_int, [_dp, i64, d, d, d, d, _ip, _dp, i64, _i64p]),
        "snow_gpu_stage_p2g_stencil": (ctypes.c_int, [_dp, i64, _dp, _dp]),
        "snow_gpu_stage_stress": (ctypes.c_int, [_dp, i64, d, d, d, _dp]),
        "snow_gpu_stage_force_scatter": (ctypes.c_int, [_dp, i64, _dp, _dp, _dp]),
        "snow_gpu_stage_grid_velocity": (ctypes.c_int, [_dp, i64, _dp, d]),
        "snow_gpu_stage_grid_collisions": (ctypes.c_int, [_ip, _dp, i64, ctypes.POINTER(Collider),
                                                          ctypes.c_int, d]),
        "snow_gpu_stage_volume": (ctypes.c_int, [_ip, _dp, i64, _dp, i64, d]),
        "snow_gpu_stage_stress_update": (ctypes.c_int, [_ip, _dp, i64, _dp, i64, d, d, d, d]),
        "snow_gpu_stage_g2p": (ctypes.c_int, [_ip, _dp, i64, _dp, i64, d, d]),
        "snow_gpu_stage_particle_collisions": (ctypes.c_int, [_dp, i64, ctypes.POINTER(Collider),
                                                              ctypes.c_int]),
        "snow_gpu_stage_position_update": (ctypes.c_int, [_dp, i64, d]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype, f.argtypes = res, args
    _LIB = L
    return L


def exported_symbols() -> list[str]:
    """Every C ABI entry point this binding expects the library to export."""
    return [n for n in dir(lib()) if n.startswith("snow_gpu_")] if _LIB else []


def _check(rc: int) -> None:
    if rc != 0:
        raise SnowError(rc, lib().snow_gpu_last_error().decode())


def _ptr(a: np.ndarray, t=_dp):
    return a.ctypes.data_as(t)


def _records(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.ndim != 2 or a.shape[1] != 26:
        raise ValueError("particle records must be an (n, 26) float64 array")
    return a


def init(device: int = 0) -> None:
    _check(lib().snow_gpu_init(device))


def make_plane(point, normal, friction: float) -> Collider:
    """make_plane (reference src/collision.cpp:5): unit normal, zero velocity."""
    c = Collider()
    p = np.asarray(point, dtype=np.float64)
    n = np.asarray(normal, dtype=np.float64)
    _check(lib().snow_gpu_make_plane(_ptr(p), _ptr(n), float(friction), ctypes.byref(c)))
    return c


def sphere(center, radius: float, friction: float, velocity=(0.0, 0.0, 0.0)) -> "Collider":
    """A solid sphere collider (phi = |x - center| - radius), moving with `velocity`."""
    c = Collider()
    c.kind = SNOW_COLLIDER_SPHERE
    for a in range(3):
        c.point[a] = float(center[a])
        c.velocity[a] = float(velocity[a])
    c.friction = float(friction)
    c.param[0] = float(radius)
    return c


def moving_plane(point, normal, friction: float, velocity) -> "Collider":
    """make_plane with a constant velocity."""
    c = make_plane(point, normal, friction)
    for a in range(3):
        c.velocity[a] = float(velocity[a])
    return c


def box(center, half_extents, axis_u, axis_w, friction: float, velocity=(0.0, 0.0, 0.0)) -> "Collider":
    """A solid oriented box collider: centre, half extents along the axes u, w and
    u x w (u and w are normalised and w made orthogonal to u), moving with `velocity`."""
    u = np.asarray(axis_u, dtype=np.float64)
    u = u / np.linalg.norm(u)
    w = np.asarray(axis_w, dtype=np.float64)
    w = w - u.dot(w) * u
    w = w / np.linalg.norm(w)
    c = Collider()
    c.kind = SNOW_COLLIDER_BOX
    for a in range(3):
        c.point[a] = float(center[a])
        c.normal[a] = float(u[a])
        c.axis[a] = float(w[a])
        c.extent[a] = float(half_extents[a])
        c.velocity[a] = float(velocity[a])
    c.friction = float(friction)
    return c


BODY_COLUMNS = 18


def body_rows(cols) -> np.ndarray:
    """(k, 18) rows (kind, point[3], normal[3], velocity[3], friction, radius, axis[3],
    extent[3]) of Collider values, the form the oracle and the reference build take."""
    out = np.zeros((len(cols), BODY_COLUMNS))
    for i, c in enumerate(cols):
        out[i] = [c.kind, *c.point, *c.normal, *c.velocity, c.friction, c.param[0], *c.axis, *c.extent]
    return out


def colliders(planes) -> ctypes.Array:
    """A ctypes array of colliders from (point, normal, friction) plane triples,
    Collider values (see sphere, moving_plane), or a (k, 7) array of point[3],
    normal[3], friction plane rows."""
    if isinstance(planes, np.ndarray):
        planes = [(r[:3], r[3:6], r[6]) for r in planes.reshape(-1, 7)]
    arr = (Collider * max(1, len(planes)))()
    for i, item in enumerate(planes):
        arr[i] = item if isinstance(item, Collider) else make_plane(*item)
    return arr


class Batch:
    """A batch of independent scenes advanced together (snow_gpu_batch_*)."""

    def __init__(self, precision: int = SNOW_FP64):
        self._h = ctypes.c_void_p()
        _check(lib().snow_gpu_batch_create(ctypes.byref(self._h), precision))
        self.sizes: dict[int, int] = {}

    def close(self) -> None:
        if self._h:
            lib().snow_gpu_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, records: np.ndarray, params, planes=(), stream: int | None = None) -> int:
        rec = _records(records)
        prm = params if isinstance(params, StepParams) else StepParams.from_array(params)
        col = colliders(planes) if len(planes) else (Collider * 1)()
        sid = ctypes.c_int32()
        _check(lib().snow_gpu_batch_add_scene(self._h, _ptr(rec), rec.shape[0], ctypes.byref(prm),
                                              col, len(planes), ctypes.byref(sid),
                                              ctypes.c_void_p(stream)))
        self.sizes[sid.value] = rec.shape[0]
        return sid.value

    def add(self, scene, stream: int | None = None) -> int:
        """Adds a :class:`snow_b200.scenes.Scene`."""
        return self.add_scene(scene.particles, scene.params(), scene.planes, stream)

    def remove_scene(self, sid: int) -> None:
        _check(lib().snow_gpu_batch_remove_scene(self._h, sid))
        self.sizes.pop(sid, None)

    def set_params(self, sid: int, params, planes=()) -> None:
        prm = params if isinstance(params, StepParams) else StepParams.from_array(params)
        col = colliders(planes) if len(planes) else (Collider * 1)()
        _check(lib().snow_gpu_batch_set_params(self._h, sid, ctypes.byref(prm), col, len(planes)))

    def upload(self, sid: int, records: np.ndarray, stream: int | None = None) -> None:
        rec = _records(records)
        _check(lib().snow_gpu_batch_upload(self._h, sid, _ptr(rec), rec.shape[0], ctypes.c_void_p(stream)))

    def download(self, sid: int, out: np.ndarray | None = None, stream: int | None = None) -> np.ndarray:
        n = self.sizes[sid]
        if out is None:
            out = np.empty((n, 26), dtype=np.float64)
        _check(lib().snow_gpu_batch_download(self._h, sid, _ptr(out), n, ctypes.c_void_p(stream)))
        return out

    def download_positions(self, sid: int) -> np.ndarray:
        """Particle positions (n x 3) in their original order (snow_gpu_batch_download_positions)."""
        n = self.sizes[sid]
        out = np.empty((n, 3))
        _check(lib().snow_gpu_batch_download_positions(self._h, sid, _ptr(out), n, None))
        return out

    def snapshot(self, sid: int, stream: int | None = None) -> None:
        """Keeps a device copy of the scene's particle state."""
        _check(lib().snow_gpu_batch_snapshot(self._h, sid, ctypes.c_void_p(stream)))

    def restore(self, sid: int, stream: int | None = None) -> None:
        """Puts the scene back to its last snapshot."""
        _check(lib().snow_gpu_batch_restore(self._h, sid, ctypes.c_void_p(stream)))

    def setup(self, sid: int, dx: float, stream: int | None = None) -> None:
        _check(lib().snow_gpu_batch_setup(self._h, sid, float(dx), ctypes.c_void_p(stream)))

    def step(self, n_steps: int = 1, timings: bool = False, stream: int | None = None):
        t = StepTimings() if timings else None
        _check(lib().snow_gpu_batch_step(self._h, int(n_steps), ctypes.byref(t) if t else None,
                                         ctypes.c_void_p(stream)))
        return t.as_dict() if t else None

    def set_graphs(self, enable: bool) -> None:
        _check(lib().snow_gpu_batch_set_graphs(self._h, int(bool(enable))))

    def sort_mode(self) -> str:
        """Particle ordering in use: "dense" (counting sort over key bins) or "radix"."""
        return "dense" if lib().snow_gpu_batch_sort_mode(self._h) == 1 else "radix"

    def graph_kernels(self) -> int:
        """Kernel launches in one replay of the captured step graph (0 before capture)."""
        return int(lib().snow_gpu_batch_graph_kernels(self._h))

    def set_dense(self, enable: bool) -> None:
        """Counting sort over dense key bins (default) or the radix sort with the block hash table."""
        _check(lib().snow_gpu_batch_set_dense(self._h, int(bool(enable))))

    def chunk(self) -> int:
        """Particles per work item of the last (or next) step."""
        c = lib().snow_gpu_batch_chunk(self._h)
        if c < 0:
            _check(c)
        return c

    def set_chunk(self, chunk: int) -> None:
        """Particles per P2G/G2P work item (power of two, 32..1024)."""
        _check(lib().snow_gpu_batch_set_chunk(self._h, int(chunk)))

    def autotune(self, trial_steps: int = 10, stream: int | None = None) -> tuple[int, float]:
        """Picks the fastest work-item size on a snapshot of the state; returns (size, ms/step)."""
        c, ms = ctypes.c_int(), ctypes.c_double()
        _check(lib().snow_gpu_batch_autotune(self._h, int(trial_steps), ctypes.byref(c), ctypes.byref(ms),
                                             ctypes.c_void_p(stream)))
        return c.value, ms.value

    def set_implicit(self, beta: float, tolerance: float = 1e-10, max_iterations: int = 100) -> None:
        """Semi-implicit velocity update (beta = 0: the explicit step)."""
        _check(lib().snow_gpu_batch_set_implicit(self._h, float(beta), float(tolerance), int(max_iterations)))

    def implicit_stats(self) -> tuple[int, float]:
        """(iterations, relative residual) of the last step's implicit solve."""
        it, res = ctypes.c_int(), ctypes.c_double()
        _check(lib().snow_gpu_batch_implicit_stats(self._h, ctypes.byref(it), ctypes.byref(res)))
        return it.value, res.value

    @property
    def fp64_projections(self) -> int:
        """Mixed form: projections redone in double during the last step."""
        return int(lib().snow_gpu_batch_fp64_projections(self._h))

    def status(self) -> tuple[int, int, int]:
        st, used, cap = ctypes.c_uint32(), ctypes.c_int64(), ctypes.c_int64()
        _check(lib().snow_gpu_batch_status(self._h, ctypes.byref(st), ctypes.byref(used), ctypes.byref(cap)))
        return st.value, used.value, cap.value

    @property
    def particles(self) -> int:
        return int(lib().snow_gpu_batch_particles(self._h))

    @property
    def device_bytes(self) -> int:
        return int(lib().snow_gpu_batch_device_bytes(self._h))


def measure_fma_peak(kind: int, stream: int | None = None) -> float:
    """Measured FMA throughput of the current device in FLOP/s (SNOW_PEAK_*)."""
    f, ms = ctypes.c_double(), ctypes.c_double()
    _check(lib().snow_gpu_measure_fma_peak(int(kind), ctypes.byref(f), ctypes.byref(ms), ctypes.c_void_p(stream)))
    return f.value


def setup(records: np.ndarray, dx: float) -> np.ndarray:
    """setup() (reference src/grid.cpp:340) in place on host records; returns them."""
    rec = _records(records)
    _check(lib().snow_gpu_setup(_ptr(rec), rec.shape[0], float(dx)))
    if rec is not records:
        records[...] = rec
    return records


def step(records: np.ndarray, params, planes=(), n_steps: int = 1, timings: bool = False):
    """n_steps of step() (reference src/grid.cpp:359) in place on host records."""
    rec = _records(records)
    prm = params if isinstance(params, StepParams) else StepParams.from_array(params)
    col = colliders(planes) if len(planes) else (Collider * 1)()
    t = StepTimings() if timings else None
    _check(lib().snow_gpu_step(_ptr(rec), rec.shape[0], ctypes.byref(prm), col, len(planes),
                               int(n_steps), ctypes.byref(t) if t else None))
    if rec is not records:
        records[...] = rec
    return t.as_dict() if t else None


# ---------------------------------------------------------------- stages
NODE_FIELDS = 10  # mass, momentum[3], velocity[3], force[3]


def _nodes_out(n_particles: int):
    cap = max(64, n_particles * 512)
    return np.empty((cap, 3), np.int32), np.empty((cap, NODE_FIELDS)), ctypes.c_int64()


def stage_p2g(records: np.ndarray, dx: float):
    """Mass and momentum contributions of the particles on an empty grid: (ijk, fields)."""
    rec = _records(records)
    ijk, f, nn = _nodes_out(rec.shape[0])
    _check(lib().snow_gpu_stage_p2g(_ptr(rec), rec.shape[0], float(dx), _ptr(ijk, _ip), _ptr(f),
                                    ijk.shape[0], ctypes.byref(nn)))
    return ijk[:nn.value], f[:nn.value]


def stage_force(records: np.ndarray, dx: float, mu0: float, lambda0: float, xi: float):
    rec = _records(records)
    ijk, f, nn = _nodes_out(rec.shape[0])
    _check(lib().snow_gpu_stage_force(_ptr(rec), rec.shape[0], float(dx), float(mu0), float(lambda0),
                                      float(xi), _ptr(ijk, _ip), _ptr(f), ijk.shape[0], ctypes.byref(nn)))
    return ijk[:nn.value], f[:nn.value]


def _nodes_in(ijk, fields):
    ijk = np.ascontiguousarray(ijk, dtype=np.int32).reshape(-1, 3)
    fields = np.ascontiguousarray(fields, dtype=np.float64).reshape(-1, NODE_FIELDS)
    return ijk, fields


def stage_grid_velocity(fields: np.ndarray, gravity, dt: float) -> np.ndarray:
    f = np.array(fields, dtype=np.float64, order="C").reshape(-1, NODE_FIELDS)
    g = np.asarray(gravity, dtype=np.float64)
    _check(lib().snow_gpu_stage_grid_velocity(_ptr(f), f.shape[0], _ptr(g), float(dt)))
    return f


def stage_grid_collisions(ijk, fields, planes, dx: float) -> np.ndarray:
    ijk, _ = _nodes_in(ijk, fields)
    f = np.array(fields, dtype=np.float64, order="C").reshape(-1, NODE_FIELDS)
    col = colliders(planes)
    _check(lib().snow_gpu_stage_grid_collisions(_ptr(ijk, _ip), _ptr(f), f.shape[0], col, len(planes), float(dx)))
    return f


def stage_volume(ijk, fields, records, dx: float) -> np.ndarray:
    ijk, fields = _nodes_in(ijk, fields)
    rec = np.array(records, dtype=np.float64, order="C")
    _check(lib().snow_gpu_stage_volume(_ptr(ijk, _ip), _ptr(fields), ijk.shape[0], _ptr(rec), rec.shape[0], float(dx)))
    return rec


def stage_stress_update(ijk, fields, records, dx, dt, theta_c, theta_s) -> np.ndarray:
    ijk, fields = _nodes_in(ijk, fields)
    rec = np.array(records, dtype=np.float64, order="C")
    _check(lib().snow_gpu_stage_stress_update(_ptr(ijk, _ip), _ptr(fields), ijk.shape[0], _ptr(rec),
                                              rec.shape[0], float(dx), float(dt), float(theta_c), float(theta_s)))
    return rec


def stage_g2p(ijk, fields, records, dx, alpha) -> np.ndarray:
    ijk, fields = _nodes_in(ijk, fields)
    rec = np.array(records, dtype=np.float64, order="C")
    _check(lib().snow_gpu_stage_g2p(_ptr(ijk, _ip), _ptr(fields), ijk.shape[0], _ptr(rec), rec.shape[0],
                                    float(dx), float(alpha)))
    return rec


def stage_particle_collisions(records, planes) -> np.ndarray:
    rec = np.array(records, dtype=np.float64, order="C")
    col = colliders(planes)
    _check(lib().snow_gpu_stage_particle_collisions(_ptr(rec), rec.shape[0], col, len(planes)))
    return rec


def stage_constitutive_differential(records, dF, mu0, lambda0, xi) -> np.ndarray:
    """dP[n][3][3] for dF[n][3][3] (row-major numpy matrices)."""
    rec = _records(records)
    dfc = np.ascontiguousarray(np.transpose(np.asarray(dF, dtype=np.float64), (0, 2, 1)).reshape(-1, 9))
    out = np.zeros_like(dfc)
    _check(lib().snow_gpu_stage_constitutive_differential(_ptr(rec), rec.shape[0], _ptr(dfc), float(mu0),
                                                          float(lambda0), float(xi), _ptr(out)))
    return np.transpose(out.reshape(-1, 3, 3), (0, 2, 1))


def stage_implicit(ijk, fields, records, dx, dt, mu0, lambda0, xi, beta, q=None, squared_tolerance=1e-24,
                   max_iterations=300):
    """A q (q given) or the conjugate-residual solution (q None) on a node list;
    returns (n_nodes x 3 values, iterations)."""
    ijk = np.ascontiguousarray(ijk, dtype=np.int32).reshape(-1, 3)
    f = np.ascontiguousarray(fields, dtype=np.float64).reshape(-1, 10)
    rec = _records(records)
    qq = None if q is None else np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 3)
    out = np.zeros((ijk.shape[0], 3))
    it = ctypes.c_int()
    _check(lib().snow_gpu_stage_implicit(_ptr(ijk, _ip), _ptr(f), ijk.shape[0], _ptr(rec), rec.shape[0], float(dx),
                                         float(dt), float(mu0), float(lambda0), float(xi), float(beta),
                                         float(squared_tolerance), int(max_iterations),
                                         None if qq is None else _ptr(qq), _ptr(out), ctypes.byref(it)))
    return out, it.value


def stage_weights(x, dx, precision: int = 0):
    """The device stencil weights along one axis: (base[n], w[n][4], dw[n][4])."""
    xs = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    n = xs.shape[0]
    base = np.zeros(n, np.int32)
    w = np.zeros((n, 4))
    dw = np.zeros((n, 4))
    _check(lib().snow_gpu_stage_weights(_ptr(xs), n, float(dx), int(precision), _ptr(base, _ip), _ptr(w), _ptr(dw)))
    return base, w, dw


def stage_position_update(records, dt) -> np.ndarray:
    rec = np.array(records, dtype=np.float64, order="C")
    _check(lib().snow_gpu_stage_position_update(_ptr(rec), rec.shape[0], float(dt)))
    return rec


class Server:
    """Continuous-batching server of independent scenes (snow_gpu_server_*)."""

    def __init__(self, precision: int = SNOW_FP64, budget_bytes: int = 150 * 10**9, max_scenes: int = 4096,
                 max_steps_per_tick: int = 16, work_item: int = 0):
        self._h = ctypes.c_void_p()
        _check(lib().snow_gpu_server_create(ctypes.byref(self._h), precision, int(budget_bytes), int(max_scenes),
                                            int(max_steps_per_tick)))
        if work_item:
            _check(lib().snow_gpu_server_set_work_item(self._h, int(work_item)))
        self.sizes: dict[int, int] = {}

    def close(self) -> None:
        if self._h:
            lib().snow_gpu_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_streaming(self, on: bool = True) -> None:
        """run() waits for further submissions until end_of_stream()."""
        _check(lib().snow_gpu_server_set_streaming(self._h, int(bool(on))))

    def end_of_stream(self) -> None:
        """No more submissions (snow_gpu_server_close): run() returns once all are done."""
        _check(lib().snow_gpu_server_close(self._h))

    def done(self, rid: int) -> bool:
        """True once request `rid` is complete (its result can be read)."""
        out = np.empty((self.sizes[rid], 26))
        rc = lib().snow_gpu_server_result(self._h, rid, _ptr(out), out.shape[0], None)
        if rc == -6:  # SNOW_E_STATE: not complete yet
            return False
        _check(rc)
        return True

    def submit(self, scene, steps: int, arrival_s: float = -1.0) -> int:
        """Queues a request; arrival_s < 0 stamps it with the current server time.
        Thread-safe: may be called while run() loops on another thread."""
        rec = _records(scene.particles)
        prm = StepParams.from_array(scene.params())
        col = colliders(scene.planes) if len(scene.planes) else (Collider * 1)()
        rid = ctypes.c_int64()
        _check(lib().snow_gpu_server_submit(self._h, _ptr(rec), rec.shape[0], ctypes.byref(prm), col,
                                            len(scene.planes), int(steps), float(arrival_s), ctypes.byref(rid)))
        self.sizes[rid.value] = rec.shape[0]
        return rid.value

    def run(self, stream: int | None = None) -> None:
        _check(lib().snow_gpu_server_run(self._h, ctypes.c_void_p(stream)))

    def result(self, rid: int) -> tuple[np.ndarray, float]:
        out = np.empty((self.sizes[rid], 26))
        lat = ctypes.c_double()
        _check(lib().snow_gpu_server_result(self._h, rid, _ptr(out), out.shape[0], ctypes.byref(lat)))
        return out, lat.value

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().snow_gpu_server_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def ticks(self) -> list[dict]:
        """Per-tick trace of the last run() (snow_gpu_server_ticks)."""
        n = ctypes.c_int64()
        _check(lib().snow_gpu_server_ticks(self._h, None, 0, ctypes.byref(n)))
        buf = (ServerTick * max(1, n.value))()
        _check(lib().snow_gpu_server_ticks(self._h, buf, n.value, ctypes.byref(n)))
        return [buf[i].as_dict() for i in range(n.value)]
