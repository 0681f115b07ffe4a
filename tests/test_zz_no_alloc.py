"""snow_gpu_step_noalloc: the step for callers that cannot allocate device memory.

Some hosts of this solver may not call cudaMalloc themselves -- a plugin inside
an application that owns the GPU memory pool, or a loop that cannot take an
allocation's implicit synchronisation.  snow_gpu_step_noalloc serves them with
all device scratch in one fixed file-scope device array.  This test drives it
through the C ABI and checks it against the ordinary entry point snow_gpu_step
on the same host records, for two calls in a row (the second call continues
from the first call's output, so leftovers in the shared array would show).
Tolerance: 1e-10 relative per quantity, as for every FP64 parity test.

The file name sorts last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

from oracle_lib import errors

pytestmark = pytest.mark.gpu

TOL = 1e-10
MAX_PARTICLES = 16384


def _noalloc(snow, rec, params, planes, steps):
    out = np.ascontiguousarray(rec, dtype=np.float64).copy()
    prm = snow.StepParams.from_array(params)
    col = snow.colliders(planes)
    rc = snow.lib().snow_gpu_step_noalloc(out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.shape[0],
                                          ctypes.byref(prm), col, len(planes), steps, None)
    return rc, out


@pytest.mark.parametrize("steps", [6, 5])
def test_noalloc_matches_step_on_two_calls(snow, steps):
    """Even and odd step counts per call (the result lies in the buffer the
    last step wrote, which alternates)."""
    from snow_b200 import scenes

    sc = scenes.cube_scene(16)  # 4,096 particles falling onto the ground plane
    sc.particles[:, 1] -= 0.448  # start just above the ground plane: collisions act in both calls
    start = snow.setup(sc.particles.copy(), sc.dx)
    ref = start.copy()
    cur = start.copy()
    for call in range(2):
        snow.step(ref, sc.params(), sc.planes, steps)
        rc, cur = _noalloc(snow, cur, sc.params(), sc.planes, steps)
        assert rc == 0, snow.lib().snow_gpu_last_error().decode()
        e = errors(cur, ref)
        assert max(e.values()) < TOL, (call, e)


def test_noalloc_setup_call_with_no_particles(snow):
    """n = 0 only does the per-device set-up and succeeds."""
    from snow_b200 import scenes

    sc = scenes.cube_scene(4)
    rc, _ = _noalloc(snow, np.zeros((0, 26)), sc.params(), sc.planes, 1)
    assert rc == 0, snow.lib().snow_gpu_last_error().decode()


def test_noalloc_capacity_error_leaves_records_unchanged(snow):
    """A sparse scene whose particles each need their own grid blocks: 1,000
    particles 0.1 m apart need far more than the 2,048 blocks the fixed array
    holds.  The call reports SNOW_E_CAPACITY and leaves the records alone."""
    from snow_b200 import scenes

    g = (np.arange(10) + 0.5) * 0.1
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    rec = scenes.records(x, np.zeros_like(x), 0.001)
    rec[:, 7] = 1e-6
    sc = scenes.cube_scene(4)
    before = rec.copy()
    rc, out = _noalloc(snow, rec, sc.params(), [], 1)
    assert rc == -3, (rc, snow.lib().snow_gpu_last_error().decode())
    assert "2048" in snow.lib().snow_gpu_last_error().decode()
    assert np.array_equal(out, before)


def test_noalloc_rejects_sizes_beyond_its_limit(snow):
    from snow_b200 import scenes

    rec = scenes.cube(26)[: MAX_PARTICLES + 1]
    sc = scenes.cube_scene(4)
    rc, _ = _noalloc(snow, rec, sc.params(), sc.planes, 1)
    assert rc == -1
    assert "16384" in snow.lib().snow_gpu_last_error().decode()
