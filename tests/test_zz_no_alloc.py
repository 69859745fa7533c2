"""The allocation-free conservation sums (aero_lbm_b200_conservation_sums_noalloc).

Callers that cannot allocate device memory (a real-time tick thread, a fixed
device-memory budget) use this entry point; its scratch is a static device
array of fixed size. It must give the same sums as the allocating entry point
(same FP64 quantities, summed in a different order: relative difference
<= 1e-12), on two calls in a row (the static array keeps the previous call's
contents), and reject contexts larger than 128^3 cells. This file is collected
last so that a failure here leaves every other test already run."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import aero_b200
import lbm_cases
import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _noalloc(lib, key) -> np.ndarray:
    out = np.full(4, np.nan, dtype=np.float64)
    ok = lib.aero_lbm_b200_conservation_sums_noalloc(key, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert ok == 1, aero_b200.last_error(lib)
    return out


def _case(n=20, seed=17):
    rng = np.random.default_rng(seed)
    obst = (rng.random((n, n, n)) < 0.07).astype(np.uint8)
    u = [np.float32(0.04) + rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32),
         rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32),
         rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32)]
    return obst, u


@pytest.mark.parametrize("faces,solver_mode", [
    ([O.PERIODIC] * 4 + [O.BOUNCE_BACK] * 2, 0),                                    # in-place FP32
    ([O.PERIODIC] * 4 + [O.BOUNCE_BACK] * 2, 3),                                    # in-place FP16
    ([O.VELOCITY, O.CONVECTIVE] + [O.SYMMETRY] * 4, 0),                             # two-buffer FP32
])
def test_noalloc_matches_allocating_sums_twice(gpu, faces, solver_mode):
    obst, u = _case()
    n = obst.shape[0]
    faces = [dict(kind=k, velocity=(0.04, 0.0, 0.0)) if k == O.VELOCITY else dict(kind=k) for k in faces]
    cfg = {"reynolds": 60.0, "initial_velocity": (0.04, 0.0, 0.0), "faces": faces, "sgs": True, "buoyancy": False}
    gpu.aero_lbm_set_realtime_solver_mode(solver_mode)
    try:
        _, ctx = lbm_cases.run_product(gpu, (n, n, n), cfg, O.packet_from(obst, *u), 12, key=501)
    finally:
        gpu.aero_lbm_set_realtime_solver_mode(0)
    for call in range(2):
        want = ctx.conservation_sums()
        got = _noalloc(gpu, ctx.key)
        assert np.all(np.isfinite(got))
        assert abs(got[0] - want[0]) <= TOL * abs(want[0]), (call, got, want)
        assert np.max(np.abs(got[1:] - want[1:])) <= TOL * abs(want[0]), (call, got, want)
        ctx.advance(3)  # the second call sees a different state


def test_noalloc_rejects_bricks_beyond_the_static_scratch(gpu):
    dims = (130, 128, 128)  # 2,129,920 cells > 128^3
    obst = np.zeros(dims, np.uint8)
    zero = np.zeros(dims, np.float32)
    cfg = {"reynolds": 60.0, "faces": [dict(kind=O.PERIODIC)] * 6, "sgs": False, "buoyancy": False}
    _, ctx = lbm_cases.run_product(gpu, dims, cfg, O.packet_from(obst, zero, zero, zero), 1, key=503)
    out = np.zeros(4, np.float64)
    assert gpu.aero_lbm_b200_conservation_sums_noalloc(ctx.key, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
    assert "2097152" in aero_b200.last_error(gpu)
    ctx.release()
