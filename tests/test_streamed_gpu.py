"""The streamed in-place step (each warp's next 64-cell tile brought into
shared memory by bulk asynchronous copies while it collides the current one)
against the same step with per-thread loads: same arithmetic on the same
inputs, so the states agree bit for bit. Cases cover partial tiles (nz not a
multiple of 64, odd nz), periodic x / y lines, equilibrium and bounce-back
faces, buoyancy, a per-cell force field and mask changes between calls; the
FP32, IEEE-half and fixed-point storages."""
from __future__ import annotations

import numpy as np
import pytest

import aero_b200
import lbm_cases
import oracle as O

pytestmark = pytest.mark.gpu

STORAGES = {"fp32": (0, 1, 0), "fp16": (3, 0, 0), "i16": (3, 0, 1)}  # solver mode, collision mode, 16-bit format


def _case(dims, seed, periodic_x):
    rng = np.random.default_rng(seed)
    obst = (rng.random(dims) < 0.08).astype(np.uint8)
    u = [np.float32(0.05) + rng.uniform(-0.01, 0.01, dims).astype(np.float32),
         rng.uniform(-0.01, 0.01, dims).astype(np.float32), rng.uniform(-0.01, 0.01, dims).astype(np.float32)]
    temp = rng.uniform(-0.5, 0.5, dims).astype(np.float32)
    faces = [{"kind": O.PERIODIC}, {"kind": O.PERIODIC}] if periodic_x else \
        [{"kind": O.VELOCITY, "velocity": (0.05, 0.01, 0.0)}, {"kind": O.PRESSURE, "pressure": 0.001}]
    faces += [{"kind": O.PERIODIC}, {"kind": O.PERIODIC},
              {"kind": O.BOUNCE_BACK}, {"kind": O.MOVING_WALL, "velocity": (0.04, 0.0, 0.0)}]
    cfg = {"reynolds": 120.0, "initial_velocity": (0.05, 0.0, 0.0), "sgs": True, "buoyancy": True, "faces": faces}
    return obst, u, temp, cfg


def _run(gpu, storage, streamed, dims, seed, periodic_x, force, steps=24, key=300):
    obst, u, temp, cfg = _case(dims, seed, periodic_x)
    obst2 = obst.copy()
    rng = np.random.default_rng(seed + 1)
    obst2[(rng.random(dims) < 0.03) & (obst == 0)] = 1
    obst2[(rng.random(dims) < 0.5) & (obst == 1)] = 0
    pk1 = O.packet_from(obst, *u, temperature=temp)
    pk2 = O.packet_from(obst2, *u, temperature=temp)
    mode, collision, fmt = STORAGES[storage]
    gpu.aero_lbm_b200_set_physics_overrides(0.1, 1e-3, 2)
    gpu.aero_lbm_b200_set_streaming_mode(2 if storage == "fp32" else 0)
    gpu.aero_lbm_b200_set_collision_mode(collision)
    gpu.aero_lbm_set_realtime_solver_mode(mode)
    assert gpu.aero_lbm_b200_set_fp16_format(fmt) == 1
    assert gpu.aero_lbm_b200_set_streamed_step(int(streamed)) == 1
    try:
        ctx = aero_b200.LbmContext(dims, input_channels=pk1.shape[1], key=key + int(streamed), lib=gpu)
        ctx.configure(lbm_cases.product_config(gpu, cfg))
        ctx.step(pk1, output=False)
        if force:
            frng = np.random.default_rng(seed + 2)
            ctx.set_force_field(*(frng.uniform(-2e-5, 2e-5, dims).astype(np.float32) for _ in range(3)))
        out = None
        for s in range(1, steps):
            out = ctx.step(pk1 if s < 10 else pk2, output=(s + 1 == steps))
        state = ctx.flow_state().copy()
        ctx.release()
    finally:
        gpu.aero_lbm_b200_set_streamed_step(0)
        gpu.aero_lbm_set_realtime_solver_mode(0)
        gpu.aero_lbm_b200_set_collision_mode(0)
        gpu.aero_lbm_b200_set_fp16_format(1)
        gpu.aero_lbm_b200_set_physics_overrides(-1.0, -1.0, -1)
    return out, state


@pytest.mark.parametrize("storage", ["fp32", "fp16", "i16"])
@pytest.mark.parametrize("dims,periodic_x,force", [((12, 10, 70), False, True), ((9, 11, 13), True, False),
                                                   ((6, 5, 128), True, True)])
def test_streamed_step_matches_per_thread_loads(gpu, storage, dims, periodic_x, force):
    seed = sum(dims)
    out_s, st_s = _run(gpu, storage, True, dims, seed, periodic_x, force)
    out_p, st_p = _run(gpu, storage, False, dims, seed, periodic_x, force)
    assert np.all(np.isfinite(st_s))
    np.testing.assert_array_equal(st_s.view(np.uint32), st_p.view(np.uint32))
    np.testing.assert_array_equal(np.asarray(out_s, np.float32).view(np.uint32),
                                  np.asarray(out_p, np.float32).view(np.uint32))
