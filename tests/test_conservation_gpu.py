"""FP64 mass/momentum sums of the streamed state (warp-shuffle reduction with
per-block partials) against the oracle, and mass conservation of a closed
periodic brick over many steps."""
from __future__ import annotations

import numpy as np
import pytest

import lbm_cases
import oracle as O

pytestmark = pytest.mark.gpu


def periodic_case(n=16, seed=3):
    rng = np.random.default_rng(seed)
    obst = (rng.random((n, n, n)) < 0.06).astype(np.uint8)
    u = [np.float32(0.03) + rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32),
         rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32),
         rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32)]
    p = rng.uniform(-0.004, 0.004, (n, n, n)).astype(np.float32)
    cfg = {"reynolds": 50.0, "initial_velocity": (0.03, 0.0, 0.0), "faces": [{"kind": O.PERIODIC}] * 6,
           "sgs": True, "buoyancy": False}
    return obst, u, p, cfg


def oracle_sums(o: O.Oracle, obst) -> np.ndarray:
    m = o.macro()
    fluid = obst.reshape(-1) == 0
    rho = m[fluid, 0]
    return np.array([rho.sum(), (rho * m[fluid, 1]).sum(), (rho * m[fluid, 2]).sum(), (rho * m[fluid, 3]).sum()])


@pytest.mark.parametrize("streaming", [1, 2])
def test_sums_match_oracle(gpu, streaming):
    obst, u, p, cfg = periodic_case()
    n = obst.shape[0]
    out, ctx = lbm_cases.run_product(gpu, (n, n, n), cfg, O.packet_from(obst, *u, pressure=p), 25,
                                     streaming_mode=streaming)
    sums = ctx.conservation_sums()
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    o.set_fields(obst, *u, pressure=p)
    o.step(25)
    ref = oracle_sums(o, obst)
    assert abs(sums[0] - ref[0]) / ref[0] < 1e-9
    assert np.max(np.abs(sums[1:] - ref[1:])) / ref[0] < 1e-9


@pytest.mark.parametrize("solver_mode,fmt,tol", [(0, 0, 2e-6), (3, 0, 5e-5), (3, 1, 5e-5)])
def test_periodic_brick_conserves_mass(gpu, solver_mode, fmt, tol):
    obst, u, p, cfg = periodic_case(n=24, seed=8)
    n = obst.shape[0]
    gpu.aero_lbm_set_realtime_solver_mode(solver_mode)
    gpu.aero_lbm_b200_set_fp16_format(fmt)
    try:
        out, ctx = lbm_cases.run_product(gpu, (n, n, n), cfg, O.packet_from(obst, *u, pressure=p), 1, key=61)
        m0 = ctx.conservation_sums()[0]
        ctx.advance(300)
        m1 = ctx.conservation_sums()[0]
    finally:
        gpu.aero_lbm_set_realtime_solver_mode(0)
        gpu.aero_lbm_b200_set_fp16_format(1)
    assert abs(m1 - m0) / m0 < tol, (m0, m1)
