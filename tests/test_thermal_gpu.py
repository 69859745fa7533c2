"""Temperature transport on the GPU (the reference's benchmark-mode update
before every collision: advection by the previous collision's velocity,
diffusion, the packet's source channel, thermal faces).

The reference-order FP32 step with the transport is bit-identical to the
reference library (golden fixture thermal_12_20.npz: flow output and
temperature state) in both layouts and both launch shapes, and to the oracle
under mask changes between calls; FP16 storage with the transport is within
the stated tolerance of the oracle's FP64 run. The mode switch selects the
packet's field instead (0) or transports without buoyancy too (1)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import aero_b200
import lbm_cases
import oracle as O
from test_d3q27_gpu import assert_bits

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def _run(gpu, n, cfg, packets, steps, streaming, preload, key, cpt=2, collision=0, mode=-1):
    """packets: list of (first_step, packet); the packet in force from that step on.
    n: the edge of a cubic brick, or its (nx, ny, nz)."""
    dims = (n, n, n) if isinstance(n, int) else tuple(n)
    gpu.aero_lbm_b200_set_physics_overrides(-1.0, -1.0, -1)
    gpu.aero_lbm_b200_set_streaming_mode(streaming)
    gpu.aero_lbm_b200_set_collision_mode(collision)
    assert gpu.aero_lbm_b200_set_cells_per_thread(cpt) == 1
    assert gpu.aero_lbm_b200_set_thermal_transport(mode) == 1
    try:
        ctx = aero_b200.LbmContext(dims, key=key, lib=gpu)
        ctx.configure(lbm_cases.product_config(gpu, cfg))
        if preload is not None:
            ctx.set_temperature_state(preload)
        out = None
        for s in range(steps):
            pk = [p for first, p in packets if first <= s][-1]
            out = ctx.step(pk, output=(s + 1 == steps))
        temp = ctx.temperature_state()
        ctx.release()
    finally:
        gpu.aero_lbm_b200_set_thermal_transport(-1)
        gpu.aero_lbm_b200_set_cells_per_thread(2)
        gpu.aero_lbm_b200_set_collision_mode(0)
    return out, temp


@pytest.mark.parametrize("streaming,cpt", [(1, 1), (2, 1), (2, 2)])
def test_thermal_transport_matches_reference_golden(gpu, streaming, cpt):
    g = np.load(GOLDEN / "thermal_12_20.npz")
    n, steps = int(g["n"]), int(g["steps"])
    obst, u, temp, src, cfg, preload = O.thermal_case(n, int(g["seed"]))
    pk = O.packet_from(obst, *u, temperature=temp, source=src)
    out, t = _run(gpu, n, cfg, [(0, pk)], steps, streaming, preload, key=600 + 2 * streaming + cpt, cpt=cpt)
    assert_bits(out, g["out"])
    assert np.array_equal(t.view(np.uint32), np.asarray(g["temperature"], np.float32).view(np.uint32))


@pytest.mark.parametrize("streaming", [1, 2])
def test_thermal_transport_mask_change_matches_oracle(gpu, streaming):
    """Solids appear and open up between calls; no preload (every cell starts
    at the configured initial temperature), no source."""
    n, steps = 12, 24
    obst, u, temp, src, cfg, _ = O.thermal_case(n, 31)
    cfg = dict(cfg, thermal_source=False)
    rng = np.random.default_rng(32)
    obst2 = obst.copy()
    obst2[(rng.random(obst.shape) < 0.03) & (obst == 0)] = 1
    obst2[(rng.random(obst.shape) < 0.5) & (obst == 1)] = 0
    pk1 = O.packet_from(obst, *u, temperature=temp)
    pk2 = O.packet_from(obst2, *u, temperature=temp)
    out, t = _run(gpu, n, cfg, [(0, pk1), (10, pk2)], steps, streaming, None, key=620 + streaming)
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    for s in range(steps):
        ob = obst if s < 10 else obst2
        o.set_fields(ob, *u, temperature=temp)
        o.step(1)
    assert_bits(out, o.output())
    assert np.array_equal(t.view(np.uint32), o.temperature().view(np.uint32))


_EDGE_FACES = [{"kind": O.PERIODIC, "thermal": O.THERMAL_PERIODIC}, {"kind": O.PERIODIC, "thermal": O.THERMAL_PERIODIC},
               {"kind": O.BOUNCE_BACK, "thermal": O.THERMAL_ADIABATIC}, {"kind": O.SYMMETRY},
               {"kind": O.VELOCITY, "velocity": (0.03, 0, 0), "thermal": O.THERMAL_DIRICHLET, "temperature": 0.25},
               {"kind": O.CONVECTIVE, "thermal": O.THERMAL_DISABLED}]


@pytest.mark.parametrize("variant,dims,steps", [("faces", (37, 19, 45), 6), ("periodic_x", (17, 9, 33), 6),
                                                ("fast", (37, 19, 45), 2), ("tiny", (5, 3, 7), 6)])
@pytest.mark.parametrize("streaming", [1, 2])
def test_thermal_transport_brick_edges_match_oracle(gpu, variant, dims, steps, streaming):
    """Non-cubic bricks: several x-chunks of the transport's column walk with
    a partial last one (a single plane for nx = 17), partial y and z tiles.
    faces: every thermal face kind incl. Neumann; periodic_x: thermally
    periodic x (the wrapped planes staged), symmetry and velocity faces, no
    Neumann face; fast: the same faces with packet speeds up to 0.6 and two
    cells beyond one cell per step (the out-of-window trilinear sample) for
    the first update; tiny: periodic_x's faces on a brick smaller than one
    tile in every axis (odd z extent: no z-pair vector access). Flow output
    and temperature state bit-identical to the oracle, both layouts."""
    _, _, _, _, cfg, _ = O.thermal_case(12, 11)
    if variant != "faces":
        cfg = dict(cfg, faces=_EDGE_FACES)
    rng = np.random.default_rng(41 + len(variant))
    obst = (rng.random(dims) < 0.08).astype(np.uint8)
    spread = 0.6 if variant == "fast" else 0.01
    u = [rng.uniform(-spread, spread, dims).astype(np.float32) for _ in range(3)]
    u[0] += np.float32(0.04)
    if variant == "fast":
        u[0][5, 5, 5], u[1][20, 10, 30], u[2][36, 18, 44] = 1.5, -1.25, -1.0
    if variant == "tiny":
        obst[2, 1, 3] = 1
    temp = rng.uniform(-0.3, 0.3, dims).astype(np.float32)
    src = rng.uniform(-0.01, 0.01, dims).astype(np.float32)
    pre = np.full(int(np.prod(dims)), 0.5, np.float32)
    pk = O.packet_from(obst, *u, temperature=temp, source=src)
    out, t = _run(gpu, dims, cfg, [(0, pk)], steps, streaming, pre, key=700 + streaming + 4 * len(variant))
    o = O.Oracle(dims, O.derive_params(cfg), "f32")
    o.set_temperature(pre)
    o.set_fields(obst, *u, temperature=temp)
    o.set_thermal_source(src)
    o.step(steps)
    assert_bits(out, o.output())
    assert np.array_equal(t.view(np.uint32), o.temperature().view(np.uint32))


def test_thermal_transport_fp16_against_fp64(gpu):
    """FP16 deviation storage with the transport on the 32^3 terrain brick
    (its temperature field loaded as the starting state) against the oracle's
    FP64 run: velocity within 1e-3 of the max speed, density within 1e-4,
    temperature state within 1e-3 after 200 steps."""
    import importlib.util
    import sys
    spec = importlib.util.spec_from_file_location(
        "aero_b200_cases_t", Path(__file__).resolve().parents[1] / "aerodynamics4mc-fabric_b200" / "cases.py")
    cases = importlib.util.module_from_spec(spec)
    sys.modules["aero_b200_cases_t"] = cases
    spec.loader.exec_module(cases)
    case = cases.c2_terrain_boussinesq(n=32, seed=7)
    steps = 200
    gpu.aero_lbm_set_realtime_solver_mode(3)
    try:
        out16, ctx = lbm_cases.run_product(gpu, case.dims, case.config_dict(), case.packet(), steps, key=640,
                                           smagorinsky_c=case.smagorinsky_c, beta=case.buoyancy_beta,
                                           axis=case.gravity_axis, temperature_state=case.temperature_state())
        t16 = ctx.temperature_state()
        ctx.release()
    finally:
        gpu.aero_lbm_set_realtime_solver_mode(0)
    o = O.Oracle(case.dims, O.derive_params(case.config_dict()), "f64")
    o.set_temperature(case.temperature_state())
    o.set_fields(case.obstacle, *case.u, temperature=case.temperature)
    o.step(steps)
    e = O.flow_errors(out16, o.output())
    assert e["u"] <= 1e-3 and e["rho"] <= 1e-4, e
    assert float(np.max(np.abs(t16 - o.temperature()))) <= 1e-3


def test_thermal_modes(gpu):
    """Mode 0: the packet's temperature is the buoyancy field of every call
    (the oracle without transport). Mode 1 with buoyancy off: the flow is the
    plain step and the temperature state evolves exactly like the
    reference's (the oracle with transport)."""
    n, steps = 10, 12
    obst, u, temp, src, cfg, preload = O.thermal_case(n, 41)
    cfg = dict(cfg, thermal_source=False)
    pk = O.packet_from(obst, *u, temperature=temp)
    out0, _ = _run(gpu, n, cfg, [(0, pk)], steps, 2, None, key=660, mode=0)
    o = O.Oracle((n, n, n), O.derive_params(dict(cfg, thermal_transport=False)), "f32")
    o.set_fields(obst, *u, temperature=temp)
    o.step(steps)
    assert_bits(out0, o.output())

    cfg_nb = dict(cfg, buoyancy=False)
    out1, t1 = _run(gpu, n, cfg_nb, [(0, pk)], steps, 2, preload, key=662, mode=1)
    o = O.Oracle((n, n, n), O.derive_params(dict(cfg_nb, thermal_transport=True)), "f32")
    o.set_temperature(preload)
    o.set_fields(obst, *u, temperature=temp)
    o.step(steps)
    assert_bits(out1, o.output())
    assert np.array_equal(t1.view(np.uint32), o.temperature().view(np.uint32))


@pytest.mark.parametrize("streaming,cpt", [(1, 1), (2, 2)])
def test_bfecc_transport_matches_reference_golden(gpu, streaming, cpt):
    """Differentially heated cavity preset (3-D): the BFECC temperature
    transport (three launches) and the preset's derived parameters,
    bit-identical to the reference library's fixture (flow output and
    temperature state)."""
    g = np.load(GOLDEN / "cavity_12_25.npz")
    n, steps = int(g["n"]), int(g["steps"])
    obst, u, temp, cfg, preload = O.heated_cavity_case(n, int(g["seed"]))
    pk = O.packet_from(obst, *u, temperature=temp)
    out, t = _run(gpu, n, cfg, [(0, pk)], steps, streaming, preload, key=680 + streaming, cpt=cpt)
    assert_bits(out, g["out"])
    assert np.array_equal(t.view(np.uint32), np.asarray(g["temperature"], np.float32).view(np.uint32))


@pytest.mark.parametrize("collision,cpt", [(0, 1), (0, 2), (1, 2)])
def test_fused_transport_equals_separate_pass(gpu, collision, cpt):
    """The in-place step computing the transport itself (default) against the
    separate transport pass, on the thermal case with mask changes between
    calls (cells opening up take their temperature from the step, then
    collide in the transition kernel): flow and temperature bit for bit."""
    n, steps = 20, 16
    obst, u, temp, src, cfg, preload = O.thermal_case(n, 41)
    rng = np.random.default_rng(42)
    obst2 = obst.copy()
    obst2[(rng.random(obst.shape) < 0.03) & (obst == 0)] = 1
    obst2[(rng.random(obst.shape) < 0.5) & (obst == 1)] = 0
    pk1 = O.packet_from(obst, *u, temperature=temp, source=src)
    pk2 = O.packet_from(obst2, *u, temperature=temp, source=src)
    res = []
    for fused in (1, 0):
        assert gpu.aero_lbm_b200_set_fused_transport(fused) == 1
        try:
            res.append(_run(gpu, n, cfg, [(0, pk1), (7, pk2)], steps, 2, preload, key=640 + fused, cpt=cpt,
                            collision=collision))
        finally:
            gpu.aero_lbm_b200_set_fused_transport(1)
    (out_f, t_f), (out_s, t_s) = res
    assert_bits(out_f, out_s)
    assert np.array_equal(t_f.view(np.uint32), t_s.view(np.uint32))
