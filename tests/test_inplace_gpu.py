"""In-place (esoteric pull) layout and FP16 deviation storage on the GPU.

FP32 in-place with the reference-order collision stores the same numbers as
the two-buffer layout, so its outputs are compared bit-for-bit with the
oracle. FP16 storage is compared with the oracle's FP64 run of the same scheme:
velocity error relative to the max flow speed <= 1e-3, density error relative
to rho <= 1e-4."""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

import aero_b200
import lbm_cases
import oracle as O
from test_d3q27_gpu import assert_bits

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]


def load_cases():
    spec = importlib.util.spec_from_file_location("aero_b200_cases", ROOT / "aerodynamics4mc-fabric_b200" / "cases.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["aero_b200_cases"] = mod
    spec.loader.exec_module(mod)
    return mod


def local_faces_case(n=12, seed=21):
    rng = np.random.default_rng(seed)
    obst = (rng.random((n, n, n)) < 0.07).astype(np.uint8)
    u = [np.float32(0.05) + rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32),
         rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32),
         rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32)]
    p = rng.uniform(-0.005, 0.005, (n, n, n)).astype(np.float32)
    cfg = {"reynolds": 80.0, "initial_velocity": (0.05, 0.0, 0.0), "sgs": True, "buoyancy": False,
           "faces": [{"kind": O.VELOCITY, "velocity": (0.05, 0.01, 0.0)}, {"kind": O.PRESSURE, "pressure": 0.001},
                     {"kind": O.PERIODIC}, {"kind": O.PERIODIC},
                     {"kind": O.BOUNCE_BACK}, {"kind": O.MOVING_WALL, "velocity": (0.04, 0.0, 0.0)}]}
    return obst, u, p, cfg


@pytest.mark.parametrize("streaming", [1, 2])
def test_local_faces_bit_identical(gpu, streaming):
    obst, u, p, cfg = local_faces_case()
    n = obst.shape[0]
    out, ctx = lbm_cases.run_product(gpu, (n, n, n), cfg, O.packet_from(obst, *u, pressure=p), 50,
                                     streaming_mode=streaming)
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    o.set_fields(obst, *u, pressure=p)
    o.step(50)
    assert_bits(out, o.output())
    for stride in (2, 4):
        assert_bits(ctx.atlas(stride), o.atlas(stride))


@pytest.mark.parametrize("streaming", [1, 2])
def test_mask_change_between_packets(gpu, streaming):
    """New solids appear and cells that were solid since initialisation open
    up between calls; both layouts must follow the reference call for call."""
    n = 12
    obst, u, p, cfg = local_faces_case(n, seed=5)
    obst2 = obst.copy()
    rng = np.random.default_rng(99)
    flip_to_solid = (rng.random(obst.shape) < 0.03) & (obst == 0)
    flip_to_fluid = (rng.random(obst.shape) < 0.5) & (obst == 1)
    obst2[flip_to_solid] = 1
    obst2[flip_to_fluid] = 0
    pk1 = O.packet_from(obst, *u, pressure=p)
    pk2 = O.packet_from(obst2, *u, pressure=p)
    gpu.aero_lbm_b200_set_streaming_mode(streaming)
    gpu.aero_lbm_b200_set_collision_mode(0)
    ctx = aero_b200.LbmContext((n, n, n), key=31, lib=gpu)
    ctx.configure(lbm_cases.product_config(gpu, cfg))
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    out = None
    for s in range(30):
        pk, ob = (pk1, obst) if s < 12 else (pk2, obst2)
        out = ctx.step(pk, output=(s + 1 == 30))
        o.set_fields(ob, *u, pressure=p)
        o.step(1)
    assert_bits(out, o.output())


def _fp16_run(gpu, case, steps, key):
    gpu.aero_lbm_set_realtime_solver_mode(3)
    try:
        out, ctx = lbm_cases.run_product(gpu, case.dims, case.config_dict(), case.packet(), steps, key=key,
                                         smagorinsky_c=case.smagorinsky_c, beta=case.buoyancy_beta,
                                         axis=case.gravity_axis, streaming_mode=0,
                                         temperature_state=case.temperature_state())
    finally:
        gpu.aero_lbm_set_realtime_solver_mode(0)
    return out, ctx


def _oracle_run(case, steps, precision):
    cfg = case.config_dict()
    o = O.Oracle(case.dims, O.derive_params(cfg), precision)
    if case.temperature_state() is not None:
        o.set_temperature(case.temperature_state())
    o.set_fields(case.obstacle, *case.u, temperature=case.temperature)
    o.step(steps)
    return o.output()


def test_fp16_terrain_against_fp64(gpu):
    cases = load_cases()
    case = cases.c2_terrain_boussinesq(n=32, seed=7)
    steps = 200
    out16, _ = _fp16_run(gpu, case, steps, key=41)
    ref64 = _oracle_run(case, steps, "f64")
    e = O.flow_errors(out16, ref64)
    assert e["u"] <= 1e-3 and e["rho"] <= 1e-4, e
    solid = case.obstacle.reshape(-1) != 0
    assert np.all(out16[solid] == 0)


@pytest.mark.parametrize("cells_per_thread", [1, 2])
@pytest.mark.parametrize("n", [24, 23])
def test_fp32_terrain_bit_identical(gpu, n, cells_per_thread):
    """Reference-order FP32 step, one cell per thread or two z-adjacent cells
    per thread with the collision in packed FP32 (odd n leaves a lone last
    cell in every line): bit-identical to the oracle's FP32 run."""
    cases = load_cases()
    case = cases.c2_terrain_boussinesq(n=n, seed=8)
    steps = 60
    assert gpu.aero_lbm_b200_set_cells_per_thread(cells_per_thread) == 1
    try:
        out, ctx = lbm_cases.run_product(gpu, case.dims, case.config_dict(), case.packet(), steps, key=43,
                                         smagorinsky_c=case.smagorinsky_c, beta=case.buoyancy_beta,
                                         axis=case.gravity_axis, temperature_state=case.temperature_state())
    finally:
        gpu.aero_lbm_b200_set_cells_per_thread(2)
    assert_bits(out, _oracle_run(case, steps, "f32"))


def test_fp16_storage_bytes_and_scale(gpu):
    """FP16 contexts keep 27 halves per padded cell; a resting brick stays at rest."""
    n = 16
    obst = np.zeros((n, n, n), np.uint8)
    zero = np.zeros((n, n, n), np.float32)
    cfg = {"reynolds": 100.0, "faces": [{"kind": O.PERIODIC}] * 6, "sgs": True, "buoyancy": False}
    gpu.aero_lbm_set_realtime_solver_mode(3)
    try:
        out, ctx = lbm_cases.run_product(gpu, (n, n, n), cfg, O.packet_from(obst, zero, zero, zero), 20, key=45)
    finally:
        gpu.aero_lbm_set_realtime_solver_mode(0)
    assert np.max(np.abs(out[:, :3])) < 1e-6
    assert np.max(np.abs(out[:, 3])) < 1e-6


def _porous_case(dims, seed):
    rng = np.random.default_rng(seed)
    obst = (rng.random(dims) < 0.06).astype(np.uint8)
    obst[:, :, 0] = 1
    u = [np.float32(0.05) + rng.uniform(-0.005, 0.005, dims).astype(np.float32),
         rng.uniform(-0.005, 0.005, dims).astype(np.float32), rng.uniform(-0.005, 0.005, dims).astype(np.float32)]
    return obst, u


@pytest.mark.parametrize("cells_per_thread", [1, 2])
@pytest.mark.parametrize("dims", [(20, 18, 24), (10, 9, 13)])
def test_fast_collision_launch_shapes(gpu, dims, cells_per_thread):
    """The factorised FP32 in-place step, one cell per thread or two z-adjacent
    cells per thread with the packed FP32 collision (odd nz leaves a lone last
    cell), against the oracle's FP64 run: velocity within 1e-4 of the max
    speed, density within 1e-5 after 60 steps."""
    obst, u = _porous_case(dims, seed=sum(dims))
    cfg = O.c1_config()
    assert gpu.aero_lbm_b200_set_cells_per_thread(cells_per_thread) == 1
    try:
        out, _ = lbm_cases.run_product(gpu, dims, cfg, O.packet_from(obst, *u), 60, key=51, streaming_mode=2,
                                       collision_mode=1)
    finally:
        gpu.aero_lbm_b200_set_collision_mode(0)
        gpu.aero_lbm_b200_set_cells_per_thread(2)
    o = O.Oracle(dims, O.derive_params(cfg), "f64")
    o.set_fields(obst, *u)
    o.step(60)
    e = O.flow_errors(out, o.output())
    assert e["u"] <= 1e-4 and e["rho"] <= 1e-5, e


def test_fast_collision_mask_change(gpu):
    """Mask changes between calls with the two-cell kernel: cells turning
    solid pass their streamed populations through, cells opening up go
    through the transition kernel."""
    n = 12
    obst, u, p, cfg = local_faces_case(n, seed=6)
    obst2 = obst.copy()
    rng = np.random.default_rng(98)
    obst2[(rng.random(obst.shape) < 0.04) & (obst == 0)] = 1
    obst2[(rng.random(obst.shape) < 0.5) & (obst == 1)] = 0
    pk1, pk2 = O.packet_from(obst, *u, pressure=p), O.packet_from(obst2, *u, pressure=p)
    gpu.aero_lbm_b200_set_streaming_mode(2)
    gpu.aero_lbm_b200_set_collision_mode(1)
    try:
        ctx = aero_b200.LbmContext((n, n, n), key=53, lib=gpu)
        ctx.configure(lbm_cases.product_config(gpu, cfg))
        o = O.Oracle((n, n, n), O.derive_params(cfg), "f64")
        out = None
        for s in range(24):
            pk, ob = (pk1, obst) if s < 10 else (pk2, obst2)
            out = ctx.step(pk, output=(s + 1 == 24))
            o.set_fields(ob, *u, pressure=p)
            o.step(1)
    finally:
        gpu.aero_lbm_b200_set_collision_mode(0)
    e = O.flow_errors(out, o.output())
    assert e["u"] <= 1e-4 and e["rho"] <= 1e-5, e


@pytest.mark.parametrize("fmt", [0, 1])
def test_sixteen_bit_formats_against_fp64(gpu, fmt):
    """16-bit deviation storage, IEEE half (0) and fixed point (1), on the
    32^3 terrain brick against the oracle's FP64 run after 200 steps: velocity
    within 1e-3 of the max speed (fixed point: within 3e-4), density 1e-4."""
    cases = load_cases()
    case = cases.c2_terrain_boussinesq(n=32, seed=7)
    assert gpu.aero_lbm_b200_set_fp16_format(fmt) == 1
    try:
        out16, _ = _fp16_run(gpu, case, 200, key=45 + fmt)
    finally:
        gpu.aero_lbm_b200_set_fp16_format(1)
    e = O.flow_errors(out16, _oracle_run(case, 200, "f64"))
    assert e["u"] <= (3e-4 if fmt else 1e-3) and e["rho"] <= 1e-4, e
