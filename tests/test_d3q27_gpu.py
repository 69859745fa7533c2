"""FP32 D3Q27 brick step on the GPU against the reference (golden fixtures made
by the reference library) and the oracle.

The default FP32 collision (collision mode 0) performs the reference's
operations in the reference's order, so its outputs must be bit-identical to
the reference's: these tests compare bits. The factorised collision (mode 1)
is the same scheme with different rounding; the porous C1 flow amplifies
rounding differences exponentially (the reference's own FP32 and FP64 runs
separate by ~1e-4 after 300 steps), so mode 1 is checked with
oracle.flow_errors <= 1e-5 (velocity relative to the max speed, density
relative to rho) over a 30-step horizon."""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np
import pytest

import aero_b200
import lbm_cases
import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
TOL = 1e-5


def channel_errors(out, ref):
    e = O.flow_errors(out, ref)
    return [e["u"], e["rho"]]


def assert_bits(out, ref):
    a = np.asarray(out, np.float32)
    b = np.asarray(ref, np.float32)
    diff = np.nonzero(a.view(np.uint32) != b.view(np.uint32))
    assert diff[0].size == 0, (f"{diff[0].size} values differ; first at {diff[0][0]},{diff[1][0]}: "
                               f"{a[diff][0]!r} vs {b[diff][0]!r}; errors {channel_errors(a, b)}")


@pytest.mark.parametrize("mode", [1, 0])
def test_c1_16_bit_identical_to_reference(gpu, mode):
    g = np.load(GOLDEN / "c1_16_200.npz")
    n, steps = int(g["n"]), int(g["steps"])
    obst, u = O.c1_inputs(seed=int(g["seed"]), n=n)
    out, ctx = lbm_cases.run_product(gpu, (n, n, n), O.c1_config(), O.packet_from(obst, *u), steps, streaming_mode=mode)
    assert_bits(out, g["out"])
    solid = obst.reshape(-1) != 0
    assert np.all(out[solid] == 0.0)


@pytest.mark.parametrize("mode", [1, 0])
def test_c1_32_1000_bit_identical_to_reference(gpu, mode):
    g = np.load(GOLDEN / "c1_32_1000.npz")
    n, steps = int(g["n"]), int(g["steps"])
    obst, u = O.c1_inputs(seed=int(g["seed"]), n=n)
    out, ctx = lbm_cases.run_product(gpu, (n, n, n), O.c1_config(), O.packet_from(obst, *u), steps, streaming_mode=mode)
    assert_bits(out, g["out"])


@pytest.mark.parametrize("streaming,cpt", [(1, 2), (2, 1), (2, 2)])
def test_tunnel_bit_identical_to_reference(gpu, streaming, cpt):
    """Velocity inlet, convective outflow and symmetry faces around a sphere:
    the two-buffer layout pulls the face values from the post-collision
    state, the in-place layout from the slots its end-of-call fill wrote."""
    g = np.load(GOLDEN / "tunnel_16_60.npz")
    obst, u, cfg = lbm_cases.tunnel_case(16)
    assert gpu.aero_lbm_b200_set_cells_per_thread(cpt) == 1
    try:
        out, ctx = lbm_cases.run_product(gpu, (16, 16, 16), cfg, O.packet_from(obst, *u), int(g["steps"]),
                                         streaming_mode=streaming)
    finally:
        gpu.aero_lbm_b200_set_cells_per_thread(2)
    assert_bits(out, g["out"])


def test_factorised_collision_within_tolerance(gpu):
    n, steps = 16, 30
    obst, u = O.c1_inputs(seed=77, n=n)
    cfg = O.c1_config()
    out, ctx = lbm_cases.run_product(gpu, (n, n, n), cfg, O.packet_from(obst, *u), steps, collision_mode=1)
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    o.set_fields(obst, *u)
    o.step(steps)
    errs = channel_errors(out, o.output())
    assert max(errs) <= TOL, errs
    gpu.aero_lbm_b200_set_collision_mode(0)


@pytest.mark.parametrize("streaming", [1, 2])
@pytest.mark.parametrize("faces", ["pressure_outlet", "closed", "inherit_game", "periodic_all"])
def test_faces_match_oracle(gpu, faces, streaming):
    n = 12
    rng = np.random.default_rng(11)
    obst = (rng.random((n, n, n)) < 0.08).astype(np.uint8)
    u = [np.float32(0.04) + rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32),
         rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32),
         rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32)]
    p = rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32)
    table = {
        "pressure_outlet": [{"kind": O.VELOCITY, "velocity": (0.04, 0.0, 0.0)}, {"kind": O.PRESSURE, "pressure": 0.002}]
                           + [{"kind": O.SYMMETRY}] * 4,
        "closed": [{"kind": O.BOUNCE_BACK}] * 5 + [{"kind": O.MOVING_WALL, "velocity": (0.05, 0.0, 0.0)}],
        "inherit_game": [{"kind": O.INHERIT_GAME}] * 6,
        "periodic_all": [{"kind": O.PERIODIC}] * 6,
    }
    cfg = {"reynolds": 60.0, "initial_velocity": (0.04, 0.0, 0.0), "faces": table[faces], "sgs": True, "buoyancy": False}
    pk = O.packet_from(obst, *u, pressure=p)
    out, ctx = lbm_cases.run_product(gpu, (n, n, n), cfg, pk, 40, streaming_mode=streaming)
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    o.set_fields(obst, *u, pressure=p)
    o.step(40)
    assert_bits(out, o.output())


def test_atlas_and_flow_state_match_oracle(gpu):
    n = 16
    obst, u = O.c1_inputs(seed=5, n=n)
    cfg = O.c1_config()
    out, ctx = lbm_cases.run_product(gpu, (n, n, n), cfg, O.packet_from(obst, *u), 30)
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    o.set_fields(obst, *u)
    o.step(30)
    for stride in (1, 3, 4):
        a = ctx.atlas(stride)
        b = o.atlas(stride)
        assert a.shape == b.shape
        assert_bits(a, b)
    assert_bits(ctx.flow_state(), o.output())


def test_cached_step_equals_packet_step(gpu):
    n = 12
    obst, u = O.c1_inputs(seed=9, n=n)
    pk = O.packet_from(obst, *u)
    cfg = O.c1_config()
    a, _ = lbm_cases.run_product(gpu, (n, n, n), cfg, pk, 10)  # first packet, then cached steps
    ctx = aero_b200.LbmContext((n, n, n), key=9, lib=gpu)
    ctx.configure(lbm_cases.product_config(gpu, cfg))
    b = None
    for s in range(10):
        b = ctx.step(pk, output=(s == 9))
    assert np.array_equal(a, b)


def test_step_argument_errors(gpu):
    ctx = aero_b200.LbmContext((8, 8, 8), key=3, lib=gpu)
    assert gpu.aero_lbm_step_rect(None, 8, 8, 8, 3, None) == 0
    assert "missing packet" in aero_b200.last_error(gpu)
    assert gpu.aero_lbm_step_rect_cached(8, 8, 8, 4242, None) == 0
    out = np.zeros(10, np.float32)
    assert gpu.aero_lbm_extract_flow_atlas_rect(8, 8, 8, 3, 4, aero_b200.fptr(out), 10) == 0
    assert gpu.aero_lbm_init_rect(8, 8, 8, 4, 4) == 0  # fewer than 9 input channels
