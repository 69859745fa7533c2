"""Seeded cases shared by the parity tests (inputs only; no expected values)."""
from __future__ import annotations

import ctypes

import numpy as np

import aero_b200
import oracle as O


def product_config(lib, cfg: dict) -> aero_b200.AeroLbmBenchmarkConfig:
    """The dict-form case configuration as the product's config struct."""
    return O.config_struct(aero_b200.AeroLbmBenchmarkConfig, cfg, lib.aero_lbm_benchmark_default_config)


def run_product(lib, dims, cfg: dict, packet: np.ndarray, steps: int, key: int = 7,
                smagorinsky_c: float = -1.0, beta: float = -1.0, axis: int = -1,
                streaming_mode: int = 0, collision_mode: int = 0,
                temperature_state: np.ndarray | None = None) -> tuple[np.ndarray, aero_b200.LbmContext]:
    lib.aero_lbm_b200_set_physics_overrides(smagorinsky_c, beta, axis)
    lib.aero_lbm_b200_set_streaming_mode(streaming_mode)
    lib.aero_lbm_b200_set_collision_mode(collision_mode)
    ctx = aero_b200.LbmContext(dims, input_channels=packet.shape[1], key=key, lib=lib)
    ctx.configure(product_config(lib, cfg))
    if temperature_state is not None:
        ctx.set_temperature_state(temperature_state)
    out = None
    for s in range(steps):
        out = ctx.step(packet if s == 0 else None, output=(s + 1 == steps))
    return out, ctx


def tunnel_case(n: int = 16):
    obst = np.zeros((n, n, n), np.uint8)
    c = np.array([n // 3, n // 2, n // 2])
    r = max(1.0, n * 0.12)
    g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1)
    obst[np.sum((g - c) ** 2, -1) <= r * r] = 1
    u_in = 0.1
    ux = np.where(obst == 0, np.float32(u_in), np.float32(0)).astype(np.float32)
    zero = np.zeros_like(ux)
    cfg = {
        "reynolds": u_in / 0.01,
        "initial_velocity": (u_in, 0.0, 0.0),
        "faces": [{"kind": O.VELOCITY, "velocity": (u_in, 0.0, 0.0)}, {"kind": O.CONVECTIVE},
                  {"kind": O.SYMMETRY}, {"kind": O.SYMMETRY}, {"kind": O.SYMMETRY}, {"kind": O.SYMMETRY}],
        "sgs": False,
        "buoyancy": False,
    }
    return obst, (ux, zero, zero.copy()), cfg
