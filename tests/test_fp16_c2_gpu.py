"""The 16-bit deviation storage at the configured precision case: a 64^3
terrain brick of the 128^3 headline case's construction (heightmap,
inflow (0.08, 0.02, 0), Boussinesq g*beta = 1e-4 with the temperature
transport moving the lapse + warm-bubble field before every collision),
1000 steps, against the oracle's FP64 run of the same scheme (the oracle's
double instantiation, pinned to the reference library in
tests/test_oracle_pin.py). Bound: max |u - u64| <= 1e-3 of the max speed
and density within 1e-4, for the default 16-bit format (fixed point)."""
from __future__ import annotations

import time

import numpy as np
import pytest

import oracle as O
from test_inplace_gpu import _fp16_run, _oracle_run, load_cases

pytestmark = pytest.mark.gpu


def test_default_sixteen_bit_format_meets_bound_on_c2_64_1000(gpu):
    cases = load_cases()
    case = cases.c2_terrain_boussinesq(n=64, seed=2024)
    steps = 1000
    t0 = time.time()
    out16, _ = _fp16_run(gpu, case, steps, key=71)
    t1 = time.time()
    ref64 = _oracle_run(case, steps, "f64")
    t2 = time.time()
    e = O.flow_errors(out16, ref64)
    print(f"C2 64^3 x {steps}: default 16-bit vs FP64 u {e['u']:.3e} rho {e['rho']:.3e} "
          f"(GPU {t1 - t0:.1f} s, oracle {t2 - t1:.1f} s)")
    assert e["u"] <= 1e-3 and e["rho"] <= 1e-4, e
    solid = case.obstacle.reshape(-1) != 0
    assert np.all(out16[solid] == 0)
