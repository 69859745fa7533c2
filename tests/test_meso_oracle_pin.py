"""Pin the D3Q19 mesoscale oracle: its float restatement must reproduce the
reference's aero_lbm_mesoscale_step_context bit-for-bit (committed golden
fixture, and live against oracle/_ref when that library is present)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module", autouse=True)
def _build_oracle():
    O.build(ref=False)


def _bits_equal(a, b) -> bool:
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def test_meso_oracle_matches_golden():
    g = np.load(GOLDEN / "meso_12x8x10_30.npz")
    dims = tuple(int(d) for d in g["dims"])
    forcing = O.meso_forcing(dims, seed=int(g["seed"]))
    o = O.MesoOracle(dims)
    for _ in range(int(g["steps"])):
        out = o.step(forcing)
    assert _bits_equal(out, g["out"])


def test_meso_oracle_f64_close_to_f32():
    dims = (10, 6, 9)
    forcing = O.meso_forcing(dims, seed=3)
    a, b = O.MesoOracle(dims, precision="f32"), O.MesoOracle(dims, precision="f64")
    for _ in range(10):
        oa, ob = a.step(forcing), b.step(forcing)
    # temperatures (K) to 1e-4 relative, winds to 1e-4 of the clamp speed
    assert np.max(np.abs(oa[:, :3] - ob[:, :3]) / np.abs(ob[:, :3])) < 1e-4
    assert np.max(np.abs(oa[:, 3:] - ob[:, 3:])) < 1e-4 * 4.48


@pytest.mark.skipif(not O.REF_LIB.exists(), reason="reference library not built here")
@pytest.mark.parametrize("dims,dt,seed,wind", [
    ((9, 5, 7), 5.0, 11, (6.0, 0.0, 3.0)),
    ((8, 1, 8), 5.0, 12, (2.0, 0.5, -4.0)),   # one layer: no vertical laplacian
    ((7, 4, 6), 0.5, 13, (20.0, 1.0, 0.0)),   # clamped winds, slower relaxation
])
def test_meso_oracle_matches_reference_live(dims, dt, seed, wind):
    forcing = O.meso_forcing(dims, seed=seed, wind=wind)
    ref = O.meso_ref_run(dims, forcing, 12, dt=dt)
    o = O.MesoOracle(dims, dt=dt)
    for _ in range(12):
        out = o.step(forcing)
    assert _bits_equal(out, ref)
