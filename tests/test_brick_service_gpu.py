"""The reference's brick-world service (aero_lbm_simulation_*, its
simulation bridge compiled from its own sources by `make -C oracle sim`)
linked against libaero_lbm_b200.so: every per-context call it makes
(aero_lbm_init_rect, step_rect, step_rect_cached, exchange_halo_layers_rect,
get_flow_state_rect, extract_flow_atlas_rect, temperature state, overlays,
shell and patches, ...) is served by the GPU library.

The service runs the reference's game-runtime physics (benchmark mode off):
fan forcing, the edge state nudge, the sponge and the stride-2 temperature
update of that mode are not modelled by this library, so the check against
the service on the reference's CPU step (fixture brickworld_16x4_6.npz) is
the run's structure (same bricks, same status counters) and a bound on the
flow difference after 6 ticks, not bit equality."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.skipif(not O.SIM_B200_LIB.exists(), reason="brick service not built (make -C oracle sim)")
def test_reference_brick_service_on_gpu_library(gpu):
    g = np.load(GOLDEN / "brickworld_16x4_6.npz")
    w = O.brick_world_case()
    r = O.BrickService(O.SIM_B200_LIB).run(w)
    assert np.array_equal(r["status"], g["status"]), (r["status"], g["status"])
    flow = np.stack(r["flow"])
    assert np.all(np.isfinite(flow)) and np.all(np.isfinite(np.stack(r["air_t"])))
    du = float(np.max(np.abs(flow[..., :3] - g["flow"][..., :3])))
    umax = float(np.max(np.abs(g["flow"][..., :3])))
    atlas_diff = int(np.max(np.abs(np.stack(r["atlas"]).astype(np.int32) - g["atlas"].astype(np.int32))))
    print(f"brick service: max |du| {du:.3e} of max |u| {umax:.3e}; atlas max diff {atlas_diff} counts")
    assert du <= 0.2 * umax, (du, umax)  # measured 0.12 (runtime-mode terms not modelled)
