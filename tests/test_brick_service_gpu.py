"""The reference's brick-world service (aero_lbm_simulation_*, its
simulation bridge compiled from its own sources by `make -C oracle sim`)
linked against libaero_lbm_b200.so: every per-context call it makes
(aero_lbm_init_rect, step_rect, step_rect_cached, exchange_halo_layers_rect,
get_flow_state_rect, extract_flow_atlas_rect, temperature state, overlays,
shell and patches, ...) is served by the GPU library.

The service runs the reference's game-runtime physics (benchmark mode off:
fan forcing, edge state nudge, sponge, the every-other-call temperature
update); on the GPU library the four-brick world matches the same service
over the reference's CPU step (fixture brickworld_16x4_6.npz) bit for bit:
dynamic bricks, air temperature, packed atlases and status counters."""
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
    for b in range(flow.shape[0]):
        bad = np.nonzero(np.any(flow[b].view(np.uint32) != np.asarray(g["flow"][b], np.float32).view(np.uint32), axis=1))[0]
        tb = np.nonzero(np.stack(r["air_t"])[b].view(np.uint32) != np.asarray(g["air_t"][b], np.float32).view(np.uint32))[0]
        n = w["n"]
        xyz = [(int(c) // (n * n), (int(c) // n) % n, int(c) % n) for c in bad[:6]]
        print(f"brick {b}: {bad.size} flow cells differ, first {xyz}; {tb.size} temperature cells differ")
    assert np.array_equal(flow.view(np.uint32), np.asarray(g["flow"], np.float32).view(np.uint32))
    assert np.array_equal(np.stack(r["air_t"]).view(np.uint32), np.asarray(g["air_t"], np.float32).view(np.uint32))
    assert np.array_equal(np.stack(r["atlas"]), g["atlas"])
