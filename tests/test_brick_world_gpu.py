"""The native brick-world service (aero_lbm_simulation_* of libaero_lbm_b200.so)
on the GPU against the reference's own service (its simulation bridge over
its CPU step, oracle/_ref/libaero_sim_ref.so, and the golden fixture made from
it): the game-runtime physics of the classic solver mode (fans, edge state
nudge, sponge, the every-other-call temperature transport, halo exchanges
between neighbouring bricks), seeding, face bootstrap, boundary references,
world deltas, queued uploads and the int16 atlas, bit for bit."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import aero_b200
import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_native_service_matches_fixture(gpu):
    g = np.load(GOLDEN / "brickworld_16x4_6.npz")
    r = O.BrickService(aero_b200.LIB_PATH).run(O.brick_world_case())
    assert np.array_equal(r["status"], g["status"]), (r["status"], g["status"])
    flow = np.stack(r["flow"])
    assert np.array_equal(_bits(flow), _bits(np.asarray(g["flow"], np.float32)))
    assert np.array_equal(_bits(np.stack(r["air_t"])), _bits(np.asarray(g["air_t"], np.float32)))
    # the int16 atlas is quantised on the device: equal to the reference's host quantisation
    assert np.array_equal(np.stack(r["atlas"]), g["atlas"])


def _compare(ref, ours):
    assert len(ref) == len(ours)
    for i, (x, y) in enumerate(zip(ref, ours)):
        assert x[0] == y[0], (i, x[0], y[0])
        if x[0] == "step":
            assert x[1] == y[1], (i, x, y)
            continue
        for j, (u, v) in enumerate(zip(x[1:], y[1:])):
            if isinstance(u, np.ndarray):
                same = u.dtype == v.dtype and np.array_equal(u.view(np.uint8), v.view(np.uint8))
                if not same and u.dtype == np.float32:
                    d = np.abs(u.astype(np.float64) - v.astype(np.float64))
                    bad = np.nonzero(u.view(np.uint32) != v.view(np.uint32))[0]
                    pytest.fail(f"record {i} ({x[0]}) field {j}: {bad.size} values differ, max |d| {d.max():.3e}, "
                                f"first at {bad[:5]}")
                assert same, (i, x[0], j, np.count_nonzero(u != v))
            else:
                assert u == v, (i, x, y)


@pytest.mark.skipif(not O.SIM_REF_LIB.exists(), reason="reference service not built (make -C oracle sim)")
def test_native_service_rich_session_matches_reference(gpu):
    script = O.brick_world_rich_script(n=12)
    ref = O.run_brick_script(O.SIM_REF_LIB, script)
    ours = O.run_brick_script(aero_b200.LIB_PATH, script)
    assert all(r[1] == 1 for r in ref if r[0] == "step")
    _compare(ref, ours)


@pytest.mark.skipif(not O.SIM_REF_LIB.exists(), reason="reference service not built (make -C oracle sim)")
def test_native_service_32_bricks_match_reference(gpu):
    """Four 32^3 bricks (the smallest brick size of the batched-brick config)."""
    w = O.brick_world_case(n=32, steps=4, seed=77)
    ref = O.BrickService(O.SIM_REF_LIB).run(w)
    ours = O.BrickService(aero_b200.LIB_PATH).run(w)
    assert np.array_equal(ref["status"], ours["status"])
    assert np.array_equal(_bits(np.stack(ref["flow"])), _bits(np.stack(ours["flow"])))
    assert np.array_equal(_bits(np.stack(ref["air_t"])), _bits(np.stack(ours["air_t"])))
    assert np.array_equal(np.stack(ref["atlas"]), np.stack(ours["atlas"]))


def test_native_service_fp16_mode_runs_cached(gpu):
    """The FP16 in-place solver mode (3): after its first packet step a brick
    steps from its resident state (the reference's GPU path); the session runs,
    stays finite and moves the flow."""
    script = [op if op[0] != "mode" else ("mode", op[1], 3) for op in O.brick_world_rich_script(n=12)]
    ours = O.run_brick_script(aero_b200.LIB_PATH, script)
    assert all(r[1] == 1 for r in ours if r[0] == "step"), [r for r in ours if r[0] == "step"]
    copies = [r for r in ours if r[0] == "copy" and r[1] == 1]
    assert copies
    for r in copies:
        assert np.all(np.isfinite(r[2])) and np.all(np.isfinite(r[3]))
    assert max(float(np.abs(r[2]).max()) for r in copies) > 1e-3
    lib = aero_b200.load_library()
    svc = aero_b200.BrickWorldService(lib)
    try:
        svc.ensure_world(2, 12, solver_mode=3)
        svc.set_hints(2, [(0, 0, 0)])
        ob = np.zeros(12 ** 3, np.uint8)
        svc.upload_static(2, (0, 0, 0), ob)
        fl = np.zeros((12 ** 3, 4), np.float32)
        fl[:, 0] = 0.04
        svc.upload_dynamic(2, (0, 0, 0), fl, np.zeros(12 ** 3, np.float32))
        svc.step(2, 4)
        info = svc.runtime_info()
        fields = dict(kv.split("=", 1) for kv in info.split("|")[1:] if "=" in kv)
        assert int(fields["compact_initial_steps"]) >= 1 and int(fields["compact_cached_steps"]) >= 3, info
        f, a, s = svc.dynamic(2, (0, 0, 0))
        assert np.all(np.isfinite(f)) and abs(float(f[:, 0].mean()) - 0.04) < 0.01
    finally:
        svc.release()
