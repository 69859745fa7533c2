"""Halo exchange between two overlapping bricks on the GPU
(aero_lbm_exchange_halo_layers_rect, native/src/aero_lbm_jni.cpp:8136-8426,
9693-9790).

Two contexts step call for call and exchange the streamed populations and
the temperature of their slabs between calls. FP32 reference-order storage
is bit-identical to the reference library's fixture (halo_12_12.npz) and to
the oracle on further offsets, halo widths and exchange periods, in both the
two-buffer and the in-place layout; the flow read right after an exchange
and the conservation sums see the exchanged state. FP16 in-place storage
with an exchange every step stays within the stated tolerance of the
oracle's FP64 run. Argument errors match the reference's checks."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import aero_b200
import lbm_cases
import oracle as O
from test_d3q27_gpu import assert_bits
from test_oracle_pin import _halo_oracles

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def _run_pair(gpu, n, cfg, pks, pre, steps, offset, halo, every, streaming, keys, cpt=2, solver_mode=0,
              after_exchange=None):
    """Step both contexts each call; exchange after every `every` calls except
    the last. after_exchange(call_index, ctx1, ctx2) runs after each exchange."""
    gpu.aero_lbm_b200_set_physics_overrides(-1.0, -1.0, -1)
    gpu.aero_lbm_b200_set_streaming_mode(streaming)
    gpu.aero_lbm_b200_set_collision_mode(0)
    gpu.aero_lbm_set_realtime_solver_mode(solver_mode)
    assert gpu.aero_lbm_b200_set_cells_per_thread(cpt) == 1
    # transport the temperature also without buoyancy, as the reference does
    assert gpu.aero_lbm_b200_set_thermal_transport(1) == 1
    try:
        c1 = aero_b200.LbmContext((n, n, n), key=keys[0], lib=gpu)
        c1.configure(lbm_cases.product_config(gpu, cfg))
        c2 = aero_b200.LbmContext((n, n, n), key=keys[1], lib=gpu, init=False)
        for c in (c1, c2):
            c.set_temperature_state(pre)
        outs = [None, None]
        for s in range(steps):
            last = s + 1 == steps
            for i, (c, pk) in enumerate(zip((c1, c2), pks)):
                o = c.step(pk, output=last)
                if last:
                    outs[i] = o
            if not last and (s + 1) % every == 0:
                assert gpu.aero_lbm_exchange_halo_layers_rect(n, n, n, halo, keys[0], keys[1], *offset) == 1, \
                    aero_b200.last_error(gpu)
                if after_exchange is not None:
                    after_exchange(s, c1, c2)
        temps = [c1.temperature_state(), c2.temperature_state()]
        c1.release()
        c2.release()
    finally:
        gpu.aero_lbm_b200_set_thermal_transport(-1)
        gpu.aero_lbm_b200_set_cells_per_thread(2)
        gpu.aero_lbm_set_realtime_solver_mode(0)
    return outs, temps


@pytest.mark.parametrize("streaming,cpt", [(1, 1), (2, 1), (2, 2)])
def test_halo_exchange_matches_reference_golden(gpu, streaming, cpt):
    g = np.load(GOLDEN / "halo_12_12.npz")
    n = int(g["n"])
    cfg, pks, pre = O.halo_case(n)
    outs, temps = _run_pair(gpu, n, cfg, pks, pre, int(g["steps"]), tuple(int(v) for v in g["offset"]), int(g["halo"]),
                            int(g["every"]), streaming, keys=(701 + 2 * streaming + cpt, 711 + 2 * streaming + cpt),
                            cpt=cpt)
    assert_bits(outs[0], g["out1"])
    assert_bits(outs[1], g["out2"])
    for t, ref in zip(temps, (g["t1"], g["t2"])):
        assert np.array_equal(t.view(np.uint32), np.asarray(ref, np.float32).view(np.uint32))


@pytest.mark.parametrize("streaming", [1, 2])
@pytest.mark.parametrize("offset,halo,buoy", [((1, 0, 0), 3, False), ((-1, 1, 1), 1, True), ((0, 0, -1), 4, True)])
def test_halo_exchange_matches_oracle(gpu, streaming, offset, halo, buoy):
    """Other offsets and widths; the flow state read right after each
    exchange (before the next call) and the FP64 conservation sums of the
    exchanged state agree with the oracle's."""
    n, steps, every = 12, 10, 3
    cfg, pks, pre = O.halo_case(n, buoyancy=buoy)
    seen = []

    def check(s, c1, c2):
        seen.append((s, c1.flow_state(), c2.flow_state(), c1.conservation_sums(), c2.conservation_sums()))

    outs, temps = _run_pair(gpu, n, cfg, pks, pre, steps, offset, halo, every, streaming,
                            keys=(730 + streaming, 740 + streaming), after_exchange=check)
    os_ = _halo_oracles(cfg, pks, pre, steps, offset, halo, every)
    for o, out, t in zip(os_, outs, temps):
        assert_bits(out, o.output())
        assert np.array_equal(t.view(np.uint32), o.temperature().view(np.uint32))
    assert [s for s, *_ in seen] == [2, 5, 8]
    # the state right after the last exchange (call 9 of 10)
    o9 = _halo_oracles(cfg, pks, pre, 9, offset, halo, every)
    # _halo_oracles exchanges only between calls; apply the exchange after call 9
    o9[0].exchange_halo(o9[1], offset, halo)
    _, f1, f2, s1, s2 = seen[-1]
    for o, f, sums, pk in zip(o9, (f1, f2), (s1, s2), pks):
        assert_bits(f, o.output())
        fluid = pk[:, 0] == 0
        pops = o.populations()[:, fluid].astype(np.float32).astype(np.float64)
        cx = np.array([(q // 9) - 1 for q in range(27)], np.float64)
        cy = np.array([((q // 3) % 3) - 1 for q in range(27)], np.float64)
        cz = np.array([(q % 3) - 1 for q in range(27)], np.float64)
        ref = np.array([pops.sum(), (cx @ pops).sum(), (cy @ pops).sum(), (cz @ pops).sum()])
        assert abs(sums[0] - ref[0]) / ref[0] < 1e-6
        assert np.max(np.abs(sums[1:] - ref[1:])) / ref[0] < 1e-6


def test_halo_exchange_fp16_against_fp64(gpu):
    """FP16 deviation storage (in-place) with an exchange after every call:
    velocity within 1e-3 of the max speed, density within 1e-4, temperature
    within 1e-3 of the oracle's FP64 pair after 20 calls."""
    n, steps, every, offset, halo = 12, 20, 1, (0, 1, 0), 2
    cfg, pks, pre = O.halo_case(n)
    outs, temps = _run_pair(gpu, n, cfg, pks, pre, steps, offset, halo, every, 2, keys=(760, 761), solver_mode=3)
    os_ = _halo_oracles(cfg, pks, pre, steps, offset, halo, every, precision="f64")
    for o, out, t in zip(os_, outs, temps):
        e = O.flow_errors(out, o.output())
        assert e["u"] <= 1e-3 and e["rho"] <= 1e-4, e
        assert float(np.max(np.abs(t - o.temperature()))) <= 1e-3


def test_halo_exchange_argument_checks(gpu):
    n = 12
    cfg, pks, pre = O.halo_case(n)
    gpu.aero_lbm_b200_set_streaming_mode(0)
    c1 = aero_b200.LbmContext((n, n, n), key=780, lib=gpu)
    c1.configure(lbm_cases.product_config(gpu, cfg))
    c2 = aero_b200.LbmContext((n, n, n), key=781, lib=gpu, init=False)
    try:
        ex = gpu.aero_lbm_exchange_halo_layers_rect
        # a context that exists but has not stepped makes the call a no-op
        c1.step(pks[0], output=False)
        c2.set_temperature_state(pre)
        assert ex(n, n, n, 2, 780, 781, 1, 0, 0) == 1
        c2.step(pks[1], output=False)
        bad = [
            ((n, n, n, 2, 780, 781, 0, 0, 0), "zero offset"),
            ((n, n, n, 2, 780, 781, 2, 0, 0), "invalid offset"),
            ((n, n, n, 0, 780, 781, 1, 0, 0), "halo_layers must be positive"),
            ((n, n, n, 6, 780, 781, 1, 0, 0), "invalid halo layout"),
            ((n, n, 10, 2, 780, 781, 1, 0, 0), "only cubic"),
            ((n, n, n, 2, 780, 799, 1, 0, 0), "missing context"),
            ((10, 10, 10, 2, 780, 781, 1, 0, 0), "differs from the requested"),
            ((n, n, n, 2, 780, 780, 1, 0, 0), "same context"),
        ]
        for args, msg in bad:
            assert ex(*args) == 0, args
            assert msg in aero_b200.last_error(gpu), (args, aero_b200.last_error(gpu))
        assert ex(n, n, n, 2, 780, 781, 1, 0, 0) == 1
        # the fixed-width form: the configured grid and max(1, n / 4) layers
        assert gpu.aero_lbm_exchange_halo(n, 780, 781, 0, 0, 1) == 1
        assert gpu.aero_lbm_exchange_halo(n + 1, 780, 781, 0, 0, 1) == 0
        assert "grid size mismatch" in aero_b200.last_error(gpu)
    finally:
        c1.release()
        c2.release()


def test_halo_exchange_runtime_mode_matches_oracle(gpu):
    """Benchmark mode off: the temperature slabs move only after a call that
    updated the temperature (every other call); the two-buffer layout."""
    n, steps, offset, halo = 12, 7, (1, 0, 0), 2
    cfg, pk1, pre = O.runtime_case(n, 74)
    _, pk2, _ = O.runtime_case(n, 75)
    gpu.aero_lbm_b200_set_streaming_mode(0)
    gpu.aero_lbm_b200_set_collision_mode(0)
    c1 = aero_b200.LbmContext((n, n, n), key=790, lib=gpu)
    gpu.aero_lbm_benchmark_reset_config()
    c2 = aero_b200.LbmContext((n, n, n), key=791, lib=gpu, init=False)
    os_ = []
    for _ in range(2):
        o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
        o.set_temperature(pre)
        os_.append(o)
    try:
        for c in (c1, c2):
            c.set_temperature_state(pre)
        for s in range(steps):
            last = s + 1 == steps
            outs = [c.step(pk, output=last) for c, pk in zip((c1, c2), (pk1, pk2))]
            for o, pk in zip(os_, (pk1, pk2)):
                O.run_script_oracle(o, cfg, pk, [("step",)])
            if not last:
                assert gpu.aero_lbm_exchange_halo_layers_rect(n, n, n, halo, 790, 791, *offset) == 1
                os_[0].exchange_halo(os_[1], offset, halo)
        for c, o, out in zip((c1, c2), os_, outs):
            assert_bits(out, o.output())
            assert np.array_equal(c.temperature_state().view(np.uint32), o.temperature().view(np.uint32))
    finally:
        c1.release()
        c2.release()
