"""The per-context entry points around the step on the GPU: sparse payload
overlays (aero_lbm_step_rect_with_sparse_overlays), the whole-state shift
(aero_lbm_shift_context), point samples, sub-box copies, the cylinder
preset's force (aero_lbm_get_last_force), memory_info,
context_compact_initialized, block edits and the boundary shell of in-place
bricks (native/src/aero_lbm_jni.cpp:1696-1721, 2454-2492, 6156-6540,
8432-8478, 8686-8745, 8899-9244, 9451-9526, 9905-10300).

The reference-order FP32 path is bit-identical to the reference library's
fixtures (ctxops_12.npz, cylinder_44x20x3.npz) in both layouts and launch
shapes, and to the oracle on another seed and call list; FP16 in-place
storage through shifts and overlays stays within the stated tolerance of the
oracle's FP64 run."""
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
_F32P = ctypes.POINTER(ctypes.c_float)


def _fp(a):
    return a.ctypes.data_as(_F32P)


def run_script_gpu(gpu, dims, cfg, pk, script, key, streaming, cpt=2, solver_mode=0, temperature_state=None,
                   collision=0):
    """The product driven through the same call list as oracle.run_script_oracle."""
    nx, ny, nz = dims
    gpu.aero_lbm_b200_set_physics_overrides(-1.0, -1.0, -1)
    gpu.aero_lbm_b200_set_streaming_mode(streaming)
    gpu.aero_lbm_b200_set_collision_mode(collision)
    gpu.aero_lbm_set_realtime_solver_mode(solver_mode)
    assert gpu.aero_lbm_b200_set_cells_per_thread(cpt) == 1
    pk = np.ascontiguousarray(pk, np.float32)
    cells = nx * ny * nz
    results = []
    try:
        ctx = aero_b200.LbmContext(dims, input_channels=pk.shape[1], key=key, lib=gpu)
        if cfg.get("benchmark", True):
            ctx.configure(lbm_cases.product_config(gpu, cfg))
        else:
            gpu.aero_lbm_benchmark_reset_config()  # the game runtime (benchmark mode off)
        if temperature_state is not None:
            ctx.set_temperature_state(temperature_state)
        for act in script:
            kind = act[0]
            if kind == "step":
                ov = act[1] if len(act) > 1 else None
                if ov is None:
                    ctx.step(pk, output=False)
                else:
                    oc = np.ascontiguousarray(ov[0], np.int32)
                    vals = np.ascontiguousarray(ov[1], np.float32)
                    assert gpu.aero_lbm_step_rect_with_sparse_overlays(_fp(pk), nx, ny, nz, key, oc.ctypes.data, _fp(vals),
                                                                       int(oc.size), None) == 1, aero_b200.last_error(gpu)
            elif kind == "cached":
                assert gpu.aero_lbm_step_rect_cached(nx, ny, nz, key, None) == 1, aero_b200.last_error(gpu)
            elif kind == "patch":
                c = np.ascontiguousarray(act[1], np.int32)
                sv = np.ascontiguousarray(act[2], np.uint8)
                fan = np.zeros(c.size, np.uint8)
                assert gpu.aero_lbm_patch_d3q27_f16_static_cells_rect(nx, ny, nz, key, int(c.size), c.ctypes.data,
                                                                      sv.ctypes.data, fan.ctypes.data) == 1, \
                    aero_b200.last_error(gpu)
            elif kind == "mode":
                gpu.aero_lbm_set_realtime_solver_mode(act[1])
            elif kind == "shell":
                fl = np.ascontiguousarray(act[1], np.float32)
                assert gpu.aero_lbm_set_d3q27_f16_boundary_shell_rect(nx, ny, nz, key, _fp(fl), fl.shape[1], act[2],
                                                                      act[3], act[4]) == 1, aero_b200.last_error(gpu)
            elif kind == "flow":
                results.append(ctx.flow_state())
            elif kind == "temp":
                results.append(ctx.temperature_state())
            elif kind == "shift":
                assert gpu.aero_lbm_shift_context(nx, key, *act[1:4]) == 1, aero_b200.last_error(gpu)
            elif kind == "force":
                f = np.zeros(3, np.float32)
                assert gpu.aero_lbm_get_last_force(key, _fp(f[0:]), _fp(f[1:]), _fp(f[2:])) == 1
                results.append(f)
            elif kind == "point":
                fl = np.zeros(4, np.float32)
                t = np.zeros(1, np.float32)
                assert gpu.aero_lbm_sample_flow_point_rect(nx, ny, nz, key, *act[1:4], _fp(fl)) == 1
                assert gpu.aero_lbm_sample_temperature_point_rect(nx, ny, nz, key, *act[1:4], _fp(t)) == 1
                results.append((fl, t))
            elif kind == "subrect":
                n = int(np.prod(act[4:7]))
                fl = np.zeros(n * 4, np.float32)
                t = np.zeros(n, np.float32)
                assert gpu.aero_lbm_copy_flow_temperature_subrect(nx, ny, nz, key, *act[1:7], _fp(fl), _fp(t)) == 1, \
                    aero_b200.last_error(gpu)
                results.append((fl.reshape(-1, 4), t))
            else:
                raise ValueError(kind)
        ctx.release()
    finally:
        gpu.aero_lbm_b200_set_cells_per_thread(2)
        gpu.aero_lbm_set_realtime_solver_mode(0)
        gpu.aero_lbm_b200_set_collision_mode(0)
    assert len(results) == sum(1 for a in script if a[0] not in ("step", "shift", "cached", "patch", "shell", "mode"))
    return results


@pytest.mark.parametrize("streaming,cpt", [(1, 1), (2, 1), (2, 2)])
def test_context_ops_match_reference_golden(gpu, streaming, cpt):
    g = np.load(GOLDEN / "ctxops_12.npz")
    n, seed = int(g["n"]), int(g["seed"])
    obst, u, temp, src, cfg, pre = O.thermal_case(n, seed)
    pk = O.packet_from(obst, *u, temperature=temp, source=src)
    res = run_script_gpu(gpu, (n, n, n), cfg, pk, O.context_ops_script(n), key=800 + 2 * streaming + cpt,
                         streaming=streaming, cpt=cpt, temperature_state=pre)
    flags = O.results_equal(res, O.load_results(GOLDEN / "ctxops_12.npz"))
    assert all(flags), flags


@pytest.mark.parametrize("streaming", [1, 2])
def test_context_ops_match_oracle(gpu, streaming):
    """Another seed and call list: shifts by up to n - 1 cells (a brick that is
    almost all shifted-in rest state), whole-brick sub-box, corner samples."""
    n, seed = 12, 32
    script = [("step",)] * 3 + [("shift", 0, 0, -5), ("point", 11, 11, 11), ("subrect", 0, 0, 0, 12, 12, 12),
                                ("step",), ("shift", 11, 0, 0), ("flow",), ("temp",), ("step",), ("flow",), ("temp",)]
    obst, u, temp, src, cfg, pre = O.thermal_case(n, seed)
    pk = O.packet_from(obst, *u, temperature=temp, source=src)
    res = run_script_gpu(gpu, (n, n, n), cfg, pk, script, key=820 + streaming, streaming=streaming,
                         temperature_state=pre)
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    o.set_temperature(pre)
    flags = O.results_equal(res, O.run_script_oracle(o, cfg, pk, script))
    assert all(flags), flags


def test_context_ops_fp16_against_fp64(gpu):
    """IEEE-half in-place storage through the same shifts and overlays:
    velocity within 1e-3 of the max speed, density within 1e-4, temperature
    within 1e-3 of the oracle's FP64 run, at every flow / temperature read."""
    n, seed = 12, 21
    obst, u, temp, src, cfg, pre = O.thermal_case(n, seed)
    pk = O.packet_from(obst, *u, temperature=temp, source=src)
    script = O.context_ops_script(n)
    res = run_script_gpu(gpu, (n, n, n), cfg, pk, script, key=830, streaming=2, solver_mode=3, temperature_state=pre)
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f64")
    o.set_temperature(pre)
    ref = O.run_script_oracle(o, cfg, pk, script)
    kinds = [a[0] for a in script if a[0] not in ("step", "shift", "cached", "patch", "shell", "mode")]
    for kind, a, b in zip(kinds, res, ref):
        if kind == "flow":
            e = O.flow_errors(a, b)
            assert e["u"] <= 1e-3 and e["rho"] <= 1e-4, e
        elif kind == "temp":
            assert float(np.max(np.abs(a - b))) <= 1e-3


@pytest.mark.parametrize("cpt", [1, 2])
def test_cylinder_force_matches_reference_golden(gpu, cpt):
    """The cylinder crossflow preset: parabolic inflow at x-, convective
    outflow, and the momentum-exchange force on the disc after each call,
    bit-identical to the reference library's fixture."""
    dims = (44, 20, 3)
    cfg, pk = O.cylinder_case(*dims)
    res = run_script_gpu(gpu, dims, cfg, pk, O.CYLINDER_SCRIPT, key=840 + cpt, streaming=0, cpt=cpt)
    flags = O.results_equal(res, O.load_results(GOLDEN / "cylinder_44x20x3.npz"))
    assert all(flags), (flags, res[0])


def test_context_ops_argument_checks(gpu):
    n = 12
    obst, u, temp, src, cfg, pre = O.thermal_case(n, 21)
    pk = O.packet_from(obst, *u, temperature=temp, source=src)
    gpu.aero_lbm_b200_set_streaming_mode(0)
    ctx = aero_b200.LbmContext((n, n, n), key=850, lib=gpu)
    ctx.configure(lbm_cases.product_config(gpu, cfg))
    try:
        f4 = np.zeros(4, np.float32)
        # nothing stepped yet: no flow to sample; the temperature state exists once created
        assert gpu.aero_lbm_sample_flow_point_rect(n, n, n, 850, 0, 0, 0, _fp(f4)) == 0
        ctx.step(pk, output=False)
        assert gpu.aero_lbm_sample_flow_point_rect(n, n, n, 850, n, 0, 0, _fp(f4)) == 0
        assert gpu.aero_lbm_sample_flow_point_rect(n, n, n, 850, 0, -1, 0, _fp(f4)) == 0
        assert gpu.aero_lbm_sample_flow_point_rect(n, n, n, 851, 0, 0, 0, _fp(f4)) == 0
        big = np.zeros(4 * 8, np.float32)
        t = np.zeros(8, np.float32)
        assert gpu.aero_lbm_copy_flow_temperature_subrect(n, n, n, 850, 10, 0, 0, 3, 1, 1, _fp(big), _fp(t)) == 0
        assert gpu.aero_lbm_copy_flow_temperature_subrect(n, n, n, 850, 0, 0, 0, 0, 1, 1, _fp(big), _fp(t)) == 0
        assert gpu.aero_lbm_shift_context(n, 850, n, 0, 0) == 0
        assert gpu.aero_lbm_shift_context(n + 1, 850, 1, 0, 0) == 0
        assert gpu.aero_lbm_shift_context(n, 851, 1, 0, 0) == 0
        assert gpu.aero_lbm_shift_context(n, 850, 0, 0, 0) == 1
        bad_cells = np.zeros(1, np.int32)
        assert gpu.aero_lbm_step_rect_with_sparse_overlays(_fp(pk), n, n, n, 850, bad_cells.ctypes.data, None, 1, None) == 0
        assert gpu.aero_lbm_step_rect_with_sparse_overlays(_fp(pk), n, n, n, 850, None, None, -1, None) == 0
        assert gpu.aero_lbm_step_rect_with_sparse_overlays(_fp(pk), n, n, n, 850, None, None, 0, None) == 1
        fx = np.zeros(1, np.float32)
        assert gpu.aero_lbm_get_last_force(850, _fp(fx), None, None) == 1 and fx[0] == 0.0  # not the cylinder preset
        assert gpu.aero_lbm_get_last_force(851, _fp(fx), None, None) == 0
        assert gpu.aero_lbm_context_compact_initialized(850) == 0
        info = gpu.aero_lbm_memory_info().decode()
        assert info.startswith("gpu_bytes(total=") and "contexts=" in info and "cells=" in info
        total = int(info.split("total=")[1].split(",")[0])
        assert total >= n ** 3 * 27 * 2
    finally:
        ctx.release()


@pytest.mark.parametrize("cpt", [1, 2])
def test_block_edits_and_shell_match_oracle(gpu, cpt):
    """In-place FP32 (reference-order collision): block edits between calls
    (cached steps after them, duplicates, out-of-range indices, solid cells
    opened and fluid ones closed) and the boundary shell, bit-identical to
    the oracle's restatement of the same operations. The context is created
    by a classic-mode call (FP32 storage); the later calls run in the FP16
    in-place solver mode, the only mode whose step applies the shell."""
    n = 12
    obst, u, temp, src, cfg, pre = O.thermal_case(n, 41)
    pk = O.packet_from(obst, *u, temperature=temp, source=src)
    ops = O.edits_script(n)
    script = ops[:1] + [("mode", 3)] + ops[1:]
    res = run_script_gpu(gpu, (n, n, n), cfg, pk, script, key=860 + cpt, streaming=2, cpt=cpt, temperature_state=pre)
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    o.set_temperature(pre)
    flags = O.results_equal(res, O.run_script_oracle(o, cfg, pk, script))
    assert all(flags), flags


def test_shell_ignored_outside_the_fp16_mode(gpu):
    """Calls in the classic solver mode leave the shell unapplied (the
    reference reads it in its FP16 in-place step only): the edit script with
    its shells, run in mode 0, equals the oracle's run without them."""
    n = 12
    obst, u, temp, src, cfg, pre = O.thermal_case(n, 41)
    pk = O.packet_from(obst, *u, temperature=temp, source=src)
    script = O.edits_script(n)
    res = run_script_gpu(gpu, (n, n, n), cfg, pk, script, key=869, streaming=2, cpt=2, temperature_state=pre)
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    o.set_temperature(pre)
    flags = O.results_equal(res, O.run_script_oracle(o, cfg, pk, [a for a in script if a[0] != "shell"]))
    assert all(flags), flags


def test_block_edits_and_shell_fp16_against_fp64(gpu):
    n = 12
    obst, u, temp, src, cfg, pre = O.thermal_case(n, 41)
    pk = O.packet_from(obst, *u, temperature=temp, source=src)
    script = O.edits_script(n)
    res = run_script_gpu(gpu, (n, n, n), cfg, pk, script, key=865, streaming=2, solver_mode=3, temperature_state=pre)
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f64")
    o.set_temperature(pre)
    ref = O.run_script_oracle(o, cfg, pk, script)
    kinds = [a[0] for a in script if a[0] in ("flow", "temp", "point", "subrect", "force")]
    for kind, a, b in zip(kinds, res, ref):
        if kind == "flow":
            e = O.flow_errors(a, b)
            assert e["u"] <= 1e-3 and e["rho"] <= 1e-4, e
        elif kind == "temp":
            assert float(np.max(np.abs(a - b))) <= 1e-3


def test_block_edits_and_shell_argument_checks(gpu):
    n = 12
    obst, u, temp, src, cfg, pre = O.thermal_case(n, 41)
    pk = O.packet_from(obst, *u, temperature=temp, source=src)
    c = np.array([5, 6], np.int32)
    sv = np.array([1, 0], np.uint8)
    fan = np.zeros(2, np.uint8)
    flow = np.zeros((n ** 3, 4), np.float32)
    patch = gpu.aero_lbm_patch_d3q27_f16_static_cells_rect
    shell = gpu.aero_lbm_set_d3q27_f16_boundary_shell_rect
    for streaming, key in ((1, 870), (2, 871)):
        gpu.aero_lbm_b200_set_streaming_mode(streaming)
        ctx = aero_b200.LbmContext((n, n, n), key=key, lib=gpu)
        ctx.configure(lbm_cases.product_config(gpu, cfg))
        try:
            assert patch(n, n, n, key, 2, c.ctypes.data, sv.ctypes.data, fan.ctypes.data) == 0  # no context yet
            ctx.step(pk, output=False)
            assert patch(n, n, n, key, 0, None, None, None) == 1
            assert patch(n, n, n, key, 2, c.ctypes.data, sv.ctypes.data, None) == 0
            assert "missing patch arrays" in aero_b200.last_error(gpu)
            assert patch(n, n, n + 1, key, 2, c.ctypes.data, sv.ctypes.data, fan.ctypes.data) == 0
            assert shell(n, n, n, key, _fp(flow), 3, 1, 2, 0.2) == 0
            assert shell(n, n, n, key, _fp(flow), 4, 0, 2, 0.2) == 1  # empty mask clears
            ok = streaming == 2
            assert patch(n, n, n, key, 2, c.ctypes.data, sv.ctypes.data, fan.ctypes.data) == (1 if ok else 0)
            assert shell(n, n, n, key, _fp(flow), 4, 1, 2, 0.2) == (1 if ok else 0)
            if ok:
                # staged edits block a shift until the next call
                assert gpu.aero_lbm_shift_context(n, key, 1, 0, 0) == 0
                assert gpu.aero_lbm_step_rect_cached(n, n, n, key, None) == 1
                assert gpu.aero_lbm_shift_context(n, key, 1, 0, 0) == 1
            assert gpu.aero_lbm_clear_d3q27_f16_boundary_shell_rect(key) == 1
            assert gpu.aero_lbm_clear_d3q27_f16_boundary_shell_rect(99999) == 1
        finally:
            ctx.release()


@pytest.mark.parametrize("streaming,cpt", [(1, 1), (2, 1), (2, 2)])
def test_fans_and_sponge_match_reference_golden(gpu, streaming, cpt):
    """Fan forcing with noise and the sponge (their DISABLE flags cleared), in
    both layouts; the runtime terms take the one-cell kernels whatever the
    launch-shape setting. Bit-identical to fixture fans_12_12.npz."""
    cfg, pk, pre = O.fan_case(12, 61)
    res = run_script_gpu(gpu, (12, 12, 12), cfg, pk, O.FAN_SCRIPT, key=880 + 2 * streaming + cpt, streaming=streaming,
                         cpt=cpt, temperature_state=pre)
    flags = O.results_equal(res, O.load_results(GOLDEN / "fans_12_12.npz"))
    assert all(flags), flags


def test_fans_and_sponge_fp16_against_fp64(gpu):
    cfg, pk, pre = O.fan_case(12, 61)
    res = run_script_gpu(gpu, (12, 12, 12), cfg, pk, O.FAN_SCRIPT, key=890, streaming=2, solver_mode=3,
                         temperature_state=pre)
    o = O.Oracle((12, 12, 12), O.derive_params(cfg), "f64")
    o.set_temperature(pre)
    ref = O.run_script_oracle(o, cfg, pk, O.FAN_SCRIPT)
    for kind, a, b in zip(("flow", "temp", "flow"), res, ref):
        if kind == "flow":
            e = O.flow_errors(a, b)
            assert e["u"] <= 1e-3 and e["rho"] <= 1e-4, e
        else:
            assert float(np.max(np.abs(a - b))) <= 1e-3


@pytest.mark.parametrize("collision", [0, 1])
def test_runtime_mode_matches_reference_golden(gpu, collision):
    """Benchmark mode off, as the reference's brick service runs the step:
    fans with noise, sponge, state nudge, the every-other-call BFECC
    transport with eddy diffusivity, convective outflow faces (two-buffer
    layout). The reference-order collision is bit-identical to fixture
    runtime_12_8.npz; the factorised one agrees to FP32 rounding."""
    cfg, pk, pre = O.runtime_case(12, 71)
    res = run_script_gpu(gpu, (12, 12, 12), cfg, pk, O.RUNTIME_SCRIPT, key=900 + collision, streaming=0,
                         temperature_state=pre, collision=collision)
    ref = O.load_results(GOLDEN / "runtime_12_8.npz")
    if collision == 0:
        flags = O.results_equal(res, ref)
        assert all(flags), flags
    else:
        for kind, a, b in zip(("flow", "temp") * 3, res, ref):
            if kind == "flow":
                e = O.flow_errors(a, b)
                assert e["u"] <= 1e-5 and e["rho"] <= 1e-6, e
            else:
                assert float(np.max(np.abs(a - b))) <= 1e-5


@pytest.mark.parametrize("channels", [9, 10])
def test_short_packets_match_oracle(gpu, channels):
    """Runtime mode with 9- or 10-channel packets: no temperature channel, and
    with 9 channels the temperature source derived from the fan channels
    (sparse overlays on fan cells keep it)."""
    cfg, pk, pre = O.runtime_case(12, 77, True, channels)
    script = O.short_packet_script(pk)
    res = run_script_gpu(gpu, (12, 12, 12), cfg, pk, script, key=910 + channels, streaming=0, temperature_state=pre)
    o = O.Oracle((12, 12, 12), O.derive_params(cfg), "f32")
    o.set_temperature(pre)
    flags = O.results_equal(res, O.run_script_oracle(o, cfg, pk, script))
    assert all(flags), flags
