"""Benchmark of the B200 D3Q27 brick step (MLUPS and fraction of the HBM roofline).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one GPU): the 128^3 terrain brick with Boussinesq buoyancy (seeded
4-octave heightmap, inflow (0.08, 0.02, 0) at x-, convective outflow at x+,
far-field lid, Smagorinsky C = 0.1, g*beta = 1e-4 along +z, the temperature
transported before every collision), stepped by the library's fused
pull-stream + cumulant-collide kernel with 16-bit fixed-point deviation
storage (the default format of the FP16 solver mode). Inputs are seeded
synthetic data of the benchmark's shape (no dataset exists).

value : device-resident MLUPS (state in HBM, one fused launch per step, CUDA
        events on the launching stream; the state is larger than L2). Each
        variant's window of K steps is repeated until the windows cover at
        least a second; the median window is reported.
e2e   : the same metric through the reference-facing C ABI with host buffers:
        every step uploads the 11-channel packet from pinned memory
        (aero_lbm_step_rect) and reads back the stride-4 velocity atlas
        (aero_lbm_extract_flow_atlas_rect). config.e2e_resident: the cached
        step (aero_lbm_step_rect_cached) + atlas; config.brick_world: the
        native brick-world service (aero_lbm_simulation_*) on the same terrain
        as eight 64^3 bricks, a tick + eight int16 atlases per step.
--impl reference: the reference's own CPU step (oracle/_ref, built from the
        reference sources) on the box's host cores, one single-threaded process
        per core, each stepping the same 128^3 brick.

With torchrun (N > 1) every rank steps its own brick (bricks are independent
work units; no data-path collective), timing is the max over ranks and value
is the aggregate.
"""
from __future__ import annotations

import argparse
import ctypes
import dataclasses
import importlib.util
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "aerodynamics4mc-fabric_b200"
METRIC = "D3Q27 cumulant MLUPS and % of HBM peak, FP16-store vs FP32 at stated error"
BYTES_PER_CELL_FP32 = 217.0  # 27*4 read + 27*4 write + 1 mask byte per cell-step


def load_pkg():
    if "aero_b200" in sys.modules:
        return sys.modules["aero_b200"]
    spec = importlib.util.spec_from_file_location("aero_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["aero_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_cases():
    spec = importlib.util.spec_from_file_location("aero_b200_cases", PKG_DIR / "cases.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["aero_b200_cases"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def traffic_record(kernel: str) -> float | None:
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        rec = json.loads(p.read_text()).get(kernel)
        return float(rec["bytes_per_launch"]) if rec else None
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.file:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for name, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- reference arm (CPU)
# Steps per reference process: each is ~5 s of one core on the 128^3 brick, so
# a run of K steps is bounded to keep the arm within a few minutes.
REF_MAX_STEPS = 20


def host_cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.lower().startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _ref_worker(args):
    """One process: the reference CPU step on the benchmark's 128^3 brick
    (same packet, configuration and starting temperature as our arm)."""
    steps, warmup, n = args
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    cases = load_cases()
    case = cases.c2_terrain_boussinesq(n)
    cfg = case.config_dict()
    ref = O.RefLib()
    lib = ref.lib
    lib.aero_lbm_init_rect(n, n, n, 11, 4)
    c = O.config_struct(O.RefBenchmarkConfig, cfg, lib.aero_lbm_benchmark_default_config)
    lib.aero_lbm_benchmark_set_config(ctypes.byref(c))
    lib.aero_lbm_set_temperature_state_rect(n, n, n, 1, np.ascontiguousarray(case.temperature.reshape(-1)).ctypes.data)
    pk = np.ascontiguousarray(case.packet())
    for _ in range(warmup):
        lib.aero_lbm_step_rect(pk.ctypes.data, n, n, n, 1, None)
    t0 = time.perf_counter()
    for _ in range(steps):
        lib.aero_lbm_step_rect(pk.ctypes.data, n, n, n, 1, None)
    dt = time.perf_counter() - t0
    return n ** 3 * steps / dt / 1e6


def _run_ref_processes(procs: int, steps: int, warmup: int, n: int) -> tuple[list, float]:
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        t0 = time.perf_counter()
        per = pool.map(_ref_worker, [(steps, warmup, n)] * procs)
        wall = time.perf_counter() - t0
    return per, wall


def run_reference_arm(steps: int, warmup: int, n: int = 128, procs: int | None = None) -> dict:
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    if not O.REF_LIB.exists():
        return {"impl": "reference", "unavailable": "oracle/_ref/libaero_lbm_ref.so was not built (reference sources absent)"}
    cores = procs or max(1, min(os.cpu_count() or 1, 16))
    ref_steps = max(1, min(steps, REF_MAX_STEPS))
    per, wall = _run_ref_processes(cores, ref_steps, min(warmup, 1), n)
    value = float(sum(per))
    cpu = host_cpu_model()
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "MLUPS",
        "n_gpus": 0,
        "steps": ref_steps,
        "warmup": min(warmup, 1),
        "ms_per_step": n ** 3 / (value / cores * 1e6) * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded terrain, heightmap, temperature field)",
        "config": {"workload": f"d3q27-cumulant {n}^3 terrain brick, SGS C=0.1, Boussinesq g*beta=1e-4, "
                               "outflow x+, temperature transport; reference CPU step",
                   "processes": cores, "same_config": True, "host_cpu": cpu},
        "cpu_baseline": {"value": value, "unit": "MLUPS", "cores": cores, "kind": "reference", "host_cpu": cpu,
                         "sample": f"{cores} single-threaded processes x {ref_steps} steps of the {n}^3 brick "
                                   f"(steps bounded to {REF_MAX_STEPS}; {wall:.1f}s wall)"},
        "e2e": {"value": value, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def cpu_baseline_single(n: int = 128, steps: int = 3) -> dict | None:
    """Reference CPU step, one core, a bounded sample of the same workload
    (a few steps of the 128^3 brick, ~15-20 s)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    if not O.REF_LIB.exists():
        return None
    per, wall = _run_ref_processes(1, steps, 1, n)
    return {"value": per[0], "unit": "MLUPS", "cores": 1, "kind": "reference", "host_cpu": host_cpu_model(),
            "sample": f"{steps} steps of the {n}^3 brick after one warm-up step, single-threaded reference CPU step "
                      f"({wall:.1f}s wall)"}


# ---------------------------------------------------------------- our arm
# Temperature transport per cell and step: state read + write (2 x 4 B) and
# the previous collision's velocity written by the collision and read by the
# transport (2 x 12 B). With the transport inside the step kernel all of them
# are that kernel's traffic; with the separate pass the step kernel reads the
# new temperature and writes the velocity (4 + 12 B).
THERMAL_BYTES = {True: 2 * 4 + 2 * 12, False: 4 + 12}
VARIANTS = {
    # name: (realtime solver mode, collision mode, 16-bit format, bytes per cell-step, storage note)
    "i16": (3, 1, 1, 27 * 2 * 2 + 1, "16-bit fixed-point deviation storage (the FP16 mode's default format), "
                                     "in-place esoteric pull, factorised collision, two cells per thread in packed FP32"),
    "fp16": (3, 1, 0, 27 * 2 * 2 + 1, "IEEE-half deviation storage, in-place esoteric pull, factorised collision"),
    "fp32_exact": (0, 0, 1, 27 * 4 * 2 + 1, "fp32, in-place esoteric pull, reference-order collision (bit-exact)"),
    "fp32_fast": (0, 1, 1, 27 * 4 * 2 + 1, "fp32, in-place esoteric pull, factorised collision"),
}
HEADLINE = "i16"


def setup_context(aero, lib, case, variant: str, key: int, streaming: int, thermal: int = -1):
    """A context of the case stepped once (with a pinned host packet). thermal:
    the temperature-transport mode (aero_lbm_b200_set_thermal_transport) left
    set for the context's later steps; with the transport the case's
    temperature field is loaded as the starting state."""
    import torch

    solver_mode, collision, fmt, _, _ = VARIANTS[variant]
    lib.aero_lbm_set_realtime_solver_mode(solver_mode)
    lib.aero_lbm_b200_set_fp16_format(fmt)
    lib.aero_lbm_b200_set_collision_mode(collision)
    lib.aero_lbm_b200_set_physics_overrides(case.smagorinsky_c, case.buoyancy_beta, case.gravity_axis)
    lib.aero_lbm_b200_set_streaming_mode(streaming)
    n = case.dims[0]
    ctx = aero.LbmContext(case.dims, key=key, lib=lib, init=False)
    cfgd = case.config_dict()
    cfg = aero.default_config(lib)
    cfg.enabled = 1
    cfg.flags = cfg.flags & ~aero.FLAG_DISABLE_SGS & ~aero.FLAG_DISABLE_BUOYANCY | aero.FLAG_DISABLE_INTERNAL_THERMAL_SOURCE
    cfg.reynolds_number = cfgd["reynolds"]
    for i, v in enumerate(case.u_ref):
        cfg.initial_velocity[i] = v
    for face, fc in zip(cfg.faces(), case.faces):
        face.hydrodynamic_kind = fc["kind"]
        face.thermal_kind = 1
        for a, v in enumerate(fc.get("velocity", (0, 0, 0))):
            face.velocity[a] = v
    ctx.configure(cfg)
    lib.aero_lbm_b200_set_thermal_transport(thermal)
    if thermal != 0 and case.temperature_state() is not None:
        ctx.set_temperature_state(case.temperature_state())
    packet = torch.from_numpy(case.packet()).pin_memory()
    pk_ptr = ctypes.cast(packet.data_ptr(), ctypes.POINTER(ctypes.c_float))
    if not lib.aero_lbm_step_rect(pk_ptr, n, n, n, key, None):
        raise RuntimeError(aero.last_error(lib))
    lib.aero_lbm_set_realtime_solver_mode(0)
    lib.aero_lbm_b200_set_collision_mode(0)
    lib.aero_lbm_b200_set_fp16_format(1)
    return ctx, packet, pk_ptr


def run_brick_world_leg(aero, lib, case, ticks: int, warmup: int, stride: int = 4) -> dict:
    """The native brick-world service (aero_lbm_simulation_*, what the mod's
    ClientL2Solver calls through JNI) on the benchmark's terrain split into
    eight 64^3 bricks (a 2 x 2 x 2 world): the reference service's game-runtime
    physics in its classic solver mode (fans, edge nudge, sponge, the
    every-other-tick temperature transport, halo exchanges between the bricks).
    A step = one tick + the eight stride-4 int16 atlases read back."""
    n = case.dims[0] // 2
    svc = aero.BrickWorldService(lib)
    try:
        svc.ensure_world(1, n, dx=1.0, dt=0.05, solver_mode=1)
        coords = [(bx, by, bz) for bx in range(2) for by in range(2) for bz in range(2)]
        svc.set_hints(1, coords)
        flow = np.zeros(case.dims + (4,), np.float32)
        for a in range(3):
            flow[..., a] = case.u[a]
        for (bx, by, bz) in coords:
            sl = (slice(bx * n, (bx + 1) * n), slice(by * n, (by + 1) * n), slice(bz * n, (bz + 1) * n))
            svc.upload_static(1, (bx, by, bz), case.obstacle[sl])
            svc.upload_dynamic(1, (bx, by, bz), flow[sl], case.temperature[sl])
        res = (n + stride - 1) // stride
        atlases = [np.zeros(res ** 3 * 4, np.int16) for _ in coords]
        for _ in range(warmup):
            svc.step(1, 1)
        launches0 = lib.aero_lbm_b200_launch_count()
        t0 = time.perf_counter()
        for _ in range(ticks):
            svc.step(1, 1)
            for c, out in zip(coords, atlases):
                svc.atlas(1, c, stride, out)
        dt = time.perf_counter() - t0
        launches = lib.aero_lbm_b200_launch_count() - launches0
        status = svc.status(1).tolist()
    finally:
        svc.release()
    cells = len(coords) * n ** 3
    return {"workload": f"brick world 2x2x2 of {n}^3 bricks (the terrain brick split), classic solver mode, "
                        "game-runtime physics, exact hints",
            "api": "aero_lbm_simulation_step_brick_world_runtime + copy_brick_world_packed_flow_atlas (stride 4)",
            "cells_per_tick": cells, "ticks": ticks, "ms_per_tick": dt / ticks * 1e3,
            "mlups": cells * ticks / dt / 1e6, "d2h_bytes_per_tick": int(sum(a.nbytes for a in atlases)),
            "h2d_bytes_per_tick": 0, "launches_per_tick": launches / ticks, "status": status}


def run_batch_leg(aero, lib, torch, stream, ticks: int, warmup: int) -> dict:
    """C4: 400 x 32^3 + 80 x 64^3 + 32 x 128^3 bricks (seeded masks with solid
    fraction U[0, 0.15], tau U[0.51, 0.6], body force U[-1e-5, 1e-5]^3),
    alternating FP32 / FP16 storage, periodic x/y and bounce-back z faces, one
    persistent launch + stride-4 int16 publish per tick, graph replay,
    autotuned launch shape."""
    rng = np.random.default_rng(4)
    b = aero.BrickBatch(lib)
    sizes = [32] * 400 + [64] * 80 + [128] * 32
    faces = [1, 1, 1, 1, 2, 2]
    for i, n in enumerate(sizes):
        frac = rng.uniform(0.0, 0.15)
        obst = (rng.random((n, n, n), dtype=np.float32) < frac).astype(np.uint8)
        obst[:, :, 0] = 1
        b.add_brick((n, n, n), obst, None, float(rng.uniform(0.51, 0.6)), rng.uniform(-1e-5, 1e-5, 3), faces,
                    precision=i % 2)
    b.finalize(stride=4, velocity_scale=20.0)
    b.set_options(use_graph=True, publish=True)
    info = b.info()
    threads, bps, tune_ms = b.autotune(trial_ticks=4)
    b.tick(warmup + (warmup & 1))
    torch.cuda.synchronize()
    launches0 = lib.aero_lbm_b200_launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    b.tick(ticks)
    end.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    launches = lib.aero_lbm_b200_launch_count() - launches0
    b.close()
    cells = info["cells"]
    return {"workload": "512 bricks (400 x 32^3, 80 x 64^3, 32 x 128^3), alternating fp32/fp16, per-brick mask/tau/force",
            "cells_per_tick": cells, "ticks": ticks, "ms_per_tick": ms / ticks,
            "mlups": cells * ticks / (ms * 1e-3) / 1e6,
            "achieved_gbs": info["bytes_per_tick"] * ticks / (ms * 1e-3) / 1e9,
            "bytes_per_tick": info["bytes_per_tick"], "autotuned": {"threads": threads, "blocks_per_sm": bps},
            "graph": True, "publish_stride": 4, "launches_in_timed_region": int(launches)}


def run_meso_leg(aero, lib, torch, stream, steps: int, warmup: int) -> dict:
    """C3: D3Q19 mesoscale grid 256 x 64 x 256 (y up): seeded terrain up to 12
    cells as the bounce-back ground, free-slip lid, periodic sides, body force
    (1e-6, 0, 0), log-profile initial wind, tau 0.52 + Smagorinsky, the
    hydrodynamic distribution in one fused launch per step. Variants: FP32 in
    the reference order (bit-identical to the restatement), and the packed
    two-cell step with FP32, FP16 and 16-bit fixed-point storage; `steps`
    steps each from the seeded state, and each variant's wind difference from
    the reference-order FP32 run at the end."""
    cases = load_cases()
    c = cases.c3_meso_terrain(steps=steps)
    variants = {"fp32": (0, 0), "fp32_packed": (0, 1), "fp16": (1, 1), "i16": (2, 1)}
    res, states = {}, {}
    for name, (storage, collision) in variants.items():
        ctx = aero.MesoscaleContext(c.dims, dx_m=c.dx_m, dt_s=c.dt_s,
                                    options={**c.options, "storage": storage, "collision": collision})
        ctx.step(c.forcing)
        ctx.advance(warmup)
        torch.cuda.synchronize()
        launches0 = lib.aero_lbm_b200_launch_count()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        ctx.advance(steps)
        end.record(stream)
        torch.cuda.synchronize()
        ms = start.elapsed_time(end)
        info = ctx.info()
        states[name] = ctx.state()
        ctx.release()
        res[name] = {"mlups": c.cells * steps / (ms * 1e-3) / 1e6, "ms_per_step": ms / steps,
                     "achieved_gbs": info["bytes_per_step"] / (ms / steps * 1e-3) / 1e9,
                     "bytes_per_cell": info["bytes_per_step"] / c.cells,
                     "launches": int(lib.aero_lbm_b200_launch_count() - launches0)}
    ref = states["fp32"][:, 3:].astype(np.float64)
    wmax = float(np.max(np.abs(ref)))
    out = {"workload": "d3q19 256x64x256 (y up) terrain <= 12 cells, free-slip lid, periodic sides, "
                       "force (1e-6,0,0), tau 0.52 + SGS C=0.1, hydrodynamic distribution",
           "steps": steps + warmup + 1, "timed_steps": steps, **{f"{k}_{m}": v[m] for k, v in res.items() for m in v}}
    for name in ("fp32_packed", "fp16", "i16"):
        out[f"{name}_vs_fp32_wind_rel"] = float(np.max(np.abs(states[name][:, 3:] - ref))) / wmax if wmax > 0 else None
    out["fp16_over_fp32"] = res["fp16"]["mlups"] / res["fp32"]["mlups"]
    return out


def run_adjoint_leg(aero, lib, torch) -> dict:
    """C5: 64^3 FP32 brick (SGS, Boussinesq, 5% obstacles), 200 calls with a
    checkpoint every 20; loss = squared velocity mismatch at 64 probes against
    a hidden run with a smooth random body-force field; gradient with respect
    to the force field and the inflow vector. Reports the device time per call
    of the forward, of the segment recomputation and of the reverse launch."""
    cases = load_cases()
    c = cases.c5_adjoint()
    b = aero.AdjointBrick(c.obstacle, c.temperature, lib=lib, **c.config)
    b.set_probes(c.probes, np.zeros((len(c.probes), 3), np.float32))
    _, t = b.forward(c.force_true, c.inflow_true, precision=1)
    b.set_probes(c.probes, t)
    b.gradient(c.force0, c.inflow0)  # warm-up
    loss, gf, gu = b.gradient(c.force0, c.inflow0)
    tm = b.timing()
    b.close()
    fwd = tm["forward_ms_per_step"]
    per_step = tm["recompute_ms_per_step"] + tm["reverse_ms_per_step"]
    # Every state kept (checkpoint every call: 200 x 28 MB of FP32 state, well
    # within one GPU's memory): no segment recomputation.
    cfg1 = dict(c.config, checkpoint_every=1)
    b1 = aero.AdjointBrick(c.obstacle, c.temperature, lib=lib, **cfg1)
    b1.set_probes(c.probes, t)
    b1.gradient(c.force0, c.inflow0)  # warm-up
    loss1, gf1, gu1 = b1.gradient(c.force0, c.inflow0)
    tm1 = b1.timing()
    b1.close()
    fwd1 = tm1["forward_ms_per_step"]
    per_step1 = tm1["recompute_ms_per_step"] + tm1["reverse_ms_per_step"]
    return {"workload": "d3q27 64^3 fp32, SGS + Boussinesq + 5% obstacles, 200 calls, checkpoint every 20, 64 probes",
            "loss": loss, "grad_inflow": [float(v) for v in gu], "grad_force_max": float(np.max(np.abs(gf))),
            **tm, "adjoint_over_forward": per_step / fwd if fwd > 0 else None,
            "reverse_only_over_forward": tm["reverse_ms_per_step"] / fwd if fwd > 0 else None,
            "store_all": {"checkpoint_every": 1, "adjoint_over_forward": per_step1 / fwd1 if fwd1 > 0 else None,
                          "forward_ms_per_step": fwd1, "reverse_ms_per_step": tm1["reverse_ms_per_step"],
                          "gradient_equal_to_checkpointed": bool(np.array_equal(gf1, gf) and np.array_equal(gu1, gu))}}


def rank_max(value: float, world: int, dist_mod=None, device=None) -> float:
    """The maximum of `value` over the ranks of the process group (every rank
    calls it with its own value); one rank returns its value untouched."""
    if world <= 1:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist_mod.all_reduce(t, op=dist_mod.ReduceOp.MAX)
    return float(t.item())


def window_count(first_window_ms: float, world: int, dist_mod=None, device=None) -> int:
    """Timed windows of a variant: enough to cover about a second at the
    first window's length (3..5000), the same count on every rank."""
    own = float(min(5000, max(3, -(-1000.0 // max(first_window_ms, 1e-3)))))
    return int(rank_max(own, world, dist_mod, device))


def run_ours(args) -> dict | None:
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    aero = load_pkg()
    cases = load_cases()
    lib = aero.load_library()
    # A dedicated stream: the library queues every kernel on it and the CUDA
    # events below are recorded on it (a null handle would select the
    # library's own stream instead).
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    lib.aero_lbm_b200_set_stream(ctypes.c_void_p(stream.cuda_stream))
    if not lib.aero_lbm_init_rect(args.n, args.n, args.n, 11, 4):
        raise RuntimeError(aero.last_error(lib))
    lib.aero_lbm_b200_set_fused_transport(args.fused_transport)

    case = cases.c2_terrain_boussinesq(args.n)
    if args.brick_world_only:
        # profiling entry: the brick-world leg alone, its record printed
        return {"brick_world": run_brick_world_leg(aero, lib, case, max(5, min(args.steps, 40)), args.warmup)}
    n = args.n
    cells = case.cells

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(v: float) -> float:
        return rank_max(v, world, dist, dev)

    def timed(variant: str, key: int, steps: int):
        """Windows of `steps` device-resident steps (one library call that
        advances the context `steps` times), repeated until they cover at
        least a second (3..5000 windows, the same count on every rank); the
        median window, each window's time the max over ranks. The step-kernel
        time comes from three further windows with the library's per-launch
        event timer on (not part of the step windows)."""
        ctx, packet, pk_ptr = setup_context(aero, lib, case, variant, key, args.streaming)
        for _ in range(args.warmup):
            ctx.advance(1)
        barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        window_ms, launches = [], 0
        with ClockSampler(local) as clk:
            windows = 3
            while len(window_ms) < windows:
                launches0 = lib.aero_lbm_b200_launch_count()
                barrier()
                start.record(stream)
                ctx.advance(steps)
                end.record(stream)
                barrier()
                launches = lib.aero_lbm_b200_launch_count() - launches0
                window_ms.append(max_over_ranks(start.elapsed_time(end)))
                if len(window_ms) == 1:
                    windows = window_count(window_ms[0], world, dist, dev)
        lib.aero_lbm_b200_kernel_timer(1)  # events around each step-kernel launch, on the library's stream
        for _ in range(3):
            ctx.advance(steps)
        barrier()
        kms, kn = ctypes.c_double(0.0), ctypes.c_int(0)
        lib.aero_lbm_b200_kernel_time(ctypes.byref(kms), ctypes.byref(kn))
        lib.aero_lbm_b200_kernel_timer(0)
        kernel_ms = max_over_ranks(kms.value / max(1, kn.value))
        ms = statistics.median(window_ms)
        return ctx, packet, pk_ptr, ms, launches, clk.summary(), kernel_ms, window_ms

    results = {}
    head = None
    for variant in [HEADLINE] + [v for v in args.variants if v != HEADLINE]:
        steps = args.steps
        ctx, packet, pk_ptr, ms, launches, clocks, kernel_ms, windows = timed(variant, 1 + rank * 8 + len(results), steps)
        ms_step = ms / steps
        nbytes = VARIANTS[variant][3]
        # achieved_gbs: the stream-collide kernel's algorithmic bytes (the
        # populations plus its share of the transport's fields) over its own
        # launch time; step_gbs: the whole step's bytes (populations and every
        # transport byte) over the step time (kernel, transport pass if
        # separate, per-call boundary fill).
        kb = nbytes + THERMAL_BYTES[bool(args.fused_transport)]
        results[variant] = {"mlups": cells * world * steps / (ms * 1e-3) / 1e6, "ms_per_step": ms_step,
                            "launches": launches, "clocks": clocks, "steps": steps, "kernel_ms": kernel_ms,
                            "windows": len(windows), "window_ms_min": min(windows), "window_ms_max": max(windows),
                            "achieved_gbs": kb * cells / (kernel_ms * 1e-3) / 1e9,
                            "population_gbs": nbytes * cells / (kernel_ms * 1e-3) / 1e9,
                            "step_gbs": (nbytes + THERMAL_BYTES[True]) * cells / (ms_step * 1e-3) / 1e9}
        if variant == HEADLINE:
            head = (ctx, packet, pk_ptr)
        else:
            ctx.release()

    # e2e through the C ABI with host buffers (headline brick): per step the
    # pinned 11-channel packet goes up (aero_lbm_step_rect) and the stride-4
    # velocity atlas comes back (aero_lbm_extract_flow_atlas_rect).
    ctx, packet, pk_ptr = head
    stride = 4
    atlas = np.zeros(((n + stride - 1) // stride) ** 3 * 4, np.float32)
    e2e_steps = max(3, min(args.steps, 50))

    def e2e_run(cached: bool) -> float:
        for _ in range(2):
            ok = (lib.aero_lbm_step_rect_cached(n, n, n, ctx.key, None) if cached
                  else lib.aero_lbm_step_rect(pk_ptr, n, n, n, ctx.key, None))
            if not ok or not lib.aero_lbm_extract_flow_atlas_rect(n, n, n, ctx.key, stride, aero.fptr(atlas), atlas.size):
                raise RuntimeError(aero.last_error(lib))
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            ok = (lib.aero_lbm_step_rect_cached(n, n, n, ctx.key, None) if cached
                  else lib.aero_lbm_step_rect(pk_ptr, n, n, n, ctx.key, None))
            if not ok or not lib.aero_lbm_extract_flow_atlas_rect(n, n, n, ctx.key, stride, aero.fptr(atlas), atlas.size):
                raise RuntimeError(aero.last_error(lib))
        barrier()
        return cells * world * e2e_steps / max_over_ranks(time.perf_counter() - t0) / 1e6

    e2e_value = e2e_run(False)
    e2e_resident = e2e_run(True)
    ctx.release()

    # Accuracy: every variant after `accuracy_steps` calls from the same
    # inputs against the FP64 run of the same scheme on the GPU (the adjoint
    # module's forward in double precision, every fluid cell probed). That
    # forward holds the temperature fixed and has no outflow face, so this leg
    # runs the brick with an equilibrium x+ face and without the transport;
    # the configured case (outflow, transport) is checked against the
    # oracle's FP64 run at 64^3 x 1000 in tests/test_fp16_c2_gpu.py.
    acc = None
    if args.accuracy_steps > 0:
        far = {"kind": 4, "velocity": case.u_ref}
        acase = dataclasses.replace(case, faces=[case.faces[0], far] + list(case.faces[2:]))
        outs = {}
        for k, variant in enumerate(("i16", "fp16", "fp32_fast", "fp32_exact")):
            c, _, _ = setup_context(aero, lib, acase, variant, 90 + 8 * rank + k, args.streaming, thermal=0)
            c.advance(args.accuracy_steps - 1)
            outs[variant] = c.flow_state()
            c.release()
        lib.aero_lbm_b200_set_thermal_transport(-1)
        fluid = np.flatnonzero(acase.obstacle.reshape(-1) == 0).astype(np.int32)
        ab = aero.AdjointBrick(acase.obstacle, acase.temperature, lib=lib, face_kind=[f["kind"] for f in acase.faces],
                               tau=acase.tau, smagorinsky_c=acase.smagorinsky_c, buoyancy_beta=acase.buoyancy_beta,
                               steps=args.accuracy_steps, checkpoint_every=20)
        ab.set_probes(fluid, np.zeros((fluid.size, 3), np.float32))
        _, u64 = ab.forward(None, acase.u_ref, precision=1)
        ab.close()
        speed64 = float(np.max(np.linalg.norm(u64.astype(np.float64), axis=1)))
        ref = outs["fp32_exact"].astype(np.float64)
        speed = float(np.max(np.linalg.norm(ref[:, :3], axis=1)))
        acc = {"steps": args.accuracy_steps,
               **{f"{v}_vs_fp64_u": float(np.max(np.abs(outs[v][fluid, :3] - u64))) / speed64 for v in outs},
               **{f"{v}_vs_fp32_exact_u": float(np.max(np.abs(outs[v][:, :3] - ref[:, :3]))) / speed
                  for v in ("i16", "fp16", "fp32_fast")},
               "i16_vs_fp32_exact_rho": float(np.max(np.abs(outs["i16"][:, 3] - ref[:, 3]))) / float(np.max(1 + ref[:, 3])),
               "metric": "max |u - u64| / max |u64| over fluid cells",
               "fp64_reference": "the library's double-precision forward (adjoint module) on the GPU",
               "case": f"the {n}^3 terrain brick with an equilibrium x+ face and the temperature held fixed",
               "configured_case_check": "tests/test_fp16_c2_gpu.py: default 16-bit format vs the oracle's FP64 run, "
                                        "64^3, outflow x+, temperature transport, 1000 steps, bound 1e-3"}

    brick_world = run_brick_world_leg(aero, lib, case, max(5, min(args.steps, 40)), args.warmup) if args.brick_world else None
    batch = None
    if args.batch_ticks > 0:
        batch = run_batch_leg(aero, lib, torch, stream, args.batch_ticks, args.warmup)
    meso = None
    if args.meso_steps > 0:
        meso = run_meso_leg(aero, lib, torch, stream, args.meso_steps, args.warmup)
    adjoint = run_adjoint_leg(aero, lib, torch) if args.adjoint else None

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None

    peak, peak_kind = measured_peaks()
    if batch is not None:
        batch["frac_of_peak"] = batch["achieved_gbs"] / peak
    if meso is not None:
        for k in ("fp32", "fp32_packed", "fp16", "i16"):
            meso[f"{k}_frac_of_peak"] = meso[f"{k}_achieved_gbs"] / peak
    h = results[HEADLINE]
    achieved = h["achieved_gbs"]
    out = {
        "metric": METRIC,
        "value": h["mlups"],
        "unit": "MLUPS",
        "n_gpus": world,
        "steps": h["steps"],
        "warmup": args.warmup,
        "ms_per_step": h["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "i16-store/f32-compute",
        "data": "synthetic (seeded 4-octave terrain, temperature lapse + warm bubble)",
        "config": {"workload": f"d3q27-cumulant {n}^3 terrain brick, inflow x-, convective outflow x+, SGS C=0.1, "
                               "Boussinesq g*beta=1e-4 with the temperature transport, 16-bit fixed-point in-place",
                   "bricks_per_gpu": 1, "cells_per_gpu": cells, "storage": VARIANTS[HEADLINE][4],
                   "l2": "inputs larger than L2 (16-bit state 119 MB + fields; fp32 state 238 MB); no flush",
                   "parallelism": f"bricks x{world}",
                   "fused_transport": bool(args.fused_transport),
                   "timing": f"windows of {h['steps']} steps repeated to >= 1 s (median of {h['windows']}: "
                             f"{h['window_ms_min']:.2f}..{h['window_ms_max']:.2f} ms)",
                   **{f"{v}_mlups": results[v]["mlups"] for v in results if v != HEADLINE},
                   **{f"{HEADLINE}_over_{v}": h["mlups"] / results[v]["mlups"] for v in results if v != HEADLINE},
                   **{f"{v}_frac_of_peak": results[v]["achieved_gbs"] / peak for v in results},
                   **{f"{v}_kernel_us": results[v]["kernel_ms"] * 1e3 for v in results},
                   **{f"{v}_step_gbs": results[v]["step_gbs"] for v in results},
                   "temperature_transport": "the reference's benchmark-mode scalar update before every collision, "
                                            + ("computed inside the step kernel" if args.fused_transport else
                                               "computed by a separate kernel before the step kernel")
                                            + "; the case's field loaded as the starting state",
                   "e2e_resident": {"value": e2e_resident, "unit": "MLUPS", "h2d_bytes_per_step": 0,
                                    "d2h_bytes_per_step": int(atlas.nbytes), "steps": e2e_steps,
                                    "api": "aero_lbm_step_rect_cached + aero_lbm_extract_flow_atlas_rect(stride 4)"},
                   "brick_world": brick_world,
                   "accuracy": acc,
                   "batch": batch,
                   "meso_d3q19": meso,
                   "adjoint": adjoint},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic_record(f"step_ip2_i16@{n}"), "peak_source": peak_kind,
                     "bytes_per_cell": VARIANTS[HEADLINE][3] + THERMAL_BYTES[bool(args.fused_transport)],
                     "kernel": "step_ip2_kernel<StoreI16Dev>" + (" (temperature transport fused)" if args.fused_transport
                                                                  else " (temperature transport as a separate kernel)"),
                     "kernel_us": h["kernel_ms"] * 1e3,
                     "timing": "CUDA events around each step-kernel launch on the library's stream, timed windows"},
        "e2e": {"value": e2e_value, "unit": "MLUPS", "h2d_bytes_per_step": int(packet.numel() * 4),
                "d2h_bytes_per_step": int(atlas.nbytes), "steps": e2e_steps,
                "api": "aero_lbm_step_rect (pinned packet) + aero_lbm_extract_flow_atlas_rect(stride 4)"},
        "gpu_launches": int(h["launches"]),
        "clocks": h["clocks"],
    }
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_single(n)
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--streaming", type=int, default=0, help="0 auto, 1 two-buffer, 2 in-place")
    ap.add_argument("--fused-transport", type=int, choices=[0, 1], default=0,
                    help="temperature transport as a separate pass (0, default) or inside the step kernel (1)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-ticks", type=int, default=500, help="ticks of the 512-brick batch leg (0 skips it)")
    ap.add_argument("--variants", default="fp16,fp32_exact,fp32_fast",
                    help="variants measured beside the 16-bit fixed-point headline (comma list, may be empty)")
    ap.add_argument("--meso-steps", type=int, default=2000, help="steps of the D3Q19 mesoscale leg (0 skips it)")
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false", help="skip the adjoint (gradient) leg")
    ap.add_argument("--accuracy-steps", type=int, default=1000,
                    help="steps of the 16-bit-vs-FP64 accuracy leg (0 skips it)")
    ap.add_argument("--no-brick-world", dest="brick_world", action="store_false",
                    help="skip the brick-world service leg")
    ap.add_argument("--brick-world-only", action="store_true",
                    help="run only the brick-world service leg and print its record (for profiling)")
    args = ap.parse_args()
    args.variants = [v for v in args.variants.split(",") if v]
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        print(json.dumps(run_reference_arm(args.steps, args.warmup, args.n)))
        return 0
    res = run_ours(args)
    if res is not None:
        print(json.dumps(res))
    return 0


if __name__ == "__main__":
    sys.exit(main())
