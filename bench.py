"""Benchmark of the B200 D3Q27 brick step (MLUPS and fraction of the HBM roofline).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one GPU): the 128^3 terrain brick with Boussinesq buoyancy (seeded
4-octave heightmap, inflow (0.08, 0.02, 0), Smagorinsky C = 0.1, g*beta = 1e-4
along +z), stepped by the library's fused pull-stream + cumulant-collide kernel.
Inputs are seeded synthetic data of the benchmark's shape (no dataset exists).

value : device-resident MLUPS (state in HBM, one fused launch per step, CUDA
        events on the launching stream; the 2 x 226 MB state is larger than L2).
e2e   : the same metric through the reference-facing C ABI with host buffers:
        every step uploads the 11-channel packet from pinned memory
        (aero_lbm_step_rect) and reads back the stride-4 velocity atlas
        (aero_lbm_extract_flow_atlas_rect).
--impl reference: the reference's own CPU step (oracle/_ref, built from the
        reference sources) on the box's host cores, one single-threaded process
        per core, each on a 64^3 window of the same workload.

With torchrun (N > 1) every rank steps its own brick (bricks are independent
work units; no data-path collective), timing is the max over ranks and value
is the aggregate.
"""
from __future__ import annotations

import argparse
import ctypes
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
                                          "--format=csv,noheader,nounits", "-lms", "100"],
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
def _ref_worker(args):
    """One process: the reference CPU step on a 64^3 window of the workload."""
    steps, warmup, q = args
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    cases = load_cases()
    case = cases.c2_terrain_boussinesq(128)
    w = 64
    obst = np.ascontiguousarray(case.obstacle[:w, :w, :w])
    u = [np.ascontiguousarray(a[:w, :w, :w]) for a in case.u]
    temp = np.ascontiguousarray(case.temperature[:w, :w, :w])
    cfg = case.config_dict()
    cfg["faces"] = case.faces
    ref = O.RefLib()
    lib = ref.lib
    lib.aero_lbm_init_rect(w, w, w, 11, 4)
    c = O.config_struct(O.RefBenchmarkConfig, cfg, lib.aero_lbm_benchmark_default_config)
    lib.aero_lbm_benchmark_set_config(ctypes.byref(c))
    pk = O.packet_from(obst, *u, temperature=temp)
    for _ in range(warmup):
        lib.aero_lbm_step_rect(pk.ctypes.data, w, w, w, 1, None)
    q.put("ready")
    t0 = time.perf_counter()
    for _ in range(steps):
        lib.aero_lbm_step_rect(pk.ctypes.data, w, w, w, 1, None)
    dt = time.perf_counter() - t0
    return w ** 3 * steps / dt / 1e6


def run_reference_arm(steps: int, warmup: int, procs: int | None = None) -> dict:
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    if not O.REF_LIB.exists():
        return {"impl": "reference", "unavailable": "oracle/_ref/libaero_lbm_ref.so was not built (reference sources absent)"}
    cores = procs or max(1, min(os.cpu_count() or 1, 16))
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        q = m.Queue()
        with ctx.Pool(cores) as pool:
            t0 = time.perf_counter()
            per = pool.map(_ref_worker, [(steps, warmup, q)] * cores)
            wall = time.perf_counter() - t0
    value = float(sum(per))
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "MLUPS",
        "n_gpus": 0,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": 64 ** 3 / (value / cores * 1e6) * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded terrain, heightmap, temperature field)",
        "config": {"workload": "d3q27-terrain-boussinesq 64^3 window of the 128^3 brick, reference CPU step",
                   "processes": cores},
        "cpu_baseline": {"value": value, "unit": "MLUPS", "cores": cores, "kind": "reference",
                         "sample": f"{cores} processes x {steps} steps of a 64^3 window ({wall:.1f}s wall)"},
        "e2e": {"value": value, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def cpu_baseline_single(seconds: float = 15.0) -> dict | None:
    """Reference CPU step, one core, bounded sample of the same workload."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    if not O.REF_LIB.exists():
        return None
    ctx = mp.get_context("spawn")
    est_steps = max(2, int(seconds / 1.0))
    with ctx.Manager() as m:
        q = m.Queue()
        with ctx.Pool(1) as pool:
            v = pool.map(_ref_worker, [(est_steps, 1, q)])[0]
    return {"value": v, "unit": "MLUPS", "cores": 1, "kind": "reference",
            "sample": f"{est_steps} steps of a 64^3 window of the workload, single-threaded reference CPU step"}


# ---------------------------------------------------------------- our arm
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

    case = cases.c2_terrain_boussinesq(args.n)
    n = args.n
    cells = case.cells
    lib.aero_lbm_b200_set_physics_overrides(case.smagorinsky_c, case.buoyancy_beta, case.gravity_axis)
    lib.aero_lbm_b200_set_streaming_mode(args.streaming)
    ctx = aero.LbmContext(case.dims, key=1 + rank, lib=lib)
    sys.path.insert(0, str(ROOT / "oracle"))
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

    packet = torch.from_numpy(case.packet()).pin_memory()
    pk_ptr = ctypes.cast(packet.data_ptr(), ctypes.POINTER(ctypes.c_float))
    if not lib.aero_lbm_step_rect(pk_ptr, n, n, n, ctx.key, None):
        raise RuntimeError(aero.last_error(lib))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        ctx.advance(1)
    barrier()
    launches0 = lib.aero_lbm_b200_launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(stream)
        for _ in range(args.steps):
            ctx.advance(1)
        end.record(stream)
        barrier()
    launches = lib.aero_lbm_b200_launch_count() - launches0
    ms = start.elapsed_time(end)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    value = cells * world * args.steps / (ms * 1e-3) / 1e6

    # e2e through the C ABI with host buffers
    stride = 4
    atlas = np.zeros(((n + stride - 1) // stride) ** 3 * 4, np.float32)
    e2e_steps = max(3, min(args.steps, 50))
    for _ in range(2):
        lib.aero_lbm_step_rect(pk_ptr, n, n, n, ctx.key, None)
        lib.aero_lbm_extract_flow_atlas_rect(n, n, n, ctx.key, stride, aero.fptr(atlas), atlas.size)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        if not lib.aero_lbm_step_rect(pk_ptr, n, n, n, ctx.key, None):
            raise RuntimeError(aero.last_error(lib))
        if not lib.aero_lbm_extract_flow_atlas_rect(n, n, n, ctx.key, stride, aero.fptr(atlas), atlas.size):
            raise RuntimeError(aero.last_error(lib))
    barrier()
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = cells * world * e2e_steps / e2e_s / 1e6

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None

    peak, peak_kind = measured_peaks()
    achieved = BYTES_PER_CELL_FP32 * cells / (ms_per_step * 1e-3) / 1e9
    traffic = traffic_record("step_ab_kernel@128")
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "MLUPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded 4-octave terrain, temperature lapse + warm bubble)",
        "config": {"workload": f"d3q27-cumulant-fp32 {n}^3 terrain brick, SGS C=0.1, Boussinesq g*beta=1e-4",
                   "bricks_per_gpu": 1, "cells_per_gpu": cells, "storage": "fp32 populations, two-buffer pull",
                   "l2": "state (2 x 226 MB) larger than L2; no flush needed", "parallelism": f"bricks x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind,
                     "bytes_per_cell": BYTES_PER_CELL_FP32},
        "e2e": {"value": e2e_value, "unit": "MLUPS", "h2d_bytes_per_step": int(packet.numel() * 4),
                "d2h_bytes_per_step": int(atlas.nbytes), "steps": e2e_steps,
                "api": "aero_lbm_step_rect (pinned packet) + aero_lbm_extract_flow_atlas_rect(stride 4)"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_single()
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--streaming", type=int, default=0, help="0 auto, 1 two-buffer, 2 in-place")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        ref_steps = max(1, min(args.steps, 10))
        print(json.dumps(run_reference_arm(ref_steps, min(args.warmup, 1))))
        return 0
    res = run_ours(args)
    if res is not None:
        print(json.dumps(res))
    return 0


if __name__ == "__main__":
    sys.exit(main())
