"""The bench's multi-rank plumbing on the CPU: two `gloo` ranks (world size 2,
rendezvous on 127.0.0.1) agree on the maximum of their window times and on
one window count, as `bench.py --gpus N` needs when each rank times its own
bricks (weak scaling, no collective on the data path)."""
from __future__ import annotations

import importlib.util
import socket
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime
    import os

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench = _load_bench()
        own_ms = [100.0, 300.0][rank]  # a first window of 100 / 300 ms
        got_max = bench.rank_max(own_ms + 0.25, world, dist, "cpu")
        got_windows = bench.window_count(own_ms, world, dist, "cpu")
        out.put((rank, got_max, got_windows))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_and_window_count():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    res = sorted(out.get(timeout=10) for _ in range(2))
    # max over ranks of 100.25 / 300.25 ms; windows: ceil(1000 / 100) = 10 on rank 0, 4 on rank 1 -> 10 on both
    assert [r[1] for r in res] == [300.25, 300.25]
    assert [r[2] for r in res] == [10, 10]


def test_single_rank_passes_values_through():
    bench = _load_bench()
    assert bench.rank_max(1.5, 1) == 1.5
    assert bench.window_count(100.0, 1) == 10
    assert bench.window_count(5000.0, 1) == 3
    assert bench.window_count(0.0, 1) == 5000
