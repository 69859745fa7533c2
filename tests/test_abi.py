"""The C-ABI library: built, loadable, exports what include/*.h declares, and
fails loudly (no CPU fallback) when no GPU is present."""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import pytest

import aero_b200
from conftest import cuda_available

ROOT = Path(__file__).resolve().parents[1]


def test_library_exists_and_loads(lib):
    assert aero_b200.LIB_PATH.exists()
    assert isinstance(lib, ctypes.CDLL)


def test_exports_every_declared_symbol():
    declared = set()
    for h in (ROOT / "include").glob("*.h"):
        declared |= set(aero_b200.declared_symbols(h))
    assert len(declared) > 40
    out = subprocess.run(["nm", "-D", "--defined-only", str(aero_b200.LIB_PATH)], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = sorted(declared - exported)
    assert not missing, f"declared but not exported: {missing}"


def test_bindings_cover_declarations():
    declared = set(aero_b200.declared_symbols())
    assert declared <= set(aero_b200.SIGNATURES), sorted(declared - set(aero_b200.SIGNATURES))


@pytest.mark.skipif(cuda_available(), reason="checks the no-GPU error path")
def test_init_without_gpu_fails_loudly(lib):
    assert lib.aero_lbm_init_rect(8, 8, 8, 11, 4) == 0
    assert "CUDA" in aero_b200.last_error(lib)


def test_config_roundtrip_without_gpu(lib):
    cfg = aero_b200.default_config(lib)
    assert cfg.struct_size == ctypes.sizeof(aero_b200.AeroLbmBenchmarkConfig)
    cfg.enabled = 1
    cfg.x_min.hydrodynamic_kind = 99  # invalid -> sanitised to INHERIT_GAME
    cfg.reynolds_number = float("nan")
    assert lib.aero_lbm_benchmark_set_config(ctypes.byref(cfg)) == 1
    back = aero_b200.AeroLbmBenchmarkConfig()
    assert lib.aero_lbm_benchmark_get_config(ctypes.byref(back)) == 1
    assert back.x_min.hydrodynamic_kind == 0
    assert back.reynolds_number == 100.0
    lib.aero_lbm_benchmark_reset_config()


def test_wind_tunnel_argument_errors(lib):
    h = ctypes.c_longlong(0)
    assert lib.aero_solver_create(0, 4, 4, 1.0, 0.05, ctypes.byref(h)) == 0
    assert b"invalid grid" in lib.aero_solver_last_error()
    assert lib.aero_solver_step_wind_tunnel(12345, None, 1, None, 0) == 0
    assert b"invalid solver handle" in lib.aero_solver_last_error()
