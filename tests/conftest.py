"""Shared test set-up.

The product package lives in a directory whose name is not an identifier
(aerodynamics4mc-fabric_b200/), so it is loaded here under the module name
``aero_b200``. The oracle (test infrastructure) is imported from oracle/.
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "aerodynamics4mc-fabric_b200"
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests"))


def _load_pkg():
    if "aero_b200" in sys.modules:
        return sys.modules["aero_b200"]
    spec = importlib.util.spec_from_file_location("aero_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["aero_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_pkg()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def cuda_available() -> bool:
    try:
        import ctypes
        lib = ctypes.CDLL("libcuda.so.1")
        n = ctypes.c_int(0)
        if lib.cuInit(0) != 0:
            return False
        return lib.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0
    except OSError:
        return False


@pytest.fixture(scope="session")
def lib():
    """The product library (fails loudly if it was not built)."""
    import aero_b200
    return aero_b200.load_library()


@pytest.fixture(autouse=True)
def _default_tuning():
    """Every test starts from the library's default tuning knobs, solver mode
    and benchmark configuration (they are process-global; a test that changes
    one must not leak it into the next)."""
    import aero_b200
    lib = aero_b200._lib
    if lib is not None:
        lib.aero_lbm_b200_reset_tuning()
        lib.aero_lbm_set_realtime_solver_mode(0)
        lib.aero_lbm_benchmark_reset_config()
    yield


@pytest.fixture(scope="session")
def gpu(lib):
    if not cuda_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return lib
