"""Python binding of libaero_lbm_b200.so (the B200 lattice-Boltzmann brick step).

This is a thin ctypes mirror of the library's C ABI (include/aero_lbm_b200.h),
which itself mirrors the reference mod's native ABI (aero_lbm_*, aero_solver_*).
It is how the reference's own Python tools drive the native step, so the same
calls work against this library. No PyTorch is involved; buffers are numpy
arrays or raw pointers.

The library runs only on a CUDA device (sm_100a). Loading fails loudly if the
shared library has not been built; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

PACKAGE_DIR = Path(__file__).resolve().parent
LIB_PATH = PACKAGE_DIR / "libaero_lbm_b200.so"
HEADER_PATH = PACKAGE_DIR.parent / "include" / "aero_lbm_b200.h"

# ---------------------------------------------------------------- enums
BENCHMARK_PRESET_NONE = 0
HYDRO_INHERIT_GAME = 0
HYDRO_PERIODIC = 1
HYDRO_BOUNCE_BACK = 2
HYDRO_MOVING_WALL = 3
HYDRO_VELOCITY = 4
HYDRO_PRESSURE = 5
HYDRO_CONVECTIVE = 6
HYDRO_SYMMETRY = 7

FLAG_DISABLE_FAN_FORCING = 1 << 0
FLAG_DISABLE_FAN_NOISE = 1 << 1
FLAG_DISABLE_SPONGE = 1 << 2
FLAG_DISABLE_CONVECTIVE_OUTFLOW = 1 << 3
FLAG_DISABLE_OBSTACLE_BOUNCE_BLEND = 1 << 4
FLAG_DISABLE_SGS = 1 << 5
FLAG_DISABLE_INTERNAL_THERMAL_SOURCE = 1 << 6
FLAG_DISABLE_BUOYANCY = 1 << 7

SOLVER_BOUNDARY_WIND_TUNNEL = 1
SOLVER_BOUNDARY_WIND_TUNNEL_PRESSURE_OUTLET = 2
SOLVER_BOUNDARY_CLOSED = 3
SOLVER_BOUNDARY_PERIODIC = 4
SOLVER_FLOW_CHANNELS = 4

PACKET_CHANNELS = 11


# ---------------------------------------------------------------- structs
class AeroLbmBoundaryFaceConfig(ctypes.Structure):
    _fields_ = [
        ("hydrodynamic_kind", ctypes.c_int),
        ("thermal_kind", ctypes.c_int),
        ("velocity", ctypes.c_float * 3),
        ("pressure", ctypes.c_float),
        ("temperature", ctypes.c_float),
        ("heat_flux", ctypes.c_float),
    ]


class AeroLbmBenchmarkConfig(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_uint32),
        ("struct_size", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
        ("enabled", ctypes.c_int),
        ("preset", ctypes.c_int),
        ("reserved0", ctypes.c_int),
        ("reynolds_number", ctypes.c_float),
        ("rayleigh_number", ctypes.c_float),
        ("prandtl_number", ctypes.c_float),
        ("mach_number", ctypes.c_float),
        ("reference_density", ctypes.c_float),
        ("reference_temperature", ctypes.c_float),
        ("reference_length", ctypes.c_float),
        ("body_force", ctypes.c_float * 3),
        ("gravity", ctypes.c_float * 3),
        ("initial_velocity", ctypes.c_float * 3),
        ("initial_pressure", ctypes.c_float),
        ("initial_temperature", ctypes.c_float),
        ("x_min", AeroLbmBoundaryFaceConfig),
        ("x_max", AeroLbmBoundaryFaceConfig),
        ("y_min", AeroLbmBoundaryFaceConfig),
        ("y_max", AeroLbmBoundaryFaceConfig),
        ("z_min", AeroLbmBoundaryFaceConfig),
        ("z_max", AeroLbmBoundaryFaceConfig),
        ("reserved", ctypes.c_uint32 * 8),
    ]

    FACE_NAMES = ("x_min", "x_max", "y_min", "y_max", "z_min", "z_max")

    def faces(self):
        return [getattr(self, n) for n in self.FACE_NAMES]


class AeroLbmTimingSnapshot(ctypes.Structure):
    _fields_ = [
        ("ticks", ctypes.c_uint64),
        ("last_payload_copy_ms", ctypes.c_double),
        ("last_solver_ms", ctypes.c_double),
        ("last_readback_ms", ctypes.c_double),
        ("last_total_ms", ctypes.c_double),
        ("avg_payload_copy_ms", ctypes.c_double),
        ("avg_solver_ms", ctypes.c_double),
        ("avg_readback_ms", ctypes.c_double),
        ("avg_total_ms", ctypes.c_double),
    ]


class AeroGridDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("dx", ctypes.c_float), ("dt", ctypes.c_float)]


class AeroBoundaryDesc(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int),
        ("inlet_vx", ctypes.c_float),
        ("inlet_vy", ctypes.c_float),
        ("inlet_vz", ctypes.c_float),
        ("outlet_pressure", ctypes.c_float),
        ("density", ctypes.c_float),
        ("viscosity", ctypes.c_float),
    ]


class AeroStepInput(ctypes.Structure):
    _fields_ = [
        ("solid_mask", ctypes.POINTER(ctypes.c_uint8)),
        ("prev_flow", ctypes.POINTER(ctypes.c_float)),
        ("grid", AeroGridDesc),
        ("boundary", AeroBoundaryDesc),
        ("steps", ctypes.c_int),
    ]


class AeroStepOutput(ctypes.Structure):
    _fields_ = [("flow_out", ctypes.POINTER(ctypes.c_float)), ("max_velocity", ctypes.c_float), ("status", ctypes.c_int)]

class AeroLbmMesoscaleConfig(ctypes.Structure):
    """native/include/aero_lbm_capi.h:124-141"""
    _fields_ = [
        ("abi_version", ctypes.c_uint32), ("struct_size", ctypes.c_uint32),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx_m", ctypes.c_float), ("dt_s", ctypes.c_float), ("molecular_nu_m2_s", ctypes.c_float),
        ("prandtl_air", ctypes.c_float), ("turbulent_prandtl", ctypes.c_float),
        ("reference_density_kg_m3", ctypes.c_float), ("ambient_air_temperature_k", ctypes.c_float),
        ("deep_ground_temperature_k", ctypes.c_float), ("background_wind_m_s", ctypes.c_float * 3),
        ("reserved", ctypes.c_uint32 * 8),
    ]


class AeroLbmMesoscaleTransport(ctypes.Structure):
    """native/include/aero_lbm_capi.h:143-149"""
    _fields_ = [(n, ctypes.c_float) for n in ("velocity_scale_m_s_per_lattice", "nu_molecular_lattice",
                                               "alpha_molecular_lattice", "tau_shear_molecular",
                                               "tau_thermal_molecular")]


class AeroLbmB200MesoscaleOptions(ctypes.Structure):
    _fields_ = [
        ("periodic_sides", ctypes.c_int), ("free_slip_top", ctypes.c_int), ("fixed_tau", ctypes.c_int),
        ("enable_sgs", ctypes.c_int), ("disable_edge_blend", ctypes.c_int), ("hydro_only", ctypes.c_int),
        ("tau_hydro", ctypes.c_double), ("smagorinsky_c", ctypes.c_double), ("body_force", ctypes.c_double * 3),
        ("storage", ctypes.c_int), ("threads", ctypes.c_int), ("collision", ctypes.c_int), ("reserved", ctypes.c_int),
    ]


class AeroLbmB200AdjointConfig(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("face_kind", ctypes.c_int * 6),
        ("tau", ctypes.c_float), ("smagorinsky_c", ctypes.c_float), ("buoyancy_beta", ctypes.c_float),
        ("steps", ctypes.c_int), ("checkpoint_every", ctypes.c_int), ("reserved", ctypes.c_int),
    ]


# ---------------------------------------------------------------- loading
_P = ctypes.c_void_p
_F32P = ctypes.POINTER(ctypes.c_float)
_I16P = ctypes.POINTER(ctypes.c_int16)
_U8P = ctypes.POINTER(ctypes.c_uint8)
_I32P = ctypes.POINTER(ctypes.c_int)
_U16P = ctypes.POINTER(ctypes.c_uint16)
_LL = ctypes.c_longlong
_I = ctypes.c_int
_F = ctypes.c_float

SIGNATURES = {
    # per-context ABI
    "aero_lbm_init": (_I, [_I, _I, _I]),
    "aero_lbm_step": (_I, [_F32P, _I, _LL, _F32P]),
    "aero_lbm_init_rect": (_I, [_I, _I, _I, _I, _I]),
    "aero_lbm_step_rect": (_I, [_F32P, _I, _I, _I, _LL, _F32P]),
    "aero_lbm_step_rect_scaled": (_I, [_F32P, _I, _I, _I, _LL, _F, _F32P]),
    "aero_lbm_step_rect_cached": (_I, [_I, _I, _I, _LL, _F32P]),
    "aero_lbm_step_rect_cached_scaled": (_I, [_I, _I, _I, _LL, _F, _F32P]),
    "aero_lbm_has_context": (_I, [_LL]),
    "aero_lbm_context_realtime_cached_initialized": (_I, [_LL]),
    "aero_lbm_exchange_halo": (_I, [_I, _LL, _LL, _I, _I, _I]),
    "aero_lbm_exchange_halo_layers_rect": (_I, [_I, _I, _I, _I, _LL, _LL, _I, _I, _I]),
    "aero_lbm_patch_d3q27_f16_static_cells_rect": (_I, [_I, _I, _I, _LL, _I, ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.c_void_p]),
    "aero_lbm_set_d3q27_f16_boundary_shell_rect": (_I, [_I, _I, _I, _LL, _F32P, _I, _I, _I, _F]),
    "aero_lbm_clear_d3q27_f16_boundary_shell_rect": (_I, [_LL]),
    "aero_lbm_step_rect_with_sparse_overlays": (_I, [_F32P, _I, _I, _I, _LL, ctypes.c_void_p, _F32P, _I, _F32P]),
    "aero_lbm_shift_context": (_I, [_I, _LL, _I, _I, _I]),
    "aero_lbm_context_compact_initialized": (_I, [_LL]),
    "aero_lbm_sample_temperature_point_rect": (_I, [_I, _I, _I, _LL, _I, _I, _I, _F32P]),
    "aero_lbm_sample_flow_point_rect": (_I, [_I, _I, _I, _LL, _I, _I, _I, _F32P]),
    "aero_lbm_copy_flow_temperature_subrect": (_I, [_I, _I, _I, _LL, _I, _I, _I, _I, _I, _I, _F32P, _F32P]),
    "aero_lbm_get_last_force": (_I, [_LL, _F32P, _F32P, _F32P]),
    "aero_lbm_memory_info": (ctypes.c_char_p, []),
    "aero_lbm_get_temperature_state_rect": (_I, [_I, _I, _I, _LL, _F32P]),
    "aero_lbm_extract_flow_atlas_rect": (_I, [_I, _I, _I, _LL, _I, _F32P, _I]),
    "aero_lbm_get_flow_state_rect": (_I, [_I, _I, _I, _LL, _F32P]),
    "aero_lbm_set_temperature_state_rect": (_I, [_I, _I, _I, _LL, _F32P]),
    "aero_lbm_release_context": (None, [_LL]),
    "aero_lbm_shutdown": (None, []),
    "aero_lbm_runtime_info": (ctypes.c_char_p, []),
    "aero_lbm_last_error": (ctypes.c_char_p, []),
    "aero_lbm_timing_info": (ctypes.c_char_p, []),
    "aero_lbm_reset_timing": (None, []),
    "aero_lbm_set_realtime_solver_mode": (None, [_I]),
    "aero_lbm_finish": (_I, []),
    "aero_lbm_get_timing_snapshot": (_I, [ctypes.POINTER(AeroLbmTimingSnapshot)]),
    "aero_lbm_benchmark_default_config": (None, [ctypes.POINTER(AeroLbmBenchmarkConfig)]),
    "aero_lbm_benchmark_default_preset_config": (_I, [_I, ctypes.POINTER(AeroLbmBenchmarkConfig)]),
    "aero_lbm_benchmark_set_config": (_I, [ctypes.POINTER(AeroLbmBenchmarkConfig)]),
    "aero_lbm_benchmark_get_config": (_I, [ctypes.POINTER(AeroLbmBenchmarkConfig)]),
    "aero_lbm_benchmark_reset_config": (None, []),
    "aero_lbm_benchmark_info": (ctypes.c_char_p, []),
    # device-resident extensions
    "aero_lbm_b200_set_stream": (None, [_P]),
    "aero_lbm_b200_launch_count": (ctypes.c_ulonglong, []),
    "aero_lbm_b200_advance_rect": (_I, [_LL, _I]),
    "aero_lbm_b200_set_streaming_mode": (_I, [_I]),
    "aero_lbm_b200_set_collision_mode": (_I, [_I]),
    "aero_lbm_b200_set_cells_per_thread": (_I, [_I]),
    "aero_lbm_b200_set_streamed_step": (_I, [_I]),
    "aero_lbm_b200_set_thermal_transport": (_I, [_I]),
    "aero_lbm_b200_kernel_timer": (_I, [_I]),
    "aero_lbm_b200_kernel_time": (_I, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]),
    "aero_lbm_b200_set_fp16_format": (_I, [_I]),
    "aero_lbm_b200_set_fused_transport": (_I, [_I]),
    "aero_lbm_b200_reset_tuning": (None, []),
    "aero_lbm_b200_conservation_sums": (_I, [_LL, ctypes.POINTER(ctypes.c_double)]),
    "aero_lbm_b200_conservation_sums_noalloc": (_I, [_LL, ctypes.POINTER(ctypes.c_double)]),
    "aero_lbm_b200_set_force_field": (_I, [_LL, _F32P, _I]),
    "aero_lbm_b200_set_physics_overrides": (None, [_F, _F, _I]),
    # batched bricks
    "aero_lbm_b200_batch_create": (_I, [ctypes.POINTER(_LL)]),
    "aero_lbm_b200_batch_add_brick": (_I, [_LL, _I, _I, _I, _I, _U8P, _F32P, _F, _F32P, _I32P, _I32P]),
    "aero_lbm_b200_batch_finalize": (_I, [_LL, _I, _F]),
    "aero_lbm_b200_batch_set_options": (_I, [_LL, _I, _I]),
    "aero_lbm_b200_batch_tick": (_I, [_LL, _I]),
    "aero_lbm_b200_batch_autotune": (_I, [_LL, _I, _I32P, _I32P, _F32P]),
    "aero_lbm_b200_batch_info": (_I, [_LL, ctypes.POINTER(_LL), ctypes.POINTER(ctypes.c_double), _I32P, _I32P,
                                     ctypes.POINTER(_LL)]),
    "aero_lbm_b200_batch_copy_atlas": (_I, [_LL, _I, _I16P, _I]),
    "aero_lbm_b200_batch_copy_flow": (_I, [_LL, _I, _F32P, _I]),
    "aero_lbm_b200_batch_destroy": (None, [_LL]),
    "aero_lbm_b200_batch_last_error": (ctypes.c_char_p, []),
    # D3Q19 mesoscale ABI
    "aero_lbm_mesoscale_default_config": (None, [ctypes.POINTER(AeroLbmMesoscaleConfig)]),
    "aero_lbm_mesoscale_derive_transport": (_I, [ctypes.POINTER(AeroLbmMesoscaleConfig),
                                                 ctypes.POINTER(AeroLbmMesoscaleTransport)]),
    "aero_lbm_mesoscale_create_context": (_I, [ctypes.POINTER(AeroLbmMesoscaleConfig), ctypes.POINTER(_LL)]),
    "aero_lbm_mesoscale_step_context": (_I, [_LL, ctypes.POINTER(AeroLbmMesoscaleConfig), _F32P, _F32P]),
    "aero_lbm_mesoscale_release_context": (None, [_LL]),
    "aero_lbm_b200_mesoscale_default_options": (None, [ctypes.POINTER(AeroLbmB200MesoscaleOptions)]),
    "aero_lbm_b200_mesoscale_set_options": (_I, [_LL, ctypes.POINTER(AeroLbmB200MesoscaleOptions)]),
    "aero_lbm_b200_mesoscale_advance": (_I, [_LL, _I]),
    "aero_lbm_b200_mesoscale_read_state": (_I, [_LL, _F32P]),
    "aero_lbm_b200_mesoscale_info": (_I, [_LL, ctypes.POINTER(_LL), ctypes.POINTER(ctypes.c_double)]),
    # discrete adjoint
    "aero_lbm_b200_adjoint_default_config": (None, [ctypes.POINTER(AeroLbmB200AdjointConfig)]),
    "aero_lbm_b200_adjoint_create": (_I, [ctypes.POINTER(AeroLbmB200AdjointConfig), _U8P, _F32P, ctypes.POINTER(_LL)]),
    "aero_lbm_b200_adjoint_set_probes": (_I, [_LL, _I, _I32P, _F32P]),
    "aero_lbm_b200_adjoint_forward": (_I, [_LL, _F32P, _F32P, _I, ctypes.POINTER(ctypes.c_double), _F32P]),
    "aero_lbm_b200_adjoint_gradient": (_I, [_LL, _F32P, _F32P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "aero_lbm_b200_adjoint_timing": (_I, [_LL, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "aero_lbm_b200_adjoint_destroy": (None, [_LL]),
    "aero_lbm_b200_adjoint_last_error": (ctypes.c_char_p, []),
    "aero_lbm_b200_adjoint_collide_vjp_host": (_I, [_I, ctypes.POINTER(AeroLbmB200AdjointConfig), ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                                                    ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    # brick-world service ABI
    "aero_lbm_simulation_create_service": (_I, [ctypes.POINTER(_LL)]),
    "aero_lbm_simulation_release_service": (None, [_LL]),
    "aero_lbm_simulation_set_focus": (_I, [_LL, _I, _I, _I, _I]),
    "aero_lbm_simulation_submit_world_deltas": (_I, [_LL, ctypes.c_void_p, _I]),
    "aero_lbm_simulation_ensure_brick_world_runtime": (_I, [_LL, _LL, _I, _F, _F]),
    "aero_lbm_simulation_set_brick_world_solver_mode": (_I, [_LL, _LL, _I]),
    "aero_lbm_simulation_set_brick_world_active_hints": (_I, [_LL, _LL, _I, _I32P, _I]),
    "aero_lbm_simulation_set_brick_world_exact_active_hints": (_I, [_LL, _LL, _I, _I32P, _I]),
    "aero_lbm_simulation_get_brick_world_runtime_status": (_I, [_LL, _LL, _I32P, _I]),
    "aero_lbm_simulation_step_brick_world_runtime": (_I, [_LL, _LL, _I]),
    "aero_lbm_simulation_get_brick_world_resident_brick_count": (_I, [_LL, _LL]),
    "aero_lbm_simulation_copy_brick_world_resident_bricks": (_I, [_LL, _LL, _I32P, _I]),
    "aero_lbm_simulation_get_brick_world_active_brick_count": (_I, [_LL, _LL]),
    "aero_lbm_simulation_copy_brick_world_active_bricks": (_I, [_LL, _LL, _I32P, _I]),
    "aero_lbm_simulation_upload_brick_world_static_brick": (_I, [_LL, _LL, _I, _I, _I, _I, _U8P, _U8P, _U16P, _F32P, _U8P, _U8P]),
    "aero_lbm_simulation_upload_brick_world_static_brick_with_sources": (
        _I, [_LL, _LL, _I, _I, _I, _I, _U8P, _U8P, _U16P, _F32P, _U8P, _F32P, _U8P, _U8P]),
    "aero_lbm_simulation_queue_brick_world_static_brick_upload": (_I, [_LL, _LL, _I, _I, _I, _I, _U8P, _U8P, _U16P, _F32P, _U8P, _U8P]),
    "aero_lbm_simulation_copy_brick_world_dynamic_brick": (_I, [_LL, _LL, _I, _I, _I, _I, _F32P, _F32P, _F32P]),
    "aero_lbm_simulation_copy_brick_world_packed_flow_atlas": (_I, [_LL, _LL, _I, _I, _I, _I, _I, _I16P, _I]),
    "aero_lbm_simulation_upload_brick_world_dynamic_brick": (_I, [_LL, _LL, _I, _I, _I, _I, _F32P, _F32P, _F32P]),
    "aero_lbm_simulation_upload_brick_world_boundary_reference_brick": (_I, [_LL, _LL, _I, _I, _I, _I, _F32P, _F32P, _F32P]),
    "aero_lbm_simulation_runtime_info": (ctypes.c_char_p, []),
    "aero_lbm_simulation_last_error": (ctypes.c_char_p, []),
    # wind-tunnel ABI
    "aero_solver_default_grid": (None, [ctypes.POINTER(AeroGridDesc)]),
    "aero_solver_default_boundary": (None, [ctypes.POINTER(AeroBoundaryDesc)]),
    "aero_solver_create": (_I, [_I, _I, _I, _F, _F, ctypes.POINTER(_LL)]),
    "aero_solver_create_with_grid": (_I, [ctypes.POINTER(AeroGridDesc), ctypes.POINTER(_LL)]),
    "aero_solver_set_solid_mask": (_I, [_LL, _U8P, _I]),
    "aero_solver_set_flow_state": (_I, [_LL, _F32P, _I]),
    "aero_solver_step_wind_tunnel": (_I, [_LL, ctypes.POINTER(AeroBoundaryDesc), _I, _F32P, _I]),
    "aero_solver_advance_wind_tunnel": (_I, [_LL, ctypes.POINTER(AeroBoundaryDesc), _I]),
    "aero_solver_run_wind_tunnel": (_I, [ctypes.POINTER(AeroStepInput), ctypes.POINTER(AeroStepOutput)]),
    "aero_solver_destroy": (None, [_LL]),
    "aero_solver_last_error": (ctypes.c_char_p, []),
    "aero_solver_runtime_info": (ctypes.c_char_p, []),
    "aero_solver_finish": (_I, []),
}

_lib = None


def load_library(path: os.PathLike | str | None = None) -> ctypes.CDLL:
    """Load libaero_lbm_b200.so and attach argument/return types.

    Raises FileNotFoundError when the library has not been built (run
    build.py): the product has no fallback implementation.
    """
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: build it with `python {PACKAGE_DIR / 'build.py'}`")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def last_error(lib: ctypes.CDLL | None = None) -> str:
    lib = lib or load_library()
    msg = lib.aero_lbm_last_error()
    return msg.decode("utf-8", "replace") if msg else ""


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_F32P)


def u8ptr(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(_U8P)


def build_packet(obstacle: np.ndarray, ux=None, uy=None, uz=None, pressure=None, temperature=None,
                 channels: int = PACKET_CHANNELS) -> np.ndarray:
    """AoS step packet in the reference's channel order (obstacle, fan mask,
    fan v, state v, pressure proxy, thermal source, temperature)."""
    cells = obstacle.size
    pk = np.zeros((cells, channels), dtype=np.float32)
    pk[:, 0] = (obstacle.reshape(-1) != 0).astype(np.float32)
    for ch, v in ((5, ux), (6, uy), (7, uz), (8, pressure)):
        if v is not None:
            pk[:, ch] = np.asarray(v, dtype=np.float32).reshape(-1)
    if temperature is not None and channels > 10:
        pk[:, 10] = np.asarray(temperature, dtype=np.float32).reshape(-1)
    return np.ascontiguousarray(pk)


def default_config(lib: ctypes.CDLL | None = None) -> AeroLbmBenchmarkConfig:
    lib = lib or load_library()
    cfg = AeroLbmBenchmarkConfig()
    lib.aero_lbm_benchmark_default_config(ctypes.byref(cfg))
    return cfg


def declared_symbols(header: Path = HEADER_PATH) -> list[str]:
    """Function names declared in include/aero_lbm_b200.h."""
    import re

    text = "\n".join(l for l in header.read_text().splitlines() if not l.lstrip().startswith("#"))
    return sorted(set(re.findall(r"AERO_LBM_B200_EXPORT\s+[^;(]*?\b(\w+)\s*\(", text)))


class AeroLbmWorldDelta(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("type", "x", "y", "z", "data0", "data1", "data2", "data3")] + \
               [(n, ctypes.c_float) for n in ("value0", "value1", "value2", "value3")]


def _ptr(a: np.ndarray, ctype):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class BrickWorldService:
    """The brick-world service (aero_lbm_simulation_*), what the mod's
    NativeSimulationBridge drives: one world of equal cubic bricks keyed by
    brick coordinates, stepped together; dynamic bricks are 4 floats per cell
    (ux, uy, uz, pressure proxy) plus air and surface temperature; the packed
    atlas is 4 int16 per sample."""

    def __init__(self, lib: ctypes.CDLL | None = None):
        self.lib = lib or load_library()
        key = ctypes.c_longlong(0)
        self._ok(self.lib.aero_lbm_simulation_create_service(ctypes.byref(key)))
        self.key = key.value

    def _ok(self, v):
        if not v:
            raise RuntimeError(self.error())
        return v

    def error(self) -> str:
        m = self.lib.aero_lbm_simulation_last_error()
        return m.decode("utf-8", "replace") if m else ""

    def ensure_world(self, world: int, brick_size: int, dx: float = 1.0, dt: float = 0.05, solver_mode: int = 1):
        self._ok(self.lib.aero_lbm_simulation_ensure_brick_world_runtime(self.key, world, brick_size, dx, dt))
        self._ok(self.lib.aero_lbm_simulation_set_brick_world_solver_mode(self.key, world, solver_mode))
        self.n = brick_size

    def set_hints(self, world: int, coords, exact: bool = True):
        c = np.ascontiguousarray(np.asarray(coords, np.int32).reshape(-1))
        fn = self.lib.aero_lbm_simulation_set_brick_world_exact_active_hints if exact \
            else self.lib.aero_lbm_simulation_set_brick_world_active_hints
        self._ok(fn(self.key, world, self.n, _ptr(c, ctypes.c_int), c.size // 3))

    def upload_static(self, world: int, coord, obstacle, surface_kind=None, open_face_mask=None, emitter=None,
                      source_fan=None, source_emitter=None):
        cells = self.n ** 3
        ob = np.ascontiguousarray(np.asarray(obstacle, np.uint8).reshape(-1))
        sk = np.ascontiguousarray(np.zeros(cells, np.uint8) if surface_kind is None else np.asarray(surface_kind, np.uint8).reshape(-1))
        of = np.ascontiguousarray(np.zeros(cells, np.uint16) if open_face_mask is None else np.asarray(open_face_mask, np.uint16).reshape(-1))
        em = np.ascontiguousarray(np.zeros(cells, np.float32) if emitter is None else np.asarray(emitter, np.float32).reshape(-1))
        faces = np.zeros(cells * 6, np.uint8)
        sf = None if source_fan is None else np.ascontiguousarray(np.asarray(source_fan, np.uint8).reshape(-1))
        se = None if source_emitter is None else np.ascontiguousarray(np.asarray(source_emitter, np.float32).reshape(-1))
        self._ok(self.lib.aero_lbm_simulation_upload_brick_world_static_brick_with_sources(
            self.key, world, self.n, *coord, _ptr(ob, ctypes.c_uint8), _ptr(sk, ctypes.c_uint8), _ptr(of, ctypes.c_uint16),
            _ptr(em, ctypes.c_float), None if sf is None else _ptr(sf, ctypes.c_uint8),
            None if se is None else _ptr(se, ctypes.c_float), _ptr(faces, ctypes.c_uint8), _ptr(faces, ctypes.c_uint8)))

    def _dynamic_args(self, flow, air, surface):
        cells = self.n ** 3
        f = np.ascontiguousarray(np.asarray(flow, np.float32).reshape(-1))
        a = np.ascontiguousarray(np.asarray(air, np.float32).reshape(-1))
        s = np.ascontiguousarray(np.zeros(cells, np.float32) if surface is None else np.asarray(surface, np.float32).reshape(-1))
        return f, a, s

    def upload_dynamic(self, world: int, coord, flow, air, surface=None):
        f, a, s = self._dynamic_args(flow, air, surface)
        self._ok(self.lib.aero_lbm_simulation_upload_brick_world_dynamic_brick(self.key, world, self.n, *coord, fptr(f), fptr(a), fptr(s)))

    def upload_reference(self, world: int, coord, flow, air, surface=None):
        f, a, s = self._dynamic_args(flow, air, surface)
        self._ok(self.lib.aero_lbm_simulation_upload_brick_world_boundary_reference_brick(
            self.key, world, self.n, *coord, fptr(f), fptr(a), fptr(s)))

    def submit_deltas(self, deltas):
        arr = (AeroLbmWorldDelta * len(deltas))(*[AeroLbmWorldDelta(*d) for d in deltas])
        self._ok(self.lib.aero_lbm_simulation_submit_world_deltas(self.key, ctypes.cast(arr, ctypes.c_void_p), len(deltas)))

    def step(self, world: int, steps: int = 1):
        self._ok(self.lib.aero_lbm_simulation_step_brick_world_runtime(self.key, world, steps))

    def atlas(self, world: int, coord, stride: int = 4, out: np.ndarray | None = None) -> np.ndarray:
        res = (self.n + stride - 1) // stride
        out = np.zeros(res ** 3 * 4, np.int16) if out is None else out
        self._ok(self.lib.aero_lbm_simulation_copy_brick_world_packed_flow_atlas(
            self.key, world, self.n, *coord, stride, out.ctypes.data_as(_I16P), out.size))
        return out

    def dynamic(self, world: int, coord):
        cells = self.n ** 3
        f = np.zeros(cells * 4, np.float32)
        a = np.zeros(cells, np.float32)
        s = np.zeros(cells, np.float32)
        self._ok(self.lib.aero_lbm_simulation_copy_brick_world_dynamic_brick(self.key, world, self.n, *coord, fptr(f), fptr(a), fptr(s)))
        return f.reshape(-1, 4), a, s

    def status(self, world: int) -> np.ndarray:
        st = np.zeros(8, np.int32)
        self._ok(self.lib.aero_lbm_simulation_get_brick_world_runtime_status(self.key, world, _ptr(st, ctypes.c_int), 8))
        return st

    def runtime_info(self) -> str:
        return self.lib.aero_lbm_simulation_runtime_info().decode()

    def release(self):
        if self.key:
            self.lib.aero_lbm_simulation_release_service(self.key)
            self.key = 0


class LbmContext:
    """One brick/grid context of the per-context ABI (aero_lbm_init_rect +
    aero_lbm_step_rect...), the calls the reference's brick runtime makes."""

    def __init__(self, dims, input_channels: int = PACKET_CHANNELS, output_channels: int = 4, key: int = 1,
                 lib: ctypes.CDLL | None = None, init: bool = True):
        self.lib = lib or load_library()
        self.dims = tuple(int(d) for d in dims)
        self.cells = int(np.prod(self.dims))
        self.key = int(key)
        self.in_ch = input_channels
        self.out_ch = output_channels
        if init and not self.lib.aero_lbm_init_rect(*self.dims, input_channels, output_channels):
            raise RuntimeError(f"aero_lbm_init_rect failed: {last_error(self.lib)}")

    def configure(self, cfg: AeroLbmBenchmarkConfig) -> None:
        if not self.lib.aero_lbm_benchmark_set_config(ctypes.byref(cfg)):
            raise RuntimeError("aero_lbm_benchmark_set_config failed")

    def step(self, packet: np.ndarray | None, output: bool = True, scale: float = 1.0) -> np.ndarray | None:
        out = np.zeros(self.cells * self.out_ch, dtype=np.float32) if output else None
        optr = fptr(out) if output else None
        if packet is None:
            ok = self.lib.aero_lbm_step_rect_cached_scaled(*self.dims, self.key, scale, optr)
        else:
            pk = np.ascontiguousarray(packet, dtype=np.float32)
            if pk.size != self.cells * self.in_ch:
                raise ValueError("packet size does not match dims x input_channels")
            ok = self.lib.aero_lbm_step_rect_scaled(fptr(pk), *self.dims, self.key, scale, optr)
        if not ok:
            raise RuntimeError(f"step failed: {last_error(self.lib)}")
        return out.reshape(self.cells, self.out_ch) if output else None

    def advance(self, steps: int) -> None:
        """Device-resident steps (no host copies, no synchronisation)."""
        if not self.lib.aero_lbm_b200_advance_rect(self.key, int(steps)):
            raise RuntimeError(f"advance failed: {last_error(self.lib)}")

    def atlas(self, stride: int) -> np.ndarray:
        n = [(d + stride - 1) // stride for d in self.dims]
        out = np.zeros(int(np.prod(n)) * 4, dtype=np.float32)
        if not self.lib.aero_lbm_extract_flow_atlas_rect(*self.dims, self.key, stride, fptr(out), out.size):
            raise RuntimeError(f"extract failed: {last_error(self.lib)}")
        return out.reshape(-1, 4)

    def flow_state(self) -> np.ndarray:
        out = np.zeros(self.cells * 4, dtype=np.float32)
        if not self.lib.aero_lbm_get_flow_state_rect(*self.dims, self.key, fptr(out)):
            raise RuntimeError(f"get_flow_state failed: {last_error(self.lib)}")
        return out.reshape(self.cells, 4)

    def temperature_state(self) -> np.ndarray:
        """The context's temperature state (cells floats)."""
        out = np.zeros(self.cells, dtype=np.float32)
        if not self.lib.aero_lbm_get_temperature_state_rect(*self.dims, self.key, fptr(out)):
            raise RuntimeError(f"get_temperature_state failed: {last_error(self.lib)}")
        return out

    def set_temperature_state(self, t) -> None:
        arr = np.ascontiguousarray(np.asarray(t, np.float32).reshape(-1))
        if not self.lib.aero_lbm_set_temperature_state_rect(*self.dims, self.key, fptr(arr)):
            raise RuntimeError(f"set_temperature_state failed: {last_error(self.lib)}")

    def set_force_field(self, fx, fy, fz) -> None:
        soa = np.ascontiguousarray(np.concatenate([np.asarray(a, np.float32).reshape(-1) for a in (fx, fy, fz)]))
        if not self.lib.aero_lbm_b200_set_force_field(self.key, fptr(soa), soa.size):
            raise RuntimeError(f"set_force_field failed: {last_error(self.lib)}")

    def conservation_sums(self) -> np.ndarray:
        """FP64 {sum rho, sum rho u} over fluid cells of the current state."""
        out = np.zeros(4, dtype=np.float64)
        if not self.lib.aero_lbm_b200_conservation_sums(self.key, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))):
            raise RuntimeError(f"conservation_sums failed: {last_error(self.lib)}")
        return out

    def release(self) -> None:
        self.lib.aero_lbm_release_context(self.key)


class BrickBatch:
    """Batched bricks advanced by one persistent launch per tick
    (aero_lbm_b200_batch_*)."""

    def __init__(self, lib: ctypes.CDLL | None = None):
        self.lib = lib or load_library()
        h = ctypes.c_longlong(0)
        if not self.lib.aero_lbm_b200_batch_create(ctypes.byref(h)):
            raise RuntimeError(self.error())
        self.handle = h.value
        self.dims: list[tuple] = []

    def error(self) -> str:
        m = self.lib.aero_lbm_b200_batch_last_error()
        return m.decode() if m else ""

    def add_brick(self, dims, obstacle=None, velocity=None, tau: float = 0.55, force=(0.0, 0.0, 0.0),
                  faces=None, precision: int = 0) -> int:
        nx, ny, nz = (int(d) for d in dims)
        cells = nx * ny * nz
        ob = None if obstacle is None else np.ascontiguousarray(np.asarray(obstacle, np.uint8).reshape(-1))
        vel = None
        if velocity is not None:
            vel = np.ascontiguousarray(np.concatenate([np.asarray(v, np.float32).reshape(-1) for v in velocity]))
            assert vel.size == 3 * cells
        fo = np.ascontiguousarray(np.asarray(force, np.float32))
        fk = None if faces is None else np.ascontiguousarray(np.asarray(faces, np.int32))
        idx = ctypes.c_int(-1)
        ok = self.lib.aero_lbm_b200_batch_add_brick(
            self.handle, nx, ny, nz, int(precision), None if ob is None else u8ptr(ob),
            None if vel is None else fptr(vel), float(tau), fptr(fo),
            None if fk is None else fk.ctypes.data_as(_I32P), ctypes.byref(idx))
        if not ok:
            raise RuntimeError(self.error())
        self.dims.append((nx, ny, nz))
        return idx.value

    def finalize(self, stride: int = 4, velocity_scale: float = 20.0) -> None:
        if not self.lib.aero_lbm_b200_batch_finalize(self.handle, int(stride), float(velocity_scale)):
            raise RuntimeError(self.error())
        self.stride = stride

    def set_options(self, use_graph: bool = True, publish: bool = True) -> None:
        if not self.lib.aero_lbm_b200_batch_set_options(self.handle, int(use_graph), int(publish)):
            raise RuntimeError(self.error())

    def tick(self, n: int = 1) -> None:
        if not self.lib.aero_lbm_b200_batch_tick(self.handle, int(n)):
            raise RuntimeError(self.error())

    def autotune(self, trial_ticks: int = 4) -> tuple[int, int, float]:
        t, b, ms = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_float(0)
        if not self.lib.aero_lbm_b200_batch_autotune(self.handle, int(trial_ticks), ctypes.byref(t), ctypes.byref(b),
                                                      ctypes.byref(ms)):
            raise RuntimeError(self.error())
        return t.value, b.value, ms.value

    def info(self) -> dict:
        c, by, a, u, t = ctypes.c_longlong(0), ctypes.c_double(0), ctypes.c_int(0), ctypes.c_int(0), ctypes.c_longlong(0)
        self.lib.aero_lbm_b200_batch_info(self.handle, ctypes.byref(c), ctypes.byref(by), ctypes.byref(a), ctypes.byref(u),
                                          ctypes.byref(t))
        return {"cells": c.value, "bytes_per_tick": by.value, "atlas_records": a.value, "units": u.value,
                "ticks": t.value}

    def atlas(self, brick: int) -> np.ndarray:
        nx, ny, nz = self.dims[brick]
        s = self.stride
        n = ((nx + s - 1) // s) * ((ny + s - 1) // s) * ((nz + s - 1) // s)
        out = np.zeros(4 * n, np.int16)
        if not self.lib.aero_lbm_b200_batch_copy_atlas(self.handle, brick, out.ctypes.data_as(_I16P), out.size):
            raise RuntimeError(self.error())
        return out.reshape(n, 4)

    def flow(self, brick: int) -> np.ndarray:
        cells = int(np.prod(self.dims[brick]))
        out = np.zeros(4 * cells, np.float32)
        if not self.lib.aero_lbm_b200_batch_copy_flow(self.handle, brick, fptr(out), out.size):
            raise RuntimeError(self.error())
        return out.reshape(cells, 4)

    def close(self) -> None:
        if self.handle:
            self.lib.aero_lbm_b200_batch_destroy(self.handle)
            self.handle = 0


class MesoscaleContext:
    """A D3Q19 mesoscale grid (aero_lbm_mesoscale_* plus the B200 options).

    ``dims`` = (nx, ny, nz) with y up; forcing arrays are (cells, 25) float32,
    outputs (cells, 6)."""

    def __init__(self, dims, dx_m: float = 64.0, dt_s: float = 5.0, nu: float = 1.5e-5, prandtl: float = 0.71,
                 options: dict | None = None, lib: ctypes.CDLL | None = None):
        self.lib = lib or load_library()
        self.cfg = AeroLbmMesoscaleConfig()
        self.lib.aero_lbm_mesoscale_default_config(ctypes.byref(self.cfg))
        self.cfg.nx, self.cfg.ny, self.cfg.nz = (int(d) for d in dims)
        self.cfg.dx_m, self.cfg.dt_s, self.cfg.molecular_nu_m2_s, self.cfg.prandtl_air = dx_m, dt_s, nu, prandtl
        self.dims = tuple(int(d) for d in dims)
        self.cells = int(np.prod(self.dims))
        key = ctypes.c_longlong(0)
        if not self.lib.aero_lbm_mesoscale_create_context(ctypes.byref(self.cfg), ctypes.byref(key)):
            raise RuntimeError("mesoscale_create_context failed: " + last_error(self.lib))
        self.key = key.value
        if options:
            self.set_options(**options)

    def set_options(self, **kw) -> None:
        o = AeroLbmB200MesoscaleOptions()
        self.lib.aero_lbm_b200_mesoscale_default_options(ctypes.byref(o))
        for k, v in kw.items():
            if k == "body_force":
                for a in range(3):
                    o.body_force[a] = float(v[a])
            else:
                setattr(o, k, v)
        if not self.lib.aero_lbm_b200_mesoscale_set_options(self.key, ctypes.byref(o)):
            raise RuntimeError("mesoscale_set_options failed: " + last_error(self.lib))

    def step(self, forcing: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
        fo = np.ascontiguousarray(forcing, np.float32)
        if out is None:
            out = np.zeros((self.cells, 6), np.float32)
        if not self.lib.aero_lbm_mesoscale_step_context(self.key, ctypes.byref(self.cfg), fptr(fo), fptr(out)):
            raise RuntimeError("mesoscale_step_context failed: " + last_error(self.lib))
        return out

    def advance(self, steps: int) -> None:
        if not self.lib.aero_lbm_b200_mesoscale_advance(self.key, int(steps)):
            raise RuntimeError("mesoscale_advance failed: " + last_error(self.lib))

    def state(self) -> np.ndarray:
        out = np.zeros((self.cells, 6), np.float32)
        if not self.lib.aero_lbm_b200_mesoscale_read_state(self.key, fptr(out)):
            raise RuntimeError("mesoscale_read_state failed: " + last_error(self.lib))
        return out

    def info(self) -> dict:
        c, b = ctypes.c_longlong(0), ctypes.c_double(0)
        self.lib.aero_lbm_b200_mesoscale_info(self.key, ctypes.byref(c), ctypes.byref(b))
        return {"cells": c.value, "bytes_per_step": b.value}

    def release(self) -> None:
        if self.key:
            self.lib.aero_lbm_mesoscale_release_context(self.key)
            self.key = 0


def _dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class AdjointBrick:
    """Differentiable brick (aero_lbm_b200_adjoint_*): loss = sum over probes of
    |u - target|^2 after `steps` calls; gradients with respect to the body-force
    field (3, nx, ny, nz) and the inflow vector."""

    def __init__(self, obstacle: np.ndarray, temperature: np.ndarray | None = None, lib: ctypes.CDLL | None = None,
                 **config):
        self.lib = lib or load_library()
        cfg = AeroLbmB200AdjointConfig()
        self.lib.aero_lbm_b200_adjoint_default_config(ctypes.byref(cfg))
        cfg.nx, cfg.ny, cfg.nz = obstacle.shape
        for k, v in config.items():
            if k == "face_kind":
                for i in range(6):
                    cfg.face_kind[i] = int(v[i])
            else:
                setattr(cfg, k, v)
        self.cfg = cfg
        self.dims = tuple(obstacle.shape)
        self.cells = int(np.prod(self.dims))
        ob = np.ascontiguousarray(obstacle, np.uint8)
        tp = None if temperature is None else np.ascontiguousarray(temperature, np.float32)
        h = ctypes.c_longlong(0)
        if not self.lib.aero_lbm_b200_adjoint_create(ctypes.byref(cfg), u8ptr(ob), fptr(tp) if tp is not None else None,
                                                     ctypes.byref(h)):
            raise RuntimeError("adjoint_create failed: " + self.error())
        self.handle = h.value

    def error(self) -> str:
        m = self.lib.aero_lbm_b200_adjoint_last_error()
        return m.decode() if m else ""

    def set_probes(self, cells: np.ndarray, targets: np.ndarray) -> None:
        c = np.ascontiguousarray(cells, np.int32)
        t = np.ascontiguousarray(targets, np.float32).reshape(-1)
        if not self.lib.aero_lbm_b200_adjoint_set_probes(self.handle, c.size, c.ctypes.data_as(_I32P), fptr(t)):
            raise RuntimeError("adjoint_set_probes failed: " + self.error())
        self.nprobe = c.size

    def forward(self, force: np.ndarray | None, inflow, precision: int = 0):
        fo = None if force is None else np.ascontiguousarray(force, np.float32).reshape(-1)
        ui = np.ascontiguousarray(inflow, np.float32)
        loss = np.zeros(1, np.float64)
        u = np.zeros(3 * self.nprobe, np.float32)
        if not self.lib.aero_lbm_b200_adjoint_forward(self.handle, fptr(fo) if fo is not None else None, fptr(ui),
                                                      precision, _dptr(loss), fptr(u)):
            raise RuntimeError("adjoint_forward failed: " + self.error())
        return float(loss[0]), u.reshape(-1, 3)

    def gradient(self, force: np.ndarray | None, inflow):
        fo = None if force is None else np.ascontiguousarray(force, np.float32).reshape(-1)
        ui = np.ascontiguousarray(inflow, np.float32)
        loss = np.zeros(1, np.float64)
        gf = np.zeros(3 * self.cells, np.float64)
        gu = np.zeros(3, np.float64)
        if not self.lib.aero_lbm_b200_adjoint_gradient(self.handle, fptr(fo) if fo is not None else None, fptr(ui),
                                                       _dptr(loss), _dptr(gf), _dptr(gu)):
            raise RuntimeError("adjoint_gradient failed: " + self.error())
        return float(loss[0]), gf.reshape((3,) + self.dims), gu

    def timing(self) -> dict:
        v = [ctypes.c_double(0) for _ in range(4)]
        self.lib.aero_lbm_b200_adjoint_timing(self.handle, *[ctypes.byref(x) for x in v])
        return {"forward_ms_per_step": v[0].value, "recompute_ms_per_step": v[1].value,
                "reverse_ms_per_step": v[2].value, "total_ms": v[3].value}

    def close(self) -> None:
        if self.handle:
            self.lib.aero_lbm_b200_adjoint_destroy(self.handle)
            self.handle = 0
