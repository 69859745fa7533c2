"""ORACLE — test infrastructure only (imported by tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg; never by the product).

Two checkers live here:

* ``RefLib`` drives the reference library itself (the unmodified reference CPU
  path compiled by ``make ref`` into oracle/_ref/libaero_lbm_ref.so) through its
  C ABI, like the reference's own ctypes tools do.
* ``Oracle`` drives liboracle.so, the C++ restatement of the reference step
  (d3q27_oracle.cpp), in float (bit-exact with the reference) or double (the
  FP64 run of the same scheme), with the knobs the reference hard-codes.

``derive_params`` restates, in float32, how the reference turns its boundary
configuration into relaxation times (native/src/aero_lbm_jni.cpp:831-1031).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libaero_lbm_ref.so"
REFERENCE_SOURCE = Path(os.environ.get("AERO_REFERENCE_NATIVE", "/root/reference/native"))

f32 = np.float32

# Face kinds / flags (same numbering as the C ABI).
PERIODIC, BOUNCE_BACK, MOVING_WALL, VELOCITY, PRESSURE, CONVECTIVE, SYMMETRY = 1, 2, 3, 4, 5, 6, 7
INHERIT_GAME = 0
# thermal face kinds (native/include/aero_lbm_capi.h:57-62)
THERMAL_INHERIT, THERMAL_DISABLED, THERMAL_PERIODIC, THERMAL_ADIABATIC, THERMAL_DIRICHLET, THERMAL_NEUMANN = 0, 1, 2, 3, 4, 5
PRESET_HEATED_CAVITY_2D, PRESET_HEATED_CAVITY_3D = 5, 6  # native/include/aero_lbm_capi.h:41-42
PRESET_CYLINDER_2D = 4  # native/include/aero_lbm_capi.h:40
FLAG_DISABLE_FAN_FORCING, FLAG_DISABLE_FAN_NOISE, FLAG_DISABLE_SPONGE = 1 << 0, 1 << 1, 1 << 2
FLAG_DISABLE_CONVECTIVE_OUTFLOW = 1 << 3
FLAG_DISABLE_SGS = 1 << 5
FLAG_DISABLE_BUOYANCY = 1 << 7


def build(ref: bool | None = None) -> None:
    """Compile liboracle.so (always) and the reference library (when its
    sources are present and ``ref`` is not False); with the product library
    built, also the reference's brick service over both libraries."""
    subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    if ref is None:
        ref = REFERENCE_SOURCE.exists()
    if ref:
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={REFERENCE_SOURCE}"], check=True)
        if (HERE.parent / "aerodynamics4mc-fabric_b200" / "libaero_lbm_b200.so").exists():
            subprocess.run(["make", "-s", "-C", str(HERE), "sim", f"REF={REFERENCE_SOURCE}"], check=True)


# ---------------------------------------------------------------- parameter derivation
class OracleParams(ctypes.Structure):
    _fields_ = [
        ("tau_shear", ctypes.c_double),
        ("tau_normal", ctypes.c_double),
        ("nu0", ctypes.c_double),
        ("sgs_c2", ctypes.c_double),
        ("sgs_nut_max_ratio", ctypes.c_double),
        ("sgs_bulk_coupling", ctypes.c_double),
        ("buoyancy_beta", ctypes.c_double),
        ("buoyancy_force_max", ctypes.c_double),
        ("body_force", ctypes.c_double * 3),
        ("max_speed", ctypes.c_double),
        ("face_velocity", (ctypes.c_double * 3) * 6),
        ("face_pressure", ctypes.c_double * 6),
        ("face_kind", ctypes.c_int * 6),
        ("enable_sgs", ctypes.c_int),
        ("enable_buoyancy", ctypes.c_int),
        ("gravity_axis", ctypes.c_int),
        ("disable_convective_outflow", ctypes.c_int),
        ("thermal_transport", ctypes.c_int),
        ("thermal_kind", ctypes.c_int * 6),
        ("face_temperature", ctypes.c_double * 6),
        ("face_heat_flux", ctypes.c_double * 6),
        ("thermal_diffusivity", ctypes.c_double),
        ("initial_temperature", ctypes.c_double),
        ("internal_thermal_source", ctypes.c_int),
        ("packet_has_temperature", ctypes.c_int),
        ("thermal_bfecc", ctypes.c_int),
        ("cylinder_force", ctypes.c_int),
        ("fan_forcing", ctypes.c_int),
        ("fan_noise_amp", ctypes.c_double),
        ("sponge", ctypes.c_int),
        ("state_nudge", ctypes.c_double),
        ("runtime_mode", ctypes.c_int),
        ("packet_has_source", ctypes.c_int),
    ]


def _clamp(v, lo, hi):
    return f32(min(f32(hi), max(f32(lo), f32(v))))


NU_MIN = f32(1.0e-8)
NU_MAX = (f32(0.95) - f32(0.5)) / f32(3.0)
TAU_MIN = f32(0.5) + f32(3.0) * f32(1.0e-8)
TAU_MAX = f32(0.95)
MAX_SPEED = f32(0.57735026919) * f32(0.60)
RUNTIME_NU0 = f32(1.50e-5) * (f32(1.0) / f32(20.0)) / (f32(1.0) * f32(1.0))
BOUSSINESQ_BETA = f32(9.81) * (f32(1.0) / f32(300.0)) * f32(20.0) * ((f32(1.0) / f32(20.0)) * (f32(1.0) / f32(20.0)) / f32(1.0))


def _norm(v):
    """sqrt(x*x + y*y + z*z) evaluated left to right in float32."""
    x, y, z = (f32(a) for a in v)
    return f32(np.sqrt(f32(f32(x * x + y * y) + z * z)))


def derive_params(cfg: dict) -> OracleParams:
    """Benchmark-mode effective parameters, restated from
    native/src/aero_lbm_jni.cpp:831-871 (reference speed), 947-979 (nu, tau),
    1023-1031 (beta). ``cfg`` keys: reynolds, reference_length,
    initial_velocity, faces (list of 6 dicts: kind, velocity, pressure),
    sgs (bool), buoyancy (bool), smagorinsky_c, buoyancy_beta, gravity_axis,
    body_force, disable_convective; temperature transport: thermal_transport
    (bool, the reference's benchmark-mode scalar transport), initial_temperature,
    thermal_source (bool), packet_channels; per face thermal (kind),
    temperature, heat_flux."""
    faces = cfg["faces"]
    length = max(f32(1.0e-6), f32(cfg.get("reference_length", 1.0)))
    cavity = int(cfg.get("preset", 0)) in (PRESET_HEATED_CAVITY_2D, PRESET_HEATED_CAVITY_3D)
    if cavity:
        # heated-cavity presets (jni.cpp:824-829, 947-954, 966-970, 1023-1031)
        speed = _clamp(cfg.get("mach", 0.15), 1.0e-4, 0.30) * f32(np.sqrt(f32(1.0) / f32(3.0)))
        ra = max(f32(1.0e-6), f32(cfg.get("rayleigh", 1.0e5)))
        pr = max(f32(1.0e-6), f32(cfg.get("prandtl", 0.71)))
        nu = _clamp(f32(speed * length) * f32(np.sqrt(f32(pr / ra))), NU_MIN, NU_MAX)
    elif int(cfg.get("preset", 0)) == PRESET_CYLINDER_2D:
        # benchmark_reference_speed, cylinder branch (jni.cpp:830-843)
        speed = _norm(cfg.get("initial_velocity", (0, 0, 0)))
        if speed <= f32(1.0e-8):
            speed = f32(f32(2.0) / f32(3.0)) * _norm(faces[0].get("velocity", (0, 0, 0)))
    else:
        speed = _norm(cfg.get("initial_velocity", (0, 0, 0)))
        for fc in faces:
            speed = max(speed, _norm(fc.get("velocity", (0, 0, 0))))
    if not cavity:
        re = f32(cfg.get("reynolds", 100.0))
        if re <= f32(1.0e-6) or speed <= f32(1.0e-8):
            nu = _clamp(RUNTIME_NU0, NU_MIN, NU_MAX)
        else:
            nu = _clamp(f32(speed * length) / re, NU_MIN, NU_MAX)
    tau_s = _clamp(f32(0.5) + f32(3.0) * _clamp(nu, NU_MIN, NU_MAX), TAU_MIN, TAU_MAX)
    tau_n = _clamp(f32(0.5) + f32(3.0) * _clamp(_clamp(nu, NU_MIN, NU_MAX), NU_MIN, NU_MAX), TAU_MIN, TAU_MAX)
    p = OracleParams()
    p.tau_shear = float(tau_s)
    p.tau_normal = float(tau_n)
    p.nu0 = float(max(f32(1e-6), nu))
    c = f32(cfg.get("smagorinsky_c", 0.025))
    p.sgs_c2 = float(f32(c * c))
    p.sgs_nut_max_ratio = 5.0
    p.sgs_bulk_coupling = float(f32(0.30))
    beta = BOUSSINESQ_BETA
    if cavity:
        temps = [f32(fc.get("temperature", 0.0)) for fc in faces if fc.get("thermal") == THERMAL_DIRICHLET]
        span = max(f32(1.0e-6), f32(max(temps) - min(temps))) if temps else f32(1.0)
        beta = f32(speed * speed) / max(f32(1.0e-6), f32(length * span))
    p.buoyancy_beta = float(f32(cfg.get("buoyancy_beta", beta)))
    p.buoyancy_force_max = float(f32(0.02))
    for i, v in enumerate(cfg.get("body_force", (0.0, 0.0, 0.0))):
        p.body_force[i] = float(f32(v))
    p.max_speed = float(MAX_SPEED)
    for i, fc in enumerate(faces):
        p.face_kind[i] = int(fc.get("kind", INHERIT_GAME))
        for a, v in enumerate(fc.get("velocity", (0, 0, 0))):
            p.face_velocity[i][a] = float(f32(v))
        p.face_pressure[i] = float(f32(fc.get("pressure", 0.0)))
    p.enable_sgs = 1 if cfg.get("sgs", False) else 0
    p.enable_buoyancy = 1 if cfg.get("buoyancy", False) else 0
    p.gravity_axis = int(cfg.get("gravity_axis", 1))
    p.disable_convective_outflow = 1 if cfg.get("disable_convective", False) else 0
    # the product's default: transport whenever buoyancy is on
    p.thermal_transport = 1 if cfg.get("thermal_transport", cfg.get("buoyancy", False)) else 0
    for i, fc in enumerate(faces):
        p.thermal_kind[i] = int(fc.get("thermal", THERMAL_DISABLED))
        p.face_temperature[i] = float(f32(fc.get("temperature", 0.0)))
        p.face_heat_flux[i] = float(f32(fc.get("heat_flux", 0.0)))
    p.thermal_diffusivity = float(f32(nu / pr) if cavity else f32(0.035))
    p.thermal_bfecc = 1 if cavity else 0
    p.initial_temperature = float(f32(cfg.get("initial_temperature", 0.0)))
    p.internal_thermal_source = 1 if cfg.get("thermal_source", False) else 0
    p.packet_has_temperature = 1 if int(cfg.get("packet_channels", 11)) > 10 else 0
    p.packet_has_source = 1 if int(cfg.get("packet_channels", 11)) > 9 else 0
    p.cylinder_force = 1 if int(cfg.get("preset", 0)) == PRESET_CYLINDER_2D else 0
    # fan forcing, fan noise and the sponge: off unless the config clears their
    # DISABLE flags (the default config sets them)
    p.fan_forcing = 1 if cfg.get("fans", False) else 0
    p.fan_noise_amp = float(f32(0.02)) if (cfg.get("fans", False) and cfg.get("fan_noise", False)) else 0.0
    p.sponge = 1 if cfg.get("sponge", False) else 0
    p.state_nudge = 0.0
    if not cfg.get("benchmark", True):
        runtime_params(p)
    return p


def runtime_params(p: OracleParams) -> None:
    """Benchmark mode off (aero_lbm_benchmark_reset_config): the reference's
    game-runtime constants (jni.cpp:87-168, 676-1031): molecular viscosity
    and diffusivity of air at 1 m cells and 1/20 s steps, SGS, buoyancy,
    fans with noise, sponge, state nudge, the temperature transport (BFECC,
    every other call, local eddy diffusivity) and the default config's faces
    (INHERIT_GAME: convective outflow, thermal self)."""
    nu = _clamp(RUNTIME_NU0, NU_MIN, NU_MAX)
    p.tau_shear = float(_clamp(f32(0.5) + f32(3.0) * nu, TAU_MIN, TAU_MAX))
    p.tau_normal = float(_clamp(f32(0.5) + f32(3.0) * RUNTIME_NU0, TAU_MIN, TAU_MAX))
    p.nu0 = float(max(f32(1e-6), nu))
    p.sgs_c2 = float(f32(f32(0.025) * f32(0.025)))
    p.enable_sgs = 1
    p.enable_buoyancy = 1
    p.buoyancy_beta = float(BOUSSINESQ_BETA)
    p.gravity_axis = 1
    for i in range(3):
        p.body_force[i] = 0.0
    for i in range(6):
        p.face_kind[i] = INHERIT_GAME
        p.thermal_kind[i] = THERMAL_INHERIT
        p.face_pressure[i] = 0.0
        for a in range(3):
            p.face_velocity[i][a] = 0.0
    p.disable_convective_outflow = 0
    p.thermal_transport = 1
    p.thermal_bfecc = 1
    alpha0 = f32(f32(f32(1.50e-5) / f32(0.71)) * f32(f32(1.0) / f32(20.0))) / f32(f32(1.0) * f32(1.0))
    p.thermal_diffusivity = float(max(f32(1.0e-8), alpha0))
    p.internal_thermal_source = 1
    p.fan_forcing = 1
    p.fan_noise_amp = float(f32(0.02))
    p.sponge = 1
    p.state_nudge = float(f32(0.08))
    p.runtime_mode = 1


# ---------------------------------------------------------------- oracle (restatement)
class Oracle:
    """CPU restatement of the reference D3Q27 step; precision 'f32' or 'f64'."""

    _lib = None

    @classmethod
    def lib(cls) -> ctypes.CDLL:
        if cls._lib is None:
            if not ORACLE_LIB.exists():
                build(ref=False)
            lib = ctypes.CDLL(str(ORACLE_LIB))
            lib.oracle_d3q27_create.restype = ctypes.c_void_p
            lib.oracle_d3q27_create.argtypes = [ctypes.c_int] * 4 + [ctypes.POINTER(OracleParams)]
            lib.oracle_d3q27_destroy.argtypes = [ctypes.c_void_p]
            lib.oracle_d3q27_set_fields.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 6
            lib.oracle_d3q27_set_force_field.argtypes = [ctypes.c_void_p] * 4
            lib.oracle_d3q27_set_params.argtypes = [ctypes.c_void_p, ctypes.POINTER(OracleParams)]
            lib.oracle_d3q27_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
            lib.oracle_d3q27_output.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p]
            lib.oracle_d3q27_extract_atlas.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
            lib.oracle_d3q27_macro.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.oracle_d3q27_get_f.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.oracle_d3q27_set_thermal_source.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.oracle_d3q27_get_temperature.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.oracle_d3q27_set_temperature.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.oracle_d3q27_exchange_halo.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 4
            lib.oracle_d3q27_apply_overlays.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
            lib.oracle_d3q27_shift.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 3
            lib.oracle_d3q27_last_force.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.oracle_d3q27_get_obstacle.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.oracle_d3q27_patch_cells.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
            lib.oracle_d3q27_set_fans.argtypes = [ctypes.c_void_p] * 5
            lib.oracle_d3q27_set_shell.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 3 + [ctypes.c_float]
            cls._lib = lib
        return cls._lib

    def __init__(self, dims, params: OracleParams, precision: str = "f32"):
        self.dims = tuple(int(d) for d in dims)
        self.cells = int(np.prod(self.dims))
        self.h = self.lib().oracle_d3q27_create(*self.dims, 0 if precision == "f32" else 1, ctypes.byref(params))
        if not self.h:
            raise ValueError("oracle_d3q27_create failed")
        self._keep = []

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().oracle_d3q27_destroy(self.h)
            self.h = None

    @staticmethod
    def _p(a, dtype):
        if a is None:
            return None, None
        arr = np.ascontiguousarray(np.asarray(a, dtype=dtype).reshape(-1))
        return arr, arr.ctypes.data

    def set_fields(self, obstacle, ux=None, uy=None, uz=None, pressure=None, temperature=None):
        arrs = [self._p(obstacle, np.uint8)] + [self._p(v, np.float32) for v in (ux, uy, uz, pressure, temperature)]
        self._keep = [a for a, _ in arrs]
        self.lib().oracle_d3q27_set_fields(self.h, *[p for _, p in arrs])

    def set_thermal_source(self, src):
        arr, ptr = self._p(src, np.float32)
        self._keep_src = arr
        self.lib().oracle_d3q27_set_thermal_source(self.h, ptr)

    def temperature(self) -> np.ndarray:
        out = np.zeros(self.cells, dtype=np.float32)
        self.lib().oracle_d3q27_get_temperature(self.h, out.ctypes.data)
        return out

    def exchange_halo(self, other: "Oracle", offset, halo_layers: int):
        if not self.lib().oracle_d3q27_exchange_halo(self.h, other.h, *[int(v) for v in offset], int(halo_layers)):
            raise RuntimeError("oracle halo exchange failed")

    def apply_overlays(self, cells, values):
        c = np.ascontiguousarray(np.asarray(cells, np.int32).reshape(-1))
        v = np.ascontiguousarray(np.asarray(values, np.float32).reshape(-1, 6))
        if not self.lib().oracle_d3q27_apply_overlays(self.h, c.ctypes.data, v.ctypes.data, int(c.size)):
            raise RuntimeError("oracle overlays failed")

    def shift(self, dx: int, dy: int, dz: int) -> bool:
        return bool(self.lib().oracle_d3q27_shift(self.h, int(dx), int(dy), int(dz)))

    def set_fans(self, mask, vx, vy, vz):
        arrs = [self._p(v, np.float32) for v in (mask, vx, vy, vz)]
        self._keep_fans = [a for a, _ in arrs]
        if not self.lib().oracle_d3q27_set_fans(self.h, *[p for _, p in arrs]):
            raise RuntimeError("oracle set_fans failed")

    def patch_cells(self, cells, solid):
        c = np.ascontiguousarray(np.asarray(cells, np.int32).reshape(-1))
        s = np.ascontiguousarray(np.asarray(solid, np.uint8).reshape(-1))
        if not self.lib().oracle_d3q27_patch_cells(self.h, c.ctypes.data, s.ctypes.data, int(c.size)):
            raise RuntimeError("oracle patch failed")

    def set_shell(self, flow, face_mask: int, layers: int, relaxation: float):
        fl = np.ascontiguousarray(np.asarray(flow, np.float32).reshape(self.cells, -1))
        self._shell_flow = fl
        self.lib().oracle_d3q27_set_shell(self.h, fl.ctypes.data, fl.shape[1], int(face_mask), int(layers),
                                          float(relaxation))

    def mask(self) -> np.ndarray:
        out = np.zeros(self.cells, np.uint8)
        self.lib().oracle_d3q27_get_obstacle(self.h, out.ctypes.data)
        return out

    def last_force(self) -> np.ndarray:
        out = np.zeros(3, np.float32)
        self.lib().oracle_d3q27_last_force(self.h, out.ctypes.data)
        return out

    def set_temperature(self, t):
        arr = np.ascontiguousarray(np.asarray(t, np.float32).reshape(-1))
        self.lib().oracle_d3q27_set_temperature(self.h, arr.ctypes.data)

    def set_force_field(self, fx, fy, fz):
        arrs = [self._p(v, np.float32) for v in (fx, fy, fz)]
        self.lib().oracle_d3q27_set_force_field(self.h, *[p for _, p in arrs])

    def set_params(self, params: OracleParams):
        self.lib().oracle_d3q27_set_params(self.h, ctypes.byref(params))

    def step(self, n: int = 1):
        if not self.lib().oracle_d3q27_step(self.h, int(n)):
            raise RuntimeError("oracle step failed")

    def output(self, scale: float = 1.0) -> np.ndarray:
        out = np.zeros(self.cells * 4, dtype=np.float32)
        self.lib().oracle_d3q27_output(self.h, ctypes.c_float(scale), out.ctypes.data)
        return out.reshape(self.cells, 4)

    def atlas(self, stride: int) -> np.ndarray:
        n = [(d + stride - 1) // stride for d in self.dims]
        out = np.zeros(int(np.prod(n)) * 4, dtype=np.float32)
        if not self.lib().oracle_d3q27_extract_atlas(self.h, stride, out.ctypes.data, out.size):
            raise RuntimeError("atlas extraction failed")
        return out.reshape(-1, 4)

    def macro(self) -> np.ndarray:
        out = np.zeros(self.cells * 4, dtype=np.float64)
        self.lib().oracle_d3q27_macro(self.h, out.ctypes.data)
        return out.reshape(self.cells, 4)

    def populations(self) -> np.ndarray:
        out = np.zeros(self.cells * 27, dtype=np.float64)
        self.lib().oracle_d3q27_get_f(self.h, out.ctypes.data)
        return out.reshape(27, self.cells)


# ---------------------------------------------------------------- the reference library itself
class _Face(ctypes.Structure):
    _fields_ = [("hydrodynamic_kind", ctypes.c_int), ("thermal_kind", ctypes.c_int), ("velocity", ctypes.c_float * 3),
                ("pressure", ctypes.c_float), ("temperature", ctypes.c_float), ("heat_flux", ctypes.c_float)]


class RefBenchmarkConfig(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_uint32), ("struct_size", ctypes.c_uint32), ("flags", ctypes.c_uint32),
        ("enabled", ctypes.c_int), ("preset", ctypes.c_int), ("reserved0", ctypes.c_int),
        ("reynolds_number", ctypes.c_float), ("rayleigh_number", ctypes.c_float), ("prandtl_number", ctypes.c_float),
        ("mach_number", ctypes.c_float), ("reference_density", ctypes.c_float), ("reference_temperature", ctypes.c_float),
        ("reference_length", ctypes.c_float), ("body_force", ctypes.c_float * 3), ("gravity", ctypes.c_float * 3),
        ("initial_velocity", ctypes.c_float * 3), ("initial_pressure", ctypes.c_float), ("initial_temperature", ctypes.c_float),
        ("x_min", _Face), ("x_max", _Face), ("y_min", _Face), ("y_max", _Face), ("z_min", _Face), ("z_max", _Face),
        ("reserved", ctypes.c_uint32 * 8),
    ]


def config_struct(struct_type, cfg: dict, default_fn):
    """Fill a reference-layout benchmark config from the dict form used by
    derive_params, starting from the library's own default config."""
    c = struct_type()
    default_fn(ctypes.byref(c))
    c.enabled = 1
    c.preset = int(cfg.get("preset", 0))
    if c.preset:
        c.rayleigh_number = cfg.get("rayleigh", 1.0e5)
        c.prandtl_number = cfg.get("prandtl", 0.71)
        c.mach_number = cfg.get("mach", 0.15)
    flags = c.flags
    flags = (flags & ~FLAG_DISABLE_SGS) if cfg.get("sgs", False) else (flags | FLAG_DISABLE_SGS)
    flags = (flags & ~FLAG_DISABLE_BUOYANCY) if cfg.get("buoyancy", False) else (flags | FLAG_DISABLE_BUOYANCY)
    if not cfg.get("thermal_source", False):
        flags |= 1 << 6  # DISABLE_INTERNAL_THERMAL_SOURCE
    else:
        flags &= ~(1 << 6)
    if cfg.get("disable_convective", False):
        flags |= FLAG_DISABLE_CONVECTIVE_OUTFLOW
    for key, bit in (("fans", FLAG_DISABLE_FAN_FORCING), ("fan_noise", FLAG_DISABLE_FAN_NOISE),
                     ("sponge", FLAG_DISABLE_SPONGE)):
        if key in cfg:
            flags = (flags & ~bit) if cfg[key] else (flags | bit)
    c.flags = flags
    c.reynolds_number = cfg.get("reynolds", 100.0)
    c.initial_temperature = cfg.get("initial_temperature", 0.0)
    c.reference_length = cfg.get("reference_length", 1.0)
    for i, v in enumerate(cfg.get("initial_velocity", (0, 0, 0))):
        c.initial_velocity[i] = v
    for i, v in enumerate(cfg.get("body_force", (0, 0, 0))):
        c.body_force[i] = v
    for name, fc in zip(("x_min", "x_max", "y_min", "y_max", "z_min", "z_max"), cfg["faces"]):
        face = getattr(c, name)
        face.hydrodynamic_kind = int(fc.get("kind", INHERIT_GAME))
        face.thermal_kind = int(fc.get("thermal", THERMAL_DISABLED))
        face.temperature = fc.get("temperature", 0.0)
        face.heat_flux = fc.get("heat_flux", 0.0)
        for a, v in enumerate(fc.get("velocity", (0, 0, 0))):
            face.velocity[a] = v
        face.pressure = fc.get("pressure", 0.0)
    return c


class RefLib:
    """The reference's CPU library (oracle/_ref), driven through its C ABI."""

    def __init__(self, path: Path = REF_LIB):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} missing (build with `make -C oracle ref`)")
        lib = ctypes.CDLL(str(path))
        lib.aero_lbm_init_rect.argtypes = [ctypes.c_int] * 5
        lib.aero_lbm_init_rect.restype = ctypes.c_int
        lib.aero_lbm_step_rect.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p]
        lib.aero_lbm_step_rect.restype = ctypes.c_int
        lib.aero_lbm_extract_flow_atlas_rect.argtypes = [ctypes.c_int] * 3 + [ctypes.c_longlong, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        lib.aero_lbm_extract_flow_atlas_rect.restype = ctypes.c_int
        lib.aero_lbm_benchmark_default_config.argtypes = [ctypes.c_void_p]
        lib.aero_lbm_benchmark_set_config.argtypes = [ctypes.c_void_p]
        lib.aero_lbm_benchmark_set_config.restype = ctypes.c_int
        lib.aero_lbm_last_error.restype = ctypes.c_char_p
        lib.aero_lbm_set_temperature_state_rect.argtypes = [ctypes.c_int] * 3 + [ctypes.c_longlong, ctypes.c_void_p]
        lib.aero_lbm_set_temperature_state_rect.restype = ctypes.c_int
        lib.aero_lbm_get_temperature_state_rect.argtypes = [ctypes.c_int] * 3 + [ctypes.c_longlong, ctypes.c_void_p]
        lib.aero_lbm_get_temperature_state_rect.restype = ctypes.c_int
        lib.aero_lbm_runtime_info.restype = ctypes.c_char_p
        self.lib = lib

    def run(self, dims, cfg: dict, packet: np.ndarray, steps: int, out_every: int | None = None, key: int = 1,
            temperature_state: np.ndarray | None = None):
        """Initialise, configure and step; returns the final write_output
        (cells x 4) from the last step. ``temperature_state``: loaded with
        aero_lbm_set_temperature_state_rect before the first step. The
        temperature state after the last step is left in ``self.temperature``."""
        nx, ny, nz = dims
        lib = self.lib
        if not lib.aero_lbm_init_rect(nx, ny, nz, packet.shape[1], 4):
            raise RuntimeError(lib.aero_lbm_last_error())
        c = config_struct(RefBenchmarkConfig, cfg, lib.aero_lbm_benchmark_default_config)
        if not lib.aero_lbm_benchmark_set_config(ctypes.byref(c)):
            raise RuntimeError("set_config failed")
        cells = nx * ny * nz
        if temperature_state is not None:
            t = np.ascontiguousarray(np.asarray(temperature_state, np.float32).reshape(-1))
            if not lib.aero_lbm_set_temperature_state_rect(nx, ny, nz, key, t.ctypes.data):
                raise RuntimeError(lib.aero_lbm_last_error())
        out = np.zeros(nx * ny * nz * 4, dtype=np.float32)
        pk = np.ascontiguousarray(packet, dtype=np.float32)
        for s in range(steps):
            want = (s + 1 == steps) or (out_every and (s + 1) % out_every == 0)
            if not lib.aero_lbm_step_rect(pk.ctypes.data, nx, ny, nz, key, out.ctypes.data if want else None):
                raise RuntimeError(lib.aero_lbm_last_error())
        self.temperature = np.zeros(cells, dtype=np.float32)
        if not lib.aero_lbm_get_temperature_state_rect(nx, ny, nz, key, self.temperature.ctypes.data):
            raise RuntimeError(lib.aero_lbm_last_error())
        return out.reshape(-1, 4)


    def run_pair(self, dims, cfg: dict, packets, steps: int, offset, halo_layers: int, exchange_every: int = 1,
                 keys=(1, 2), temperature_states=(None, None)):
        """Two contexts stepped call for call, aero_lbm_exchange_halo_layers_rect
        between them after every ``exchange_every`` calls (not after the
        last); returns both write_output results of the last call and leaves
        both temperature states in ``self.temperatures``."""
        nx, ny, nz = dims
        lib = self.lib
        lib.aero_lbm_exchange_halo_layers_rect.argtypes = [ctypes.c_int] * 4 + [ctypes.c_longlong] * 2 + [ctypes.c_int] * 3
        lib.aero_lbm_exchange_halo_layers_rect.restype = ctypes.c_int
        if not lib.aero_lbm_init_rect(nx, ny, nz, packets[0].shape[1], 4):
            raise RuntimeError(lib.aero_lbm_last_error())
        if cfg.get("benchmark", True):
            c = config_struct(RefBenchmarkConfig, cfg, lib.aero_lbm_benchmark_default_config)
            if not lib.aero_lbm_benchmark_set_config(ctypes.byref(c)):
                raise RuntimeError("set_config failed")
        else:
            lib.aero_lbm_benchmark_reset_config()
        for key, ts in zip(keys, temperature_states):
            if ts is not None:
                t = np.ascontiguousarray(np.asarray(ts, np.float32).reshape(-1))
                if not lib.aero_lbm_set_temperature_state_rect(nx, ny, nz, key, t.ctypes.data):
                    raise RuntimeError(lib.aero_lbm_last_error())
        outs = [np.zeros(nx * ny * nz * 4, dtype=np.float32) for _ in keys]
        pks = [np.ascontiguousarray(p, dtype=np.float32) for p in packets]
        for s in range(steps):
            last = s + 1 == steps
            for key, pk, out in zip(keys, pks, outs):
                if not lib.aero_lbm_step_rect(pk.ctypes.data, nx, ny, nz, key, out.ctypes.data if last else None):
                    raise RuntimeError(lib.aero_lbm_last_error())
            if not last and (s + 1) % exchange_every == 0:
                if not lib.aero_lbm_exchange_halo_layers_rect(nx, ny, nz, halo_layers, keys[0], keys[1], *offset):
                    raise RuntimeError(lib.aero_lbm_last_error())
        self.temperatures = []
        for key in keys:
            t = np.zeros(nx * ny * nz, dtype=np.float32)
            lib.aero_lbm_get_temperature_state_rect(nx, ny, nz, key, t.ctypes.data)
            self.temperatures.append(t)
        return [o.reshape(-1, 4) for o in outs]


    def run_script(self, dims, cfg: dict, packet: np.ndarray, script, key: int = 1, temperature_state=None):
        """A context driven through a list of calls (see ``run_script_oracle``
        for the actions); returns the recorded results in order."""
        nx, ny, nz = dims
        lib = self.lib
        vp, i, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
        lib.aero_lbm_step_rect_with_sparse_overlays.argtypes = [vp, i, i, i, ll, vp, vp, i, vp]
        lib.aero_lbm_get_flow_state_rect.argtypes = [i, i, i, ll, vp]
        lib.aero_lbm_shift_context.argtypes = [i, ll, i, i, i]
        lib.aero_lbm_get_last_force.argtypes = [ll, vp, vp, vp]
        lib.aero_lbm_sample_flow_point_rect.argtypes = [i, i, i, ll, i, i, i, vp]
        lib.aero_lbm_sample_temperature_point_rect.argtypes = [i, i, i, ll, i, i, i, vp]
        lib.aero_lbm_copy_flow_temperature_subrect.argtypes = [i, i, i, ll] + [i] * 6 + [vp, vp]
        if not lib.aero_lbm_init_rect(nx, ny, nz, packet.shape[1], 4):
            raise RuntimeError(lib.aero_lbm_last_error())
        if cfg.get("benchmark", True):
            c = config_struct(RefBenchmarkConfig, cfg, lib.aero_lbm_benchmark_default_config)
            if not lib.aero_lbm_benchmark_set_config(ctypes.byref(c)):
                raise RuntimeError("set_config failed")
        else:
            lib.aero_lbm_benchmark_reset_config()
        cells = nx * ny * nz
        if temperature_state is not None:
            t = np.ascontiguousarray(np.asarray(temperature_state, np.float32).reshape(-1))
            if not lib.aero_lbm_set_temperature_state_rect(nx, ny, nz, key, t.ctypes.data):
                raise RuntimeError(lib.aero_lbm_last_error())
        pk = np.ascontiguousarray(packet, dtype=np.float32)
        results = []
        for act in script:
            kind = act[0]
            if kind == "step":
                ov = act[1] if len(act) > 1 else None
                if ov is None:
                    ok = lib.aero_lbm_step_rect(pk.ctypes.data, nx, ny, nz, key, None)
                else:
                    oc = np.ascontiguousarray(ov[0], np.int32)
                    vals = np.ascontiguousarray(ov[1], np.float32)
                    ok = lib.aero_lbm_step_rect_with_sparse_overlays(pk.ctypes.data, nx, ny, nz, key, oc.ctypes.data,
                                                                     vals.ctypes.data, int(oc.size), None)
                if not ok:
                    raise RuntimeError(lib.aero_lbm_last_error())
            elif kind == "flow":
                out = np.zeros(cells * 4, np.float32)
                if not lib.aero_lbm_get_flow_state_rect(nx, ny, nz, key, out.ctypes.data):
                    raise RuntimeError(lib.aero_lbm_last_error())
                results.append(out.reshape(-1, 4))
            elif kind == "temp":
                t = np.zeros(cells, np.float32)
                lib.aero_lbm_get_temperature_state_rect(nx, ny, nz, key, t.ctypes.data)
                results.append(t)
            elif kind == "shift":
                if not lib.aero_lbm_shift_context(nx, key, *act[1:4]):
                    raise RuntimeError("shift failed")
            elif kind == "force":
                f = np.zeros(3, np.float32)
                lib.aero_lbm_get_last_force(key, f[0:].ctypes.data, f[1:].ctypes.data, f[2:].ctypes.data)
                results.append(f)
            elif kind == "point":
                fl = np.zeros(4, np.float32)
                t = np.zeros(1, np.float32)
                if not (lib.aero_lbm_sample_flow_point_rect(nx, ny, nz, key, *act[1:4], fl.ctypes.data) and
                        lib.aero_lbm_sample_temperature_point_rect(nx, ny, nz, key, *act[1:4], t.ctypes.data)):
                    raise RuntimeError("point sample failed")
                results.append((fl, t))
            elif kind == "subrect":
                n = int(np.prod(act[4:7]))
                fl = np.zeros(n * 4, np.float32)
                t = np.zeros(n, np.float32)
                if not lib.aero_lbm_copy_flow_temperature_subrect(nx, ny, nz, key, *act[1:7], fl.ctypes.data, t.ctypes.data):
                    raise RuntimeError("subrect copy failed")
                results.append((fl.reshape(-1, 4), t))
            else:
                raise ValueError(kind)
        return results


def fan_thermal_source(pk: np.ndarray) -> np.ndarray:
    """thermal_source_term without a source channel (native/src/aero_lbm_jni.cpp:
    1783-1797): mask * clamp(|fan velocity| * 0.0012, 0, 0.006), in float32."""
    m = np.minimum(np.float32(1), np.maximum(np.float32(0), pk[:, 1].astype(np.float32)))
    m = np.where(np.isnan(pk[:, 1]), np.float32(0), m)
    f = [np.where(np.isfinite(pk[:, c]), pk[:, c], 0).astype(np.float32) for c in (2, 3, 4)]
    n = np.sqrt((f[0] * f[0] + f[1] * f[1]) + f[2] * f[2]).astype(np.float32)
    capped = np.minimum(np.float32(0.006), np.maximum(np.float32(0), (n * np.float32(0.0012)).astype(np.float32)))
    return np.where((m > 0) & (n > np.float32(1e-8)), (m * capped).astype(np.float32), np.float32(0)).astype(np.float32)


def short_packet_script(packet: np.ndarray, seed: int = 5):
    """Steps of a 9/10-channel packet, two of them with sparse overlays on
    fan cells and other fluid cells (non-zero source values), reading the
    flow and the temperature state in between."""
    rng = np.random.default_rng(seed)
    pk = np.asarray(packet, np.float32)
    fans = np.nonzero((pk[:, 1] > 0) & (pk[:, 0] <= 0.5))[0]
    fluid = np.nonzero(pk[:, 0] <= 0.5)[0]
    cells = np.concatenate([fans[:12], rng.choice(fluid, 12, replace=False)]).astype(np.int32)
    k = cells.size
    vals = np.stack([rng.uniform(-0.05, 0.05, k), rng.uniform(-0.05, 0.05, k), rng.uniform(-0.05, 0.05, k),
                     rng.uniform(-0.01, 0.01, k), rng.uniform(-0.5, 0.5, k), rng.uniform(-0.01, 0.01, k)],
                    axis=1).astype(np.float32)
    ov = (cells, np.ascontiguousarray(vals))
    # overlays on even calls: runtime mode transports the temperature on those
    return [("step",)] * 4 + [("flow",), ("temp",)] + [("step", ov), ("step",), ("step", ov), ("step",)] + \
        [("flow",), ("temp",)]


def run_script_oracle(o: "Oracle", cfg: dict, packet: np.ndarray, script):
    """The same call list on the oracle. Actions: ("step", overlays|None) with
    overlays = (cells int32, values float32 x 6); ("cached",) a step with the
    resident inputs; ("patch", cells, solid) block edits; ("shell", flow
    cells x 4, face_mask, layers, relaxation); ("flow",) write_output of
    the streamed state; ("temp",) temperature state; ("shift", dx, dy, dz);
    ("force",) last_force; ("point", x, y, z) -> (flow 4, [T]); ("subrect",
    ox, oy, oz, cx, cy, cz) -> (flow cells x 4, T with solids 0, clamped)."""
    n = o.dims
    pk = np.asarray(packet, np.float32)
    obst = pk[:, 0] > 0.5
    transport = bool(derive_params(cfg).thermal_transport)
    results = []
    for act in script:
        kind = act[0]
        if kind == "step":
            o.set_fields(obst.reshape(n).astype(np.uint8), *(pk[:, 5 + a].reshape(n) for a in range(3)),
                         pressure=pk[:, 8].reshape(n),
                         temperature=pk[:, 10].reshape(n) if pk.shape[1] > 10 else None)
            if transport:
                if not cfg.get("thermal_source", False):
                    src = np.zeros(pk.shape[0], np.float32)
                elif pk.shape[1] > 9:
                    src = pk[:, 9]
                else:
                    src = fan_thermal_source(pk)
                o.set_thermal_source(src)
            if cfg.get("fans", False):
                o.set_fans(pk[:, 1], pk[:, 2], pk[:, 3], pk[:, 4])
            ov = act[1] if len(act) > 1 else None
            if ov is not None:
                o.apply_overlays(ov[0], ov[1])
            o.step(1)
        elif kind == "cached":
            o.step(1)
        elif kind == "patch":
            o.patch_cells(act[1], act[2])
        elif kind == "shell":
            o.set_shell(act[1], act[2], act[3], act[4])
        elif kind == "mode":
            # the realtime solver mode of the product's later calls; the shell
            # restatement above models calls in the FP16 in-place mode (3),
            # the only mode whose step reads the shell (jni.cpp:6779-6790)
            pass
        elif kind == "flow":
            results.append(o.output())
        elif kind == "temp":
            results.append(o.temperature())
        elif kind == "shift":
            if not o.shift(*act[1:4]):
                raise RuntimeError("oracle shift failed")
        elif kind == "force":
            results.append(o.last_force())
        elif kind == "point":
            x, y, z = act[1:4]
            cell = (x * n[1] + y) * n[2] + z
            results.append((o.output()[cell].copy(), o.temperature()[cell:cell + 1].copy()))
        elif kind == "subrect":
            ox, oy, oz, cx, cy, cz = act[1:7]
            flow = o.output().reshape(n + (4,))[ox:ox + cx, oy:oy + cy, oz:oz + cz].reshape(-1, 4)
            t = o.temperature().reshape(n)[ox:ox + cx, oy:oy + cy, oz:oz + cz].reshape(-1)
            solid = o.mask().reshape(n)[ox:ox + cx, oy:oy + cy, oz:oz + cz].reshape(-1) != 0
            t = np.where(solid, np.float32(0), np.nan_to_num(np.clip(t, -1, 1), nan=0.0, posinf=0.0, neginf=0.0))
            results.append((flow.copy(), t.astype(np.float32)))
        else:
            raise ValueError(kind)
    return results


def context_ops_script(n: int, seed: int = 23):
    """A call list over the per-context entry points around the step: four
    steps, a read of flow and temperature, a shift, point and sub-box reads,
    steps with sparse overlays (40 cells plus two out-of-range indices), a
    second shift, a step and the last force."""
    rng = np.random.default_rng(seed)
    cells = np.concatenate([rng.choice(n ** 3, 40, replace=False), [-1, n ** 3 + 5]]).astype(np.int32)
    k = cells.size
    vals = np.stack([rng.uniform(-0.05, 0.05, k), rng.uniform(-0.05, 0.05, k), rng.uniform(-0.05, 0.05, k),
                     rng.uniform(-0.05, 0.05, k), rng.uniform(-1.5, 1.5, k), rng.uniform(-0.01, 0.01, k)],
                    1).astype(np.float32)
    ov = (cells, vals)
    return ([("step",)] * 4 + [("flow",), ("temp",), ("shift", 1, -2, 0), ("flow",), ("temp",), ("point", 3, 4, 5),
            ("subrect", 2, 3, 1, 5, 4, 6), ("step",), ("step", ov), ("step", ov), ("flow",), ("temp",),
            ("shift", -3, 0, 2), ("step",), ("flow",), ("temp",), ("point", 0, 0, 0), ("force",)])


CYLINDER_SCRIPT = [("step",), ("force",)] * 5 + [("flow",)]
FAN_SCRIPT = [("step",)] * 6 + [("flow",), ("temp",)] + [("step",)] * 6 + [("flow",)]
RUNTIME_SCRIPT = ([("step",)] + [("flow",), ("temp",)] + [("step",)] * 2 + [("flow",), ("temp",)] + [("step",)] * 5
                  + [("flow",), ("temp",)])


def feq_rest(q: int) -> float:
    """Rest equilibrium weight of direction q (q = (ix*3+iy)*3+iz)."""
    w1 = (1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0)
    return float(np.float32(np.float32(np.float32(w1[q // 9]) * np.float32(w1[(q // 3) % 3])) * np.float32(w1[q % 3])))


def load_results(path) -> list:
    """The recorded results of a script fixture (r<i> or the pair r<i>_0, r<i>_1)."""
    g = np.load(path)
    out = []
    for i in range(int(g["count"])):
        out.append((g[f"r{i}_0"], g[f"r{i}_1"]) if f"r{i}_0" in g.files else g[f"r{i}"])
    return out


def results_equal(a, b) -> list:
    """Per result: bit-identical (float32 views compared as integers)?"""
    flags = []
    for x, y in zip(a, b):
        if isinstance(x, tuple):
            flags.append(all(np.array_equal(np.asarray(p, np.float32).view(np.uint32),
                                            np.asarray(q, np.float32).view(np.uint32)) for p, q in zip(x, y)))
        else:
            flags.append(np.array_equal(np.asarray(x, np.float32).view(np.uint32), np.asarray(y, np.float32).view(np.uint32)))
    return flags


def edits_script(n: int, seed: int = 43):
    """Block edits and the boundary shell between steps: patches that close
    fluid cells, open solid ones, reset fluid cells (duplicates and an
    out-of-range index included), cached steps, a shell on three faces, a
    second round of patches, the shell cleared."""
    rng = np.random.default_rng(seed)

    def patches(k):
        cells = np.concatenate([rng.choice(n ** 3, k, replace=False), [n ** 3 + 7]]).astype(np.int32)
        cells = np.concatenate([cells, cells[:3]])
        solid = (rng.random(cells.size) < 0.4).astype(np.uint8)
        return cells, solid

    flow = np.zeros((n ** 3, 4), np.float32)
    flow[:, 0] = 0.02 + rng.uniform(-0.005, 0.005, n ** 3)
    flow[:, 1] = 0.01
    flow[:, 2] = rng.uniform(-0.01, 0.01, n ** 3)
    flow[:, 3] = 0.001
    p1, p2, p3 = patches(30), patches(20), patches(25)
    return ([("step",)] * 3 + [("patch",) + p1, ("cached",), ("cached",), ("flow",), ("temp",),
                               ("shell", flow, 0b010011, 3, 0.3), ("step",), ("step",), ("flow",),
                               ("patch",) + p2, ("patch",) + p3, ("cached",), ("flow",), ("temp",),
                               ("shell", flow, 0, 3, 0.3), ("step",), ("flow",), ("temp",)])


def fan_case(n: int = 12, seed: int = 61, noise: bool = True, sponge: bool = True):
    """The thermal case with the fan forcing, fan noise and sponge of the
    reference's collide switched on (their DISABLE flags cleared): 3 % of the
    fluid cells carry a fan (mask U(0.3, 1), direction and speed up to 3 m/s,
    so the target exceeds the soft cap in places)."""
    obst, u, temp, src, cfg, pre = thermal_case(n, seed)
    rng = np.random.default_rng(seed + 1)
    dims = (n, n, n)
    fan = (rng.random(dims) < 0.03) & (obst == 0)
    mask = np.where(fan, rng.uniform(0.3, 1.0, dims), 0.0).astype(np.float32)
    fv = [np.where(fan, rng.uniform(-3.0, 3.0, dims), 0.0).astype(np.float32) for _ in range(3)]
    cfg = dict(cfg, fans=True, fan_noise=noise, sponge=sponge)
    pk = packet_from(obst, *u, temperature=temp, source=src, fans=(mask, *fv))
    return cfg, pk, pre


def runtime_case(n: int = 12, seed: int = 71, fans: bool = True, channels: int = 11):
    """Benchmark mode off (the reference's game runtime, as its brick service
    runs it): the thermal case's brick and fields with fans on 3 % of the
    fluid cells; the faces are the default config's (convective outflow)."""
    cfg, pk, pre = fan_case(n, seed)
    if not fans:
        pk = pk.copy()
        pk[:, 1:5] = 0.0
    cfg = {"benchmark": False, "faces": cfg["faces"], "fans": True, "thermal_transport": True,
           "thermal_source": True, "packet_channels": channels}
    return cfg, np.ascontiguousarray(pk[:, :channels]), pre


def cylinder_case(nx: int = 44, ny: int = 20, nz: int = 3, sgs: bool = True):
    """The 2-D cylinder crossflow preset (native/src/aero_lbm_jni.cpp:341-…,
    geometry 201-227) as a configuration: inflow 0.12 at x-, convective
    outflow at x+, walls y, periodic z, Re 100, u0 = (0.08, 0, 0); the packet
    marks the disc of cylinder_benchmark_solid_cell solid. Returns the config
    and the packet."""
    length_cells = np.float32(max(1, nx - 1))
    channel_height = np.float32(max(1, ny - 1))
    diameter = max(np.float32(2.5), np.float32(np.float32(0.1) / np.float32(2.2)) * length_cells)
    diameter = min(diameter, max(np.float32(2.5), np.float32(channel_height - np.float32(4.0))))
    radius = np.float32(np.float32(0.5) * diameter)
    cxf = np.float32(np.float32(np.float32(0.2) / np.float32(2.2)) * length_cells)
    cyf = np.float32(np.float32(0.0) + np.float32(np.float32(0.2) / np.float32(0.41)) * channel_height)
    xs = np.arange(nx, dtype=np.float32)[:, None] - cxf
    ys = np.arange(ny, dtype=np.float32)[None, :] - cyf
    disc = (xs * xs + ys * ys) <= radius * radius
    obst = np.repeat(disc[:, :, None], nz, axis=2).astype(np.uint8)
    u = (np.where(obst == 0, np.float32(0.08), np.float32(0)).astype(np.float32), np.zeros(obst.shape, np.float32),
         np.zeros(obst.shape, np.float32))
    faces = [{"kind": VELOCITY, "velocity": (0.12, 0, 0)}, {"kind": CONVECTIVE},
             {"kind": BOUNCE_BACK}, {"kind": BOUNCE_BACK},
             {"kind": PERIODIC, "thermal": THERMAL_PERIODIC}, {"kind": PERIODIC, "thermal": THERMAL_PERIODIC}]
    cfg = {"preset": PRESET_CYLINDER_2D, "reynolds": 100.0, "initial_velocity": (0.08, 0.0, 0.0), "faces": faces,
           "sgs": sgs, "buoyancy": False, "thermal_source": False}
    return cfg, packet_from(obst, *u)


# ---------------------------------------------------------------- the reference's brick service
SIM_REF_LIB = REF_LIB.parent / "libaero_sim_ref.so"
SIM_B200_LIB = REF_LIB.parent / "libaero_sim_b200.so"


class BrickService:
    """The reference's brick-world service (its simulation bridge, built by
    `make -C oracle sim`), driven through its C ABI. ``libaero_sim_ref.so``
    runs it over the reference's CPU step; ``libaero_sim_b200.so`` is the same
    service source linked against libaero_lbm_b200.so."""

    def __init__(self, path: Path):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} missing (build with `make -C oracle sim`)")
        lib = ctypes.CDLL(str(path))
        vp, i, ll, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_float
        for name, args in (
                ("aero_lbm_simulation_create_service", [vp]),
                ("aero_lbm_simulation_ensure_brick_world_runtime", [ll, ll, i, f, f]),
                ("aero_lbm_simulation_set_brick_world_solver_mode", [ll, ll, i]),
                ("aero_lbm_simulation_set_brick_world_exact_active_hints", [ll, ll, i, vp, i]),
                ("aero_lbm_simulation_upload_brick_world_static_brick_with_sources",
                 [ll, ll, i, i, i, i, vp, vp, vp, vp, vp, vp, vp, vp]),
                ("aero_lbm_simulation_upload_brick_world_dynamic_brick", [ll, ll, i, i, i, i, vp, vp, vp]),
                ("aero_lbm_simulation_step_brick_world_runtime", [ll, ll, i]),
                ("aero_lbm_simulation_copy_brick_world_packed_flow_atlas", [ll, ll, i, i, i, i, i, vp, i]),
                ("aero_lbm_simulation_copy_brick_world_dynamic_brick", [ll, ll, i, i, i, i, vp, vp, vp]),
                ("aero_lbm_simulation_get_brick_world_runtime_status", [ll, ll, vp, i])):
            getattr(lib, name).argtypes = args
            getattr(lib, name).restype = ctypes.c_int
        lib.aero_lbm_simulation_release_service.argtypes = [ll]
        lib.aero_lbm_simulation_last_error.restype = ctypes.c_char_p
        self.lib = lib

    def _ok(self, v):
        if not v:
            raise RuntimeError(self.lib.aero_lbm_simulation_last_error())

    def run(self, world: dict) -> dict:
        """world: n, bricks [(bx, by, bz)], solver_mode, steps, dx, dt, and per
        brick the static obstacle (n^3 u8) and dynamic flow (n^3 x 4), air and
        surface temperature. Returns per brick the stride-4 packed atlas and
        the dynamic brick after ``steps`` ticks, and the runtime status."""
        lib, n = self.lib, int(world["n"])
        key = ctypes.c_longlong(0)
        self._ok(lib.aero_lbm_simulation_create_service(ctypes.byref(key)))
        svc, wk = key.value, 1
        try:
            self._ok(lib.aero_lbm_simulation_ensure_brick_world_runtime(svc, wk, n, world["dx"], world["dt"]))
            self._ok(lib.aero_lbm_simulation_set_brick_world_solver_mode(svc, wk, int(world["solver_mode"])))
            coords = np.ascontiguousarray(np.array(world["bricks"], np.int32).reshape(-1))
            self._ok(lib.aero_lbm_simulation_set_brick_world_exact_active_hints(svc, wk, n, coords.ctypes.data,
                                                                                len(world["bricks"])))
            cells = n ** 3
            zeros_u8 = np.zeros(cells, np.uint8)
            zeros_u16 = np.zeros(cells, np.uint16)
            zeros_f = np.zeros(cells, np.float32)
            faces = np.zeros(cells * 6, np.uint8)
            keep = []
            for b, (bx, by, bz) in enumerate(world["bricks"]):
                ob = np.ascontiguousarray(world["obstacle"][b], np.uint8)
                self._ok(lib.aero_lbm_simulation_upload_brick_world_static_brick_with_sources(
                    svc, wk, n, bx, by, bz, ob.ctypes.data, zeros_u8.ctypes.data, zeros_u16.ctypes.data,
                    zeros_f.ctypes.data, None, None, faces.ctypes.data, faces.ctypes.data))
                fl = np.ascontiguousarray(world["flow"][b], np.float32)
                at = np.ascontiguousarray(world["air_t"][b], np.float32)
                st = np.ascontiguousarray(world["surface_t"][b], np.float32)
                keep += [ob, fl, at, st]
                self._ok(lib.aero_lbm_simulation_upload_brick_world_dynamic_brick(
                    svc, wk, n, bx, by, bz, fl.ctypes.data, at.ctypes.data, st.ctypes.data))
            self._ok(lib.aero_lbm_simulation_step_brick_world_runtime(svc, wk, int(world["steps"])))
            out = {"atlas": [], "flow": [], "air_t": []}
            s = (n + 3) // 4
            for bx, by, bz in world["bricks"]:
                atlas = np.zeros(s ** 3 * 4, np.int16)
                self._ok(lib.aero_lbm_simulation_copy_brick_world_packed_flow_atlas(svc, wk, n, bx, by, bz, 4,
                                                                                    atlas.ctypes.data, atlas.size))
                fl = np.zeros(cells * 4, np.float32)
                at = np.zeros(cells, np.float32)
                st = np.zeros(cells, np.float32)
                self._ok(lib.aero_lbm_simulation_copy_brick_world_dynamic_brick(svc, wk, n, bx, by, bz, fl.ctypes.data,
                                                                                at.ctypes.data, st.ctypes.data))
                out["atlas"].append(atlas)
                out["flow"].append(fl.reshape(-1, 4))
                out["air_t"].append(at)
            status = np.zeros(8, np.int32)
            lib.aero_lbm_simulation_get_brick_world_runtime_status(svc, wk, status.ctypes.data, 8)
            out["status"] = status
            return out
        finally:
            lib.aero_lbm_simulation_release_service(svc)


class WorldDelta(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("type", "x", "y", "z", "data0", "data1", "data2", "data3")] + \
               [(n, ctypes.c_float) for n in ("value0", "value1", "value2", "value3")]


def run_brick_script(path: Path, script: list) -> list:
    """Run a list of brick-world service operations through the C ABI of the
    library at ``path`` (the reference's service, or any library exporting
    aero_lbm_simulation_*) and return what the reading operations returned, in
    order. Operations (tuples): ("ensure", world, n, dx, dt), ("mode", world,
    m), ("hints", world, n, coords, exact), ("static", world, n, coord,
    obstacle, surface_kind, open_faces, emitter, source_fan|None,
    source_emitter|None), ("queue_static", world, n, coord, obstacle,
    surface_kind, open_faces, emitter), ("dynamic" | "reference", world, n,
    coord, flow, air, surface), ("deltas", [12-tuples]), ("step", world,
    count), ("atlas", world, n, coord, stride), ("copy", world, n, coord),
    ("status", world), ("coords", world, resident). Every operation's return
    code is recorded too, so failures must match as well."""
    lib = ctypes.CDLL(str(path))
    vp, i, ll, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_float
    sig = {
        "aero_lbm_simulation_create_service": [vp],
        "aero_lbm_simulation_ensure_brick_world_runtime": [ll, ll, i, f, f],
        "aero_lbm_simulation_set_brick_world_solver_mode": [ll, ll, i],
        "aero_lbm_simulation_set_brick_world_active_hints": [ll, ll, i, vp, i],
        "aero_lbm_simulation_set_brick_world_exact_active_hints": [ll, ll, i, vp, i],
        "aero_lbm_simulation_upload_brick_world_static_brick_with_sources": [ll, ll, i, i, i, i] + [vp] * 8,
        "aero_lbm_simulation_queue_brick_world_static_brick_upload": [ll, ll, i, i, i, i] + [vp] * 6,
        "aero_lbm_simulation_upload_brick_world_dynamic_brick": [ll, ll, i, i, i, i, vp, vp, vp],
        "aero_lbm_simulation_upload_brick_world_boundary_reference_brick": [ll, ll, i, i, i, i, vp, vp, vp],
        "aero_lbm_simulation_submit_world_deltas": [ll, vp, i],
        "aero_lbm_simulation_step_brick_world_runtime": [ll, ll, i],
        "aero_lbm_simulation_copy_brick_world_packed_flow_atlas": [ll, ll, i, i, i, i, i, vp, i],
        "aero_lbm_simulation_copy_brick_world_dynamic_brick": [ll, ll, i, i, i, i, vp, vp, vp],
        "aero_lbm_simulation_get_brick_world_runtime_status": [ll, ll, vp, i],
        "aero_lbm_simulation_get_brick_world_resident_brick_count": [ll, ll],
        "aero_lbm_simulation_get_brick_world_active_brick_count": [ll, ll],
        "aero_lbm_simulation_copy_brick_world_resident_bricks": [ll, ll, vp, i],
        "aero_lbm_simulation_copy_brick_world_active_bricks": [ll, ll, vp, i],
    }
    for name, args in sig.items():
        getattr(lib, name).argtypes = args
        getattr(lib, name).restype = ctypes.c_int
    lib.aero_lbm_simulation_release_service.argtypes = [ll]
    lib.aero_lbm_simulation_last_error.restype = ctypes.c_char_p
    key = ctypes.c_longlong(0)
    assert lib.aero_lbm_simulation_create_service(ctypes.byref(key)) == 1
    svc = key.value
    keep, out = [], []

    def arr(a, dt):
        a = np.ascontiguousarray(np.asarray(a, dt).reshape(-1))
        keep.append(a)
        return a.ctypes.data

    try:
        for op in script:
            kind = op[0]
            if kind == "ensure":
                out.append(("rc", lib.aero_lbm_simulation_ensure_brick_world_runtime(svc, *op[1:])))
            elif kind == "mode":
                out.append(("rc", lib.aero_lbm_simulation_set_brick_world_solver_mode(svc, op[1], op[2])))
            elif kind == "hints":
                _, w, n, coords, exact = op
                fn = lib.aero_lbm_simulation_set_brick_world_exact_active_hints if exact else \
                    lib.aero_lbm_simulation_set_brick_world_active_hints
                out.append(("rc", fn(svc, w, n, arr(coords, np.int32), len(coords))))
            elif kind in ("static", "queue_static"):
                w, n, c = op[1], op[2], op[3]
                cells = n ** 3
                faces = arr(np.zeros(cells * 6, np.uint8), np.uint8)
                ob, sk, of, em = arr(op[4], np.uint8), arr(op[5], np.uint8), arr(op[6], np.uint16), arr(op[7], np.float32)
                if kind == "static":
                    sf = None if op[8] is None else arr(op[8], np.uint8)
                    se = None if op[9] is None else arr(op[9], np.float32)
                    out.append(("rc", lib.aero_lbm_simulation_upload_brick_world_static_brick_with_sources(
                        svc, w, n, *c, ob, sk, of, em, sf, se, faces, faces)))
                else:
                    out.append(("rc", lib.aero_lbm_simulation_queue_brick_world_static_brick_upload(
                        svc, w, n, *c, ob, sk, of, em, faces, faces)))
            elif kind in ("dynamic", "reference"):
                w, n, c, fl, air, sf = op[1:]
                fn = lib.aero_lbm_simulation_upload_brick_world_dynamic_brick if kind == "dynamic" else \
                    lib.aero_lbm_simulation_upload_brick_world_boundary_reference_brick
                out.append(("rc", fn(svc, w, n, *c, arr(fl, np.float32), arr(air, np.float32), arr(sf, np.float32))))
            elif kind == "deltas":
                ds = (WorldDelta * len(op[1]))(*[WorldDelta(*d) for d in op[1]])
                keep.append(ds)
                out.append(("rc", lib.aero_lbm_simulation_submit_world_deltas(svc, ctypes.addressof(ds), len(op[1]))))
            elif kind == "step":
                rc = lib.aero_lbm_simulation_step_brick_world_runtime(svc, op[1], op[2])
                out.append(("step", rc, b"" if rc else lib.aero_lbm_simulation_last_error()))
            elif kind == "atlas":
                w, n, c, stride = op[1:]
                res = (n + stride - 1) // stride
                a = np.zeros(res ** 3 * 4, np.int16)
                rc = lib.aero_lbm_simulation_copy_brick_world_packed_flow_atlas(svc, w, n, *c, stride, a.ctypes.data, a.size)
                out.append(("atlas", rc, a))
            elif kind == "copy":
                w, n, c = op[1:]
                cells = n ** 3
                fl, air, sf = np.zeros(cells * 4, np.float32), np.zeros(cells, np.float32), np.zeros(cells, np.float32)
                rc = lib.aero_lbm_simulation_copy_brick_world_dynamic_brick(svc, w, n, *c, fl.ctypes.data, air.ctypes.data,
                                                                            sf.ctypes.data)
                out.append(("copy", rc, fl, air, sf))
            elif kind == "status":
                st = np.zeros(8, np.int32)
                rc = lib.aero_lbm_simulation_get_brick_world_runtime_status(svc, op[1], st.ctypes.data, 8)
                out.append(("status", rc, st))
            elif kind == "coords":
                w, resident = op[1], op[2]
                cnt = (lib.aero_lbm_simulation_get_brick_world_resident_brick_count if resident else
                       lib.aero_lbm_simulation_get_brick_world_active_brick_count)(svc, w)
                buf = np.zeros(max(cnt, 0) * 3, np.int32)
                got = (lib.aero_lbm_simulation_copy_brick_world_resident_bricks if resident else
                       lib.aero_lbm_simulation_copy_brick_world_active_bricks)(svc, w, buf.ctypes.data, max(cnt, 0))
                rows = sorted(map(tuple, buf.reshape(-1, 3).tolist()))
                out.append(("coords", cnt, got, rows))
            else:
                raise ValueError(kind)
    finally:
        lib.aero_lbm_simulation_release_service(svc)
    return out


def brick_world_rich_script(n: int = 12, seed: int = 57) -> list:
    """A brick-world session exercising the service's bookkeeping around the
    step: an L-shaped set of bricks (one not hinted), dynamic uploads for some
    bricks only (the others seed from their neighbours' means or from a
    boundary reference), fan surface kinds and heat emitters in the static
    fields, source fields rebuilt into fan footprints and plumes, a boundary
    reference, world deltas (a cell patch and a source patch), a queued static
    upload and a mid-run dynamic upload; reads after each phase."""
    rng = np.random.default_rng(seed)
    cells = n ** 3
    W = 1
    bricks = [(0, 0, 0), (1, 0, 0), (2, 0, 0), (0, 0, 1), (1, 0, 1), (0, 1, 0)]
    hinted = bricks[:5]

    def obstacle():
        ob = (rng.random((n, n, n)) < 0.05).astype(np.uint8)
        ob[:, 0, :] = 1
        return ob.reshape(-1)

    def flow(scale=1.0):
        fl = np.zeros((cells, 4), np.float32)
        fl[:, 0] = scale * (0.05 + rng.uniform(-0.01, 0.01, cells))
        fl[:, 1] = scale * rng.uniform(-0.005, 0.005, cells)
        fl[:, 2] = scale * (0.02 + rng.uniform(-0.01, 0.01, cells))
        fl[:, 3] = rng.uniform(-0.002, 0.002, cells)
        return fl

    def temps():
        return rng.uniform(-0.05, 0.05, cells).astype(np.float32), rng.uniform(0, 0.02, cells).astype(np.float32)

    s = [("ensure", W, n, 1.0, 0.05), ("mode", W, 1), ("hints", W, n, hinted, True), ("status", W)]
    zeros_u8 = np.zeros(cells, np.uint8)
    zeros_u16 = np.zeros(cells, np.uint16)
    zeros_f = np.zeros(cells, np.float32)
    for b in bricks:
        ob = obstacle()
        sk, of, em, sf, se = zeros_u8.copy(), zeros_u16.copy(), zeros_f.copy(), None, None
        if b == (0, 0, 0):
            sk.reshape(n, n, n)[2:4, 3:6, 3:6] = 33  # fans blowing +x
        if b == (1, 0, 0):
            em.reshape(n, n, n)[5:7, 2, 5:7] = 400.0
            of.reshape(n, n, n)[:, 1, :] = 2
        if b == (0, 0, 1):
            sf = zeros_u8.copy()
            sf.reshape(n, n, n)[4, 3, 4] = 2  # a fan block pointing +x
            se = zeros_f.copy()
            se.reshape(n, n, n)[7, 2, 7] = 600.0
        s.append(("static", W, n, b, ob, sk, of, em, sf, se))
    for b in [(0, 0, 0), (1, 0, 0), (0, 0, 1)]:
        air, surf = temps()
        s.append(("dynamic", W, n, b, flow(), air, surf))
    air, surf = temps()
    s.append(("reference", W, n, (2, 0, 0), flow(0.8), air, surf))
    reads = lambda: [("status", W), ("coords", W, True), ("coords", W, False)] + \
        [("atlas", W, n, b, 4) for b in hinted] + [("copy", W, n, b) for b in hinted]
    s += [("step", W, 3)] + reads()
    # world deltas: a cell patch that solidifies a fluid cell of (1,0,0), a
    # source patch placing a fan block in (0,0,0), a queued static upload
    wx, wy, wz = 1 * n + 6, 5, 6
    s.append(("deltas", [(8, wx, wy, wz, W, 0x1, 0, 0, 0.0, 0.0, 0.0, 0.0),
                         (10, 3, 6, 4, W, 0x0 | (0 << 8) | (2 << 16), 0, 0, 0.0, 0.0, 0.0, 0.0)]))
    ob = obstacle()
    s.append(("queue_static", W, n, (1, 0, 1), ob, zeros_u8, zeros_u16, zeros_f))
    s += [("step", W, 3)] + reads()
    air, surf = temps()
    s.append(("dynamic", W, n, (0, 0, 0), flow(1.2), air, surf))
    s += [("step", W, 2)] + reads() + [("atlas", W, n, (1, 0, 0), 3)]
    return s


def brick_world_case(n: int = 16, steps: int = 6, seed: int = 51, solver_mode: int = 1):
    """Four face-adjacent bricks (2 x 2 in x-z) of n^3 cells: a solid ground
    layer in the lower bricks plus 5 % random solids, a seeded flow of about
    0.05 (lattice units), small air temperature deviations."""
    rng = np.random.default_rng(seed)
    bricks = [(0, 0, 0), (1, 0, 0), (0, 0, 1), (1, 0, 1)]
    cells = n ** 3
    obstacle, flow, air_t, surface_t = [], [], [], []
    for _ in bricks:
        ob = (rng.random((n, n, n)) < 0.05).astype(np.uint8)
        ob[:, 0, :] = 1
        obstacle.append(ob.reshape(-1))
        fl = np.zeros((cells, 4), np.float32)
        fl[:, 0] = 0.05 + rng.uniform(-0.01, 0.01, cells)
        fl[:, 1] = rng.uniform(-0.005, 0.005, cells)
        fl[:, 2] = 0.02 + rng.uniform(-0.01, 0.01, cells)
        fl[ob.reshape(-1) != 0] = 0.0
        flow.append(fl)
        air_t.append(rng.uniform(-0.05, 0.05, cells).astype(np.float32))
        surface_t.append(np.zeros(cells, np.float32))
    return {"n": n, "bricks": bricks, "solver_mode": solver_mode, "steps": steps, "dx": 1.0, "dt": 0.05,
            "obstacle": obstacle, "flow": flow, "air_t": air_t, "surface_t": surface_t}


# ---------------------------------------------------------------- configs
def c1_inputs(seed: int = 1234, n: int = 32, solid_p: float = 0.05, u0=(0.05, 0.0, 0.0), noise: float = 0.005):
    """Plain FP32 brick (32^3): solid floor z=0 + Bernoulli(p) interior,
    u = u0 + U(-noise, noise) per component, rho = 1."""
    rng = np.random.default_rng(seed)
    obstacle = (rng.random((n, n, n)) < solid_p).astype(np.uint8)
    obstacle[:, :, 0] = 1
    u = [np.float32(u0[a]) + rng.uniform(-noise, noise, size=(n, n, n)).astype(np.float32) for a in range(3)]
    return obstacle, u


def c1_config(tau: float = 0.55, u0: float = 0.05, sgs: bool = True) -> dict:
    nu = (tau - 0.5) / 3.0
    return {
        "reynolds": u0 / nu,
        "reference_length": 1.0,
        "initial_velocity": (u0, 0.0, 0.0),
        "faces": [{"kind": PERIODIC}, {"kind": PERIODIC}, {"kind": PERIODIC}, {"kind": PERIODIC},
                  {"kind": BOUNCE_BACK}, {"kind": BOUNCE_BACK}],
        "sgs": sgs,
        "buoyancy": False,
    }


def packet_from(obstacle, ux, uy, uz, pressure=None, temperature=None, channels: int = 11, source=None,
                fans=None) -> np.ndarray:
    cells = obstacle.size
    pk = np.zeros((cells, channels), dtype=np.float32)
    pk[:, 0] = (obstacle.reshape(-1) != 0)
    pk[:, 5] = np.asarray(ux, np.float32).reshape(-1)
    pk[:, 6] = np.asarray(uy, np.float32).reshape(-1)
    pk[:, 7] = np.asarray(uz, np.float32).reshape(-1)
    if pressure is not None:
        pk[:, 8] = np.asarray(pressure, np.float32).reshape(-1)
    if temperature is not None and channels > 10:
        pk[:, 10] = np.asarray(temperature, np.float32).reshape(-1)
    if source is not None and channels > 9:
        pk[:, 9] = np.asarray(source, np.float32).reshape(-1)
    if fans is not None:  # (mask, vx, vy, vz): channels 1-4
        for c, v in enumerate(fans):
            pk[:, 1 + c] = np.asarray(v, np.float32).reshape(-1)
    return pk


def thermal_case(n: int = 12, seed: int = 11):
    """Buoyancy with the reference's temperature transport on an n^3 brick:
    8% random solids, u = (0.04,0,0) + U(-0.01,0.01), packet temperature
    U(-0.3,0.3) and source U(-0.01,0.01), every thermal face kind (Dirichlet
    0.2 / -0.4, Neumann 0.05, periodic y, adiabatic ground), initial
    temperature 0.1, temperature state preloaded with 0.5 (so that fluid cells
    start from the packet's temperature). Returns obstacle, (ux, uy, uz),
    temperature, source, the config dict and the preload."""
    rng = np.random.default_rng(seed)
    dims = (n, n, n)
    obst = (rng.random(dims) < 0.08).astype(np.uint8)
    u = (np.float32(0.04) + rng.uniform(-0.01, 0.01, dims).astype(np.float32),
         rng.uniform(-0.01, 0.01, dims).astype(np.float32), rng.uniform(-0.01, 0.01, dims).astype(np.float32))
    temp = rng.uniform(-0.3, 0.3, dims).astype(np.float32)
    src = rng.uniform(-0.01, 0.01, dims).astype(np.float32)
    faces = [{"kind": VELOCITY, "velocity": (0.04, 0, 0), "thermal": THERMAL_DIRICHLET, "temperature": 0.2},
             {"kind": PRESSURE, "pressure": 0.001, "thermal": THERMAL_NEUMANN, "heat_flux": 0.05},
             {"kind": PERIODIC, "thermal": THERMAL_PERIODIC}, {"kind": PERIODIC, "thermal": THERMAL_PERIODIC},
             {"kind": BOUNCE_BACK, "thermal": THERMAL_ADIABATIC},
             {"kind": MOVING_WALL, "velocity": (0.03, 0, 0), "thermal": THERMAL_DIRICHLET, "temperature": -0.4}]
    cfg = {"reynolds": 60.0, "initial_velocity": (0.04, 0.0, 0.0), "faces": faces, "sgs": True, "buoyancy": True,
           "thermal_transport": True, "initial_temperature": 0.1, "thermal_source": True}
    preload = np.full(n ** 3, 0.5, np.float32)
    return obst, u, temp, src, cfg, preload


def halo_case(n: int = 12, buoyancy: bool = True):
    """Two bricks for the halo exchange: thermal_case(n, 11) (source off) and
    a second brick with 8% solids (seed 5), u = (0.03,0,0) + U(-0.01,0.01),
    temperature U(-0.3,0.3). Returns the config, both packets and the
    temperature state both start from."""
    obst, u, temp, src, cfg, pre = thermal_case(n, 11)
    cfg = dict(cfg, thermal_source=False, buoyancy=buoyancy)
    rng = np.random.default_rng(5)
    dims = (n, n, n)
    obst2 = (rng.random(dims) < 0.08).astype(np.uint8)
    u2 = [np.float32(0.03) + rng.uniform(-0.01, 0.01, dims).astype(np.float32) for _ in range(3)]
    temp2 = rng.uniform(-0.3, 0.3, dims).astype(np.float32)
    return cfg, [packet_from(obst, *u, temperature=temp), packet_from(obst2, *u2, temperature=temp2)], pre


def heated_cavity_case(n: int = 12, seed: int = 3, preset: int = PRESET_HEATED_CAVITY_3D):
    """The reference's differentially heated cavity preset (Ra 1e5, Pr 0.71,
    Mach 0.15; hot x- face 0.5, cold x+ face -0.5, bounce-back walls; 2-D:
    periodic z) on an n^3 brick with 4% random solids, u = U(-0.01, 0.01),
    packet temperature U(-0.2, 0.2), state preloaded with 0.3; the 3-D case
    makes z- a Neumann face (flux 0.02). Its temperature transport is the
    BFECC branch. Returns obstacle, (ux, uy, uz), temperature, config, preload."""
    rng = np.random.default_rng(seed)
    dims = (n, n, n)
    obst = (rng.random(dims) < 0.04).astype(np.uint8)
    u = tuple(rng.uniform(-0.01, 0.01, dims).astype(np.float32) for _ in range(3))
    temp = rng.uniform(-0.2, 0.2, dims).astype(np.float32)
    faces = [{"kind": BOUNCE_BACK, "thermal": THERMAL_DIRICHLET, "temperature": 0.5},
             {"kind": BOUNCE_BACK, "thermal": THERMAL_DIRICHLET, "temperature": -0.5},
             {"kind": BOUNCE_BACK, "thermal": THERMAL_ADIABATIC}, {"kind": BOUNCE_BACK, "thermal": THERMAL_ADIABATIC}]
    if preset == PRESET_HEATED_CAVITY_2D:
        faces += [{"kind": PERIODIC, "thermal": THERMAL_PERIODIC}] * 2
    else:
        faces += [{"kind": BOUNCE_BACK, "thermal": THERMAL_NEUMANN, "heat_flux": 0.02},
                  {"kind": BOUNCE_BACK, "thermal": THERMAL_ADIABATIC}]
    cfg = {"preset": preset, "rayleigh": 1e5, "prandtl": 0.71, "mach": 0.15, "faces": faces, "sgs": True,
           "buoyancy": True, "thermal_transport": True, "initial_temperature": 0.0}
    return obst, u, temp, cfg, np.full(n ** 3, 0.3, np.float32)


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """max |a - b| / max |b| (normwise max-relative error)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b))) / (den if den > 0 else 1.0)


def flow_errors(out: np.ndarray, ref: np.ndarray) -> dict:
    """Parity metric on write_output-style arrays (cells x 4: ux, uy, uz, rho-1).

    u   : max over cells and components |u - u_ref| / max cell speed of ref
    rho : max |rho - rho_ref| / max rho_ref, with rho = 1 + channel 3
    (velocity error relative to the flow speed scale and density error relative
    to the density; the pressure proxy rho - 1 is ~1e-3, so its own relative
    error would only measure FP32 rounding of rho ~ 1)."""
    out = np.asarray(out, np.float64)
    ref = np.asarray(ref, np.float64)
    speed = float(np.max(np.linalg.norm(ref[:, :3], axis=1)))
    u = float(np.max(np.abs(out[:, :3] - ref[:, :3]))) / (speed if speed > 0 else 1.0)
    rho = float(np.max(np.abs(out[:, 3] - ref[:, 3]))) / float(np.max(1.0 + ref[:, 3]))
    return {"u": u, "rho": rho}


# ---------------------------------------------------------------- D3Q19 mesoscale
MESO_CHANNELS = 25
MESO_OUT = 6


class MesoConfig(ctypes.Structure):
    """AeroLbmMesoscaleConfig (native/include/aero_lbm_capi.h:124-140)."""
    _fields_ = [
        ("abi_version", ctypes.c_uint32), ("struct_size", ctypes.c_uint32),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx_m", ctypes.c_float), ("dt_s", ctypes.c_float), ("molecular_nu_m2_s", ctypes.c_float),
        ("prandtl_air", ctypes.c_float), ("turbulent_prandtl", ctypes.c_float),
        ("reference_density_kg_m3", ctypes.c_float), ("ambient_air_temperature_k", ctypes.c_float),
        ("deep_ground_temperature_k", ctypes.c_float), ("background_wind_m_s", ctypes.c_float * 3),
        ("reserved", ctypes.c_uint32 * 8),
    ]


class MesoTransport(ctypes.Structure):
    _fields_ = [("velocity_scale", ctypes.c_double), ("tau_shear", ctypes.c_double), ("tau_thermal", ctypes.c_double)]


class MesoOptions(ctypes.Structure):
    _fields_ = [
        ("periodic_sides", ctypes.c_int), ("free_slip_top", ctypes.c_int), ("fixed_tau", ctypes.c_int),
        ("enable_sgs", ctypes.c_int), ("disable_edge_blend", ctypes.c_int), ("hydro_only", ctypes.c_int),
        ("tau_hydro", ctypes.c_double), ("smagorinsky_c", ctypes.c_double), ("body_force", ctypes.c_double * 3),
    ]


def meso_transport(dx: float, dt: float, nu: float, pr: float) -> MesoTransport:
    """derive_transport in float32 (mesoscale.cpp:45-68, hydro_core.h:109-115,
    thermal_core.cpp:5-15)."""
    dx, dt, nu, pr = f32(dx), f32(dt), f32(nu), f32(pr)
    t = MesoTransport()
    t.velocity_scale = float(dx / dt)
    nu_lat = f32(nu * dt) / f32(dx * dx)
    t.tau_shear = float(f32(0.5) + f32(3.0) * nu_lat)
    alpha = f32(nu / pr)
    alpha_lat = f32(alpha * dt) / f32(dx * dx)
    t.tau_thermal = float(f32(0.5) + alpha_lat / f32(0.25))
    return t


class MesoOracle:
    """Restated D3Q19 mesoscale step; precision 'f32' or 'f64'."""

    def __init__(self, dims, dx=64.0, dt=5.0, nu=1.5e-5, pr=0.71, precision="f32", options: MesoOptions | None = None):
        lib = Oracle.lib()
        lib.oracle_d3q19_create.restype = ctypes.c_void_p
        lib.oracle_d3q19_create.argtypes = [ctypes.c_int] * 4 + [ctypes.POINTER(MesoTransport), ctypes.POINTER(MesoOptions), ctypes.c_double]
        lib.oracle_d3q19_step.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_d3q19_destroy.argtypes = [ctypes.c_void_p]
        self.lib = lib
        self.dims = tuple(int(d) for d in dims)
        self.cells = int(np.prod(self.dims))
        tr = meso_transport(dx, dt, nu, pr)
        self.h = lib.oracle_d3q19_create(*self.dims, 0 if precision == "f32" else 1, ctypes.byref(tr),
                                         ctypes.byref(options) if options else None, float(np.float32(dt)))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oracle_d3q19_destroy(self.h)
            self.h = None

    def step(self, forcing: np.ndarray) -> np.ndarray:
        fo = np.ascontiguousarray(forcing, np.float32)
        out = np.zeros(self.cells * MESO_OUT, np.float32)
        if not self.lib.oracle_d3q19_step(self.h, fo.ctypes.data, out.ctypes.data):
            raise RuntimeError("oracle d3q19 step failed")
        return out.reshape(self.cells, MESO_OUT)


def meso_ref_run(dims, forcing: np.ndarray, steps: int, dx=64.0, dt=5.0, nu=1.5e-5, pr=0.71, path: Path = REF_LIB):
    """The reference library's aero_lbm_mesoscale_step_context, `steps` calls."""
    lib = ctypes.CDLL(str(path))
    lib.aero_lbm_mesoscale_default_config.argtypes = [ctypes.POINTER(MesoConfig)]
    lib.aero_lbm_mesoscale_create_context.argtypes = [ctypes.POINTER(MesoConfig), ctypes.POINTER(ctypes.c_longlong)]
    lib.aero_lbm_mesoscale_create_context.restype = ctypes.c_int
    lib.aero_lbm_mesoscale_step_context.argtypes = [ctypes.c_longlong, ctypes.POINTER(MesoConfig), ctypes.c_void_p, ctypes.c_void_p]
    lib.aero_lbm_mesoscale_step_context.restype = ctypes.c_int
    lib.aero_lbm_mesoscale_release_context.argtypes = [ctypes.c_longlong]
    cfg = MesoConfig()
    lib.aero_lbm_mesoscale_default_config(ctypes.byref(cfg))
    cfg.nx, cfg.ny, cfg.nz = dims
    cfg.dx_m, cfg.dt_s, cfg.molecular_nu_m2_s, cfg.prandtl_air = dx, dt, nu, pr
    key = ctypes.c_longlong(0)
    if not lib.aero_lbm_mesoscale_create_context(ctypes.byref(cfg), ctypes.byref(key)):
        raise RuntimeError("mesoscale create failed")
    fo = np.ascontiguousarray(forcing, np.float32)
    out = np.zeros(int(np.prod(dims)) * MESO_OUT, np.float32)
    for _ in range(steps):
        if not lib.aero_lbm_mesoscale_step_context(key.value, ctypes.byref(cfg), fo.ctypes.data, out.ctypes.data):
            raise RuntimeError("mesoscale step failed")
    lib.aero_lbm_mesoscale_release_context(key.value)
    return out.reshape(-1, MESO_OUT)


def meso_forcing(dims, seed: int = 0, terrain_max: float = 3.0, wind=(6.0, 0.0, 3.0)) -> np.ndarray:
    """Seeded 25-channel forcing: heightmap terrain (cells below it solid, the
    mesoscale grid is y-up), temperatures, roughness, humidity, background wind."""
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    F = np.zeros((nx, ny, nz, MESO_CHANNELS), np.float32)
    h = rng.uniform(0.0, terrain_max, (nx, nz)).astype(np.float32)
    y = np.arange(ny)[None, :, None]
    F[..., 0] = h[:, None, :]
    F[..., 1] = 288.0
    F[..., 2] = 288.15 + rng.uniform(-2, 2, (nx, ny, nz))
    F[..., 3] = 289.65
    F[..., 4] = 290.0 + rng.uniform(-3, 3, (nx, 1, nz))
    F[..., 5] = rng.uniform(0.0, 2.0, (nx, 1, nz))
    F[..., 6] = wind[0]
    F[..., 7] = wind[2]
    F[..., 9] = rng.uniform(0.2, 0.8, (nx, ny, nz))
    F[..., 19] = wind[1]
    F[..., 24] = (y < np.floor(h)[:, None, :]).astype(np.float32)
    return F.reshape(-1, MESO_CHANNELS)
