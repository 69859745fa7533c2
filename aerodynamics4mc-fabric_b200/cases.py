"""Seeded synthetic inputs for the benchmark configurations of the brick step.

Each builder returns plain numpy arrays (obstacle mask, initial velocity,
temperature) plus the boundary/physics settings, in the packet conventions of
the C ABI (cell = (x*ny + y)*nz + z, z up). Nothing here runs on the GPU.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

PERIODIC, BOUNCE_BACK, MOVING_WALL, VELOCITY, PRESSURE, CONVECTIVE, SYMMETRY = 1, 2, 3, 4, 5, 6, 7


@dataclass
class BrickCase:
    name: str
    dims: tuple
    obstacle: np.ndarray            # uint8 (nx, ny, nz)
    u: tuple                        # three float32 arrays (nx, ny, nz)
    temperature: np.ndarray | None  # float32 (nx, ny, nz) or None
    faces: list                     # 6 dicts: kind, velocity, pressure
    tau: float
    u_ref: tuple
    sgs: bool = True
    smagorinsky_c: float = 0.025
    buoyancy: bool = False
    buoyancy_beta: float = 0.0
    gravity_axis: int = 2
    steps: int = 1000
    extra: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return int(np.prod(self.dims))

    def config_dict(self) -> dict:
        """Dict form understood by the parity tooling (Reynolds number chosen so
        that the effective shear tau equals ``tau``)."""
        speed = float(np.linalg.norm(np.asarray(self.u_ref, np.float64)))
        for fc in self.faces:
            speed = max(speed, float(np.linalg.norm(np.asarray(fc.get("velocity", (0, 0, 0)), np.float64))))
        nu = (self.tau - 0.5) / 3.0
        return {
            "reynolds": speed / nu,
            "reference_length": 1.0,
            "initial_velocity": tuple(float(v) for v in self.u_ref),
            "faces": self.faces,
            "sgs": self.sgs,
            "buoyancy": self.buoyancy,
            "smagorinsky_c": self.smagorinsky_c,
            "buoyancy_beta": self.buoyancy_beta,
            "gravity_axis": self.gravity_axis,
        }

    def temperature_state(self) -> np.ndarray | None:
        """Temperature state to load (aero_lbm_set_temperature_state_rect)
        before the first step. With the temperature transport, the first call
        keeps a non-zero state's fluid cells at the packet's temperature
        (otherwise every cell starts at the configured initial temperature),
        so loading the case's field makes the run start from it."""
        if self.temperature is None:
            return None
        return np.ascontiguousarray(self.temperature.reshape(-1), dtype=np.float32)

    def packet(self, channels: int = 11) -> np.ndarray:
        pk = np.zeros((self.cells, channels), dtype=np.float32)
        pk[:, 0] = (self.obstacle.reshape(-1) != 0)
        for a in range(3):
            pk[:, 5 + a] = self.u[a].reshape(-1)
        if self.temperature is not None and channels > 10:
            pk[:, 10] = self.temperature.reshape(-1)
        return pk


def value_noise_heightmap(n_x: int, n_y: int, octaves: int, amplitude: float, seed: int) -> np.ndarray:
    """Fractal value noise: octave k is a (4*2^k + 1)^2 random lattice
    bilinearly interpolated to the grid, weight 2^-k; rescaled to [0, amplitude]."""
    rng = np.random.default_rng(seed)
    h = np.zeros((n_x, n_y), np.float64)
    for k in range(octaves):
        m = 4 * 2 ** k + 1
        lat = rng.random((m, m))
        gx = np.linspace(0, m - 1, n_x)
        gy = np.linspace(0, m - 1, n_y)
        ix = np.minimum(gx.astype(int), m - 2)
        iy = np.minimum(gy.astype(int), m - 2)
        fx = (gx - ix)[:, None]
        fy = (gy - iy)[None, :]
        a = lat[ix][:, iy]
        b = lat[ix + 1][:, iy]
        c = lat[ix][:, iy + 1]
        d = lat[ix + 1][:, iy + 1]
        h += 0.5 ** k * ((1 - fx) * (1 - fy) * a + fx * (1 - fy) * b + (1 - fx) * fy * c + fx * fy * d)
    h -= h.min()
    if h.max() > 0:
        h *= amplitude / h.max()
    return h


def c1_plain_fp32(n: int = 32, seed: int = 1234, tau: float = 0.55, steps: int = 1000) -> BrickCase:
    """One n^3 brick, periodic x/y, bounce-back floor z=0 (solid plane and
    face), Bernoulli(0.05) interior solids, u = (0.05,0,0) + U(-0.005,0.005)."""
    rng = np.random.default_rng(seed)
    obstacle = (rng.random((n, n, n)) < 0.05).astype(np.uint8)
    obstacle[:, :, 0] = 1
    u0 = (0.05, 0.0, 0.0)
    u = tuple(np.float32(u0[a]) + rng.uniform(-0.005, 0.005, size=(n, n, n)).astype(np.float32) for a in range(3))
    faces = [{"kind": PERIODIC}] * 4 + [{"kind": BOUNCE_BACK}] * 2
    return BrickCase("c1-plain-fp32", (n, n, n), obstacle, u, None, faces, tau, u0, sgs=True, steps=steps)


def c2_terrain_boussinesq(n: int = 128, seed: int = 2024, tau: float = 0.55, steps: int = 1000) -> BrickCase:
    """One n^3 brick over a seeded 4-octave heightmap (amplitude 24 cells at
    n=128, scaled with n), inflow u=(0.08,0.02,0) at x=0 (velocity face),
    convective outflow at x=n-1, a far-field equilibrium lid at the inflow
    velocity, periodic y, bounce-back ground. Boussinesq along +z with
    g*beta = 1e-4 and T = -1e-3 z plus a Gaussian warm bubble (amplitude
    0.01, radius 8, centre (n/2, n/2, 20))."""
    s = n / 128.0
    h = value_noise_heightmap(n, n, 4, 24.0 * s, seed)
    z = np.arange(n)[None, None, :]
    obstacle = (z < h[:, :, None]).astype(np.uint8)
    obstacle[:, :, 0] = 1
    u_in = (0.08, 0.02, 0.0)
    fluid = obstacle == 0
    u = tuple(np.where(fluid, np.float32(u_in[a]), np.float32(0)).astype(np.float32) for a in range(3))
    g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1).astype(np.float64)
    centre = np.array([n / 2, n / 2, 20.0 * s])
    r2 = np.sum((g - centre) ** 2, -1)
    temp = (-1e-3 * g[..., 2] + 0.01 * np.exp(-r2 / (2 * (8.0 * s) ** 2))).astype(np.float32)
    far = {"kind": VELOCITY, "velocity": u_in}
    faces = [far, {"kind": CONVECTIVE}, {"kind": PERIODIC}, {"kind": PERIODIC}, {"kind": BOUNCE_BACK}, far]
    return BrickCase("c2-terrain-boussinesq", (n, n, n), obstacle, u, temp, faces, tau, u_in, sgs=True,
                     smagorinsky_c=0.1, buoyancy=True, buoyancy_beta=1e-4, gravity_axis=2, steps=steps)


MESO_CHANNELS = 25


@dataclass
class MesoCase:
    """A D3Q19 mesoscale grid (y up, cell = (x*ny + y)*nz + z): the 25-channel
    forcing of aero_lbm_mesoscale_step_context plus the step options."""
    name: str
    dims: tuple                     # (nx, ny, nz), ny vertical
    forcing: np.ndarray             # float32 (cells, 25)
    dx_m: float
    dt_s: float
    options: dict                   # periodic_sides, free_slip_top, fixed_tau, tau_hydro, enable_sgs,
                                    # smagorinsky_c, body_force, hydro_only, disable_edge_blend
    steps: int = 2000

    @property
    def cells(self) -> int:
        return int(np.prod(self.dims))

    @property
    def velocity_scale(self) -> float:
        return float(np.float32(self.dx_m) / np.float32(self.dt_s))


def c3_meso_terrain(nx: int = 256, nz: int = 256, ny: int = 64, seed: int = 77, steps: int = 2000,
                    dx_m: float = 64.0, dt_s: float = 5.0) -> MesoCase:
    """Mesoscale boundary layer: seeded smooth terrain (3-octave value noise up
    to 12 cells at ny=64, scaled with ny) as the bounce-back ground, a free-slip
    lid, periodic sides, a body force (1e-6, 0, 0), tau 0.52 with Smagorinsky
    (C = 0.1), initial u_x(y) = 0.06 ln(1+y) / ln(ny+1) (as the background
    wind channel, which seeds the state). The hydrodynamic distribution runs
    alone (no thermal distribution, no target relaxation)."""
    h = value_noise_heightmap(nx, nz, 3, 12.0 * ny / 64.0, seed)
    y = np.arange(ny, dtype=np.float64)[None, :, None]
    F = np.zeros((nx, ny, nz, MESO_CHANNELS), np.float32)
    solid = (y < h[:, None, :])
    vs = float(np.float32(dx_m) / np.float32(dt_s))
    ux = 0.06 * np.log1p(y) / np.log(ny + 1.0)
    F[..., 0] = h[:, None, :]
    F[..., 2] = 288.15
    F[..., 3] = 289.65
    F[..., 4] = 290.0
    F[..., 6] = np.broadcast_to(ux * vs, (nx, ny, nz))
    F[..., 24] = solid.astype(np.float32)
    opts = {"periodic_sides": 1, "free_slip_top": 1, "fixed_tau": 1, "tau_hydro": 0.52, "enable_sgs": 1,
            "smagorinsky_c": 0.1, "body_force": (1e-6, 0.0, 0.0), "hydro_only": 1, "disable_edge_blend": 1}
    return MesoCase("c3-meso-terrain", (nx, ny, nz), F.reshape(-1, MESO_CHANNELS), dx_m, dt_s, opts, steps)


@dataclass
class AdjointCase:
    """Inverse problem on one brick: probes, their targets from a hidden run,
    and the point (force field, inflow) the gradient is taken at."""
    name: str
    dims: tuple
    obstacle: np.ndarray          # uint8 (nx, ny, nz)
    temperature: np.ndarray       # float32 (nx, ny, nz)
    config: dict                  # AeroLbmB200AdjointConfig fields
    force_true: np.ndarray        # float32 (3, nx, ny, nz), the hidden run's body force
    inflow_true: tuple
    probes: np.ndarray            # int32 cell indices
    force0: np.ndarray            # gradient point
    inflow0: tuple


def smooth_force_field(dims, amplitude: float, sigma: float, seed: int) -> np.ndarray:
    """3 x dims Gaussian-filtered (periodic) white noise, each component scaled
    to a maximum magnitude of `amplitude`."""
    from scipy.ndimage import gaussian_filter

    rng = np.random.default_rng(seed)
    out = np.zeros((3,) + tuple(dims), np.float32)
    for a in range(3):
        g = gaussian_filter(rng.normal(size=dims), sigma, mode="wrap")
        out[a] = (amplitude * g / np.max(np.abs(g))).astype(np.float32)
    return out


def c5_adjoint(n: int = 64, steps: int = 200, checkpoint_every: int = 20, seed: int = 55, nprobe: int = 64) -> AdjointCase:
    """n^3 brick with SGS (C = 0.1), Boussinesq (g*beta = 1e-4, temperature
    -1e-3 z plus a warm bubble), a seeded 5% obstacle mask, inflow faces at x-,
    x+ and z+ (equilibrium at the inflow vector), periodic y, bounce-back
    ground; hidden body force: smooth random field (amplitude 1e-5, Gaussian
    sigma 6 at n = 64) with inflow (0.05, 0.01, 0); 64 interior fluid probes.
    The gradient is taken at half the hidden force and a perturbed inflow."""
    rng = np.random.default_rng(seed)
    obstacle = (rng.random((n, n, n)) < 0.05).astype(np.uint8)
    s = n / 64.0
    g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1).astype(np.float64)
    centre = np.array([n / 2, n / 2, 16.0 * s])
    temp = (-1e-3 * g[..., 2] + 0.01 * np.exp(-np.sum((g - centre) ** 2, -1) / (2 * (6.0 * s) ** 2))).astype(np.float32)
    force = smooth_force_field((n, n, n), 1e-5, 6.0 * s, seed + 1)
    lo, hi = max(2, n // 8), n - max(2, n // 8)
    cand = [(x, y, z) for x, y, z in rng.integers(lo, hi, (nprobe * 4, 3)) if obstacle[x, y, z] == 0]
    cells = sorted({(x * n + y) * n + z for x, y, z in cand})
    probes = np.array(rng.permutation(cells)[:nprobe], np.int32)
    config = {"face_kind": (4, 4, 1, 1, 2, 4), "tau": 0.55, "smagorinsky_c": 0.1, "buoyancy_beta": 1e-4,
              "steps": steps, "checkpoint_every": checkpoint_every}
    return AdjointCase("c5-adjoint", (n, n, n), obstacle, temp, config, force, (0.05, 0.01, 0.0), probes,
                       (0.5 * force).astype(np.float32), (0.045, 0.012, 0.002))
