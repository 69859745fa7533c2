"""The per-cell reverse sweep of the cumulant collision against central finite
differences of the forward collision, both in FP64 on the host CPU (no GPU):
the vector-Jacobian product lam_out^T J must match the directional
derivatives to 1e-6 relative, with SGS, buoyancy, body force, the speed clamp
and the clamped relaxation rates exercised."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import aero_b200


@pytest.fixture(scope="module")
def lib():
    return aero_b200.load_library()


def cfg(lib, **kw):
    c = aero_b200.AeroLbmB200AdjointConfig()
    lib.aero_lbm_b200_adjoint_default_config(ctypes.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


W1 = np.array([1 / 6, 2 / 3, 1 / 6])
C = np.array([[ix - 1, iy - 1, iz - 1] for ix in range(3) for iy in range(3) for iz in range(3)], float)
W = np.array([W1[ix] * W1[iy] * W1[iz] for ix in range(3) for iy in range(3) for iz in range(3)])


def feq(rho, u):
    cu = 3 * C @ u
    return W * rho * (1 + cu + 0.5 * cu * cu - 1.5 * u @ u)


def call(lib, c, f, temp, force, lam, precision=1):
    f = np.ascontiguousarray(f, np.float64)
    force = np.ascontiguousarray(force, np.float64)
    lam = np.ascontiguousarray(lam, np.float64)
    fo, li, lf = np.zeros(27), np.zeros(27), np.zeros(3)
    assert lib.aero_lbm_b200_adjoint_collide_vjp_host(precision, ctypes.byref(c), aero_b200._dptr(f), float(temp),
                                                      aero_b200._dptr(force), aero_b200._dptr(lam), aero_b200._dptr(fo),
                                                      aero_b200._dptr(li), aero_b200._dptr(lf)) == 1
    return fo, li, lf


def check(lib, c, f, temp, force, seed):
    rng = np.random.default_rng(seed)
    lam = rng.normal(size=27)
    _, li, lf = call(lib, c, f, temp, force, lam)
    for trial in range(6):
        v = rng.normal(size=27) * 1e-3
        g = rng.normal(size=3) * 1e-6
        h = 1e-4
        fp, _, _ = call(lib, c, f + h * v, temp, force + h * g, lam)
        fm, _, _ = call(lib, c, f - h * v, temp, force - h * g, lam)
        fd = lam @ (fp - fm) / (2 * h)
        ad = li @ v + lf @ g
        assert abs(fd - ad) <= 1e-6 * max(abs(fd), 1e-9) + 1e-14, (trial, fd, ad)


@pytest.mark.parametrize("u", [(0.05, 0.01, 0.0), (0.0, -0.08, 0.03), (0.3, 0.2, -0.1)])
@pytest.mark.parametrize("sgs", [0.0, 0.1])
def test_vjp_matches_finite_differences(lib, u, sgs):
    rng = np.random.default_rng(3)
    u = np.array(u)
    f = feq(1.01, u) * (1 + rng.uniform(-0.02, 0.02, 27))  # off-equilibrium populations
    c = cfg(lib, tau=0.56, smagorinsky_c=sgs, buoyancy_beta=1e-4)
    check(lib, c, f, 0.7, np.array([2e-5, -1e-5, 3e-6]), seed=11)


def test_vjp_speed_clamp_branch(lib):
    """|u| above the clamp (0.3464): the clamp's projection enters the adjoint."""
    f = feq(1.0, np.array([0.33, 0.12, 0.05]))
    c = cfg(lib, tau=0.6, smagorinsky_c=0.1, buoyancy_beta=0.0)
    fo, _, _ = call(lib, c, f, 0.0, np.zeros(3), np.zeros(27))
    assert np.isfinite(fo).all()
    check(lib, c, f, 0.0, np.array([1e-5, 0.0, 0.0]), seed=5)


def test_vjp_float_close_to_double(lib):
    rng = np.random.default_rng(8)
    f = feq(0.99, np.array([0.04, 0.02, -0.01])) * (1 + rng.uniform(-0.01, 0.01, 27))
    lam = rng.normal(size=27)
    c = cfg(lib, tau=0.55, smagorinsky_c=0.1, buoyancy_beta=1e-4)
    fo64, li64, lf64 = call(lib, c, f, 0.3, np.array([1e-5, 0, 0]), lam, precision=1)
    fo32, li32, lf32 = call(lib, c, f, 0.3, np.array([1e-5, 0, 0]), lam, precision=0)
    assert np.max(np.abs(fo32 - fo64)) < 1e-6
    assert np.max(np.abs(li32 - li64)) < 1e-4 * np.max(np.abs(li64))
    assert np.max(np.abs(lf32 - lf64)) < 1e-4 * np.max(np.abs(lf64))


def test_collision_conserves_mass_and_momentum(lib):
    """The forward collision conserves rho and, without force, rho u."""
    rng = np.random.default_rng(2)
    f = feq(1.0, np.array([0.05, -0.02, 0.01])) * (1 + rng.uniform(-0.02, 0.02, 27))
    c = cfg(lib, tau=0.58, smagorinsky_c=0.1, buoyancy_beta=0.0)
    fo, _, _ = call(lib, c, f, 0.0, np.zeros(3), np.zeros(27))
    assert abs(fo.sum() - f.sum()) < 1e-13
    assert np.max(np.abs(C.T @ fo - C.T @ f)) < 1e-13
