"""Host-side checks of the D3Q19 mesoscale ABI (no GPU needed): default
config, transport derivation (bit-equal to the reference library when it is
built here), context keys and option validation."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import aero_b200
import oracle as O


@pytest.fixture(scope="module")
def lib():
    return aero_b200.load_library()


def cfg_of(lib, **kw):
    c = aero_b200.AeroLbmMesoscaleConfig()
    lib.aero_lbm_mesoscale_default_config(ctypes.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def test_default_config(lib):
    c = cfg_of(lib)
    assert (c.abi_version, c.struct_size) == (3, ctypes.sizeof(aero_b200.AeroLbmMesoscaleConfig))
    assert (c.nx, c.ny, c.nz) == (32, 4, 32)
    assert (c.dx_m, c.dt_s) == (64.0, 5.0)
    assert np.float32(c.molecular_nu_m2_s) == np.float32(1.5e-5)


@pytest.mark.parametrize("dx,dt,nu,pr", [(64.0, 5.0, 1.5e-5, 0.71), (8.0, 0.25, 1.5e-5, 0.71), (1.0, 1.0, 0.02, 0.9)])
def test_derive_transport(lib, dx, dt, nu, pr):
    c = cfg_of(lib, dx_m=dx, dt_s=dt, molecular_nu_m2_s=nu, prandtl_air=pr)
    t = aero_b200.AeroLbmMesoscaleTransport()
    assert lib.aero_lbm_mesoscale_derive_transport(ctypes.byref(c), ctypes.byref(t)) == 1
    want = O.meso_transport(dx, dt, nu, pr)
    assert np.float32(t.velocity_scale_m_s_per_lattice) == np.float32(want.velocity_scale)
    assert np.float32(t.tau_shear_molecular) == np.float32(want.tau_shear)
    assert np.float32(t.tau_thermal_molecular) == np.float32(want.tau_thermal)
    if O.REF_LIB.exists():
        ref = ctypes.CDLL(str(O.REF_LIB))
        rc = O.MesoConfig()
        ref.aero_lbm_mesoscale_default_config(ctypes.byref(rc))
        rc.dx_m, rc.dt_s, rc.molecular_nu_m2_s, rc.prandtl_air = dx, dt, nu, pr
        rt = aero_b200.AeroLbmMesoscaleTransport()
        assert ref.aero_lbm_mesoscale_derive_transport(ctypes.byref(rc), ctypes.byref(rt)) == 1
        assert bytes(rt) == bytes(t)


def test_invalid_config_rejected(lib):
    t = aero_b200.AeroLbmMesoscaleTransport()
    key = ctypes.c_longlong(0)
    for bad in ({"abi_version": 2}, {"nx": 0}, {"dt_s": 0.0}, {"prandtl_air": float("nan")}, {"struct_size": 8}):
        c = cfg_of(lib, **bad)
        assert lib.aero_lbm_mesoscale_derive_transport(ctypes.byref(c), ctypes.byref(t)) == 0
        assert lib.aero_lbm_mesoscale_create_context(ctypes.byref(c), ctypes.byref(key)) == 0


def test_keys_and_options(lib):
    c = cfg_of(lib)
    k1, k2 = ctypes.c_longlong(0), ctypes.c_longlong(0)
    assert lib.aero_lbm_mesoscale_create_context(ctypes.byref(c), ctypes.byref(k1)) == 1
    assert lib.aero_lbm_mesoscale_create_context(ctypes.byref(c), ctypes.byref(k2)) == 1
    assert k2.value == k1.value + 1
    o = aero_b200.AeroLbmB200MesoscaleOptions()
    lib.aero_lbm_b200_mesoscale_default_options(ctypes.byref(o))
    assert lib.aero_lbm_b200_mesoscale_set_options(k1.value, ctypes.byref(o)) == 1
    o.storage = 1  # FP16 without hydro_only
    assert lib.aero_lbm_b200_mesoscale_set_options(k1.value, ctypes.byref(o)) == 0
    assert "hydro_only" in aero_b200.last_error(lib)
    o.hydro_only, o.threads = 1, 96
    assert lib.aero_lbm_b200_mesoscale_set_options(k1.value, ctypes.byref(o)) == 0
    o.threads, o.fixed_tau, o.tau_hydro = 128, 1, 0.5
    assert lib.aero_lbm_b200_mesoscale_set_options(k1.value, ctypes.byref(o)) == 0
    o.tau_hydro = 0.52
    assert lib.aero_lbm_b200_mesoscale_set_options(k1.value, ctypes.byref(o)) == 1
    assert lib.aero_lbm_b200_mesoscale_set_options(987654, ctypes.byref(o)) == 0
    assert lib.aero_lbm_b200_mesoscale_advance(k1.value, 1) == 0  # never stepped
    lib.aero_lbm_mesoscale_release_context(k1.value)
    lib.aero_lbm_mesoscale_release_context(k2.value)
    lib.aero_lbm_mesoscale_release_context(k2.value)  # unknown key: no-op
