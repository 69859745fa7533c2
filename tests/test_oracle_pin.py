"""Pin the oracle: its float restatement must reproduce the reference CPU step
bit-for-bit (against the committed golden fixtures made by the reference
library, and live against oracle/_ref when that library is present)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import oracle as O
import lbm_cases

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module", autouse=True)
def _build_oracle():
    O.build(ref=False)


def _bits_equal(a, b) -> bool:
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def test_oracle_f32_matches_golden_c1_16():
    g = np.load(GOLDEN / "c1_16_200.npz")
    n, steps = int(g["n"]), int(g["steps"])
    obst, u = O.c1_inputs(seed=int(g["seed"]), n=n)
    o = O.Oracle((n, n, n), O.derive_params(O.c1_config()), "f32")
    o.set_fields(obst, *u)
    o.step(steps)
    assert _bits_equal(o.output(), g["out"])


def test_oracle_f32_matches_golden_tunnel():
    g = np.load(GOLDEN / "tunnel_16_60.npz")
    obst, u, cfg = lbm_cases.tunnel_case(16)
    assert np.array_equal(obst, g["obstacle"])
    o = O.Oracle((16, 16, 16), O.derive_params(cfg), "f32")
    o.set_fields(obst, *u)
    o.step(int(g["steps"]))
    assert _bits_equal(o.output(), g["out"])


@pytest.mark.skipif(not O.REF_LIB.exists(), reason="reference library not built here")
@pytest.mark.parametrize("faces", [
    "pressure_outlet", "closed", "periodic_all", "inherit_game", "inherit_bounce",
])
def test_oracle_f32_matches_reference_live(faces):
    n = 12
    rng = np.random.default_rng(7)
    obst = (rng.random((n, n, n)) < 0.08).astype(np.uint8)
    u = [np.float32(0.04) + rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32),
         rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32),
         rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32)]
    p = rng.uniform(-0.01, 0.01, (n, n, n)).astype(np.float32)
    table = {
        "pressure_outlet": [{"kind": O.VELOCITY, "velocity": (0.04, 0.0, 0.0)}, {"kind": O.PRESSURE, "pressure": 0.002}]
                           + [{"kind": O.SYMMETRY}] * 4,
        "closed": [{"kind": O.BOUNCE_BACK}] * 5 + [{"kind": O.MOVING_WALL, "velocity": (0.05, 0.0, 0.0)}],
        "periodic_all": [{"kind": O.PERIODIC}] * 6,
        "inherit_game": [{"kind": O.INHERIT_GAME}] * 6,
        "inherit_bounce": [{"kind": O.INHERIT_GAME}] * 6,
    }
    cfg = {"reynolds": 60.0, "initial_velocity": (0.04, 0.0, 0.0), "faces": table[faces], "sgs": True,
           "buoyancy": False, "disable_convective": faces == "inherit_bounce"}
    pk = O.packet_from(obst, *u, pressure=p)
    ref = O.RefLib().run((n, n, n), cfg, pk, 25)
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    o.set_fields(obst, *u, pressure=p)
    o.step(25)
    assert _bits_equal(o.output(), ref)


def test_oracle_f64_is_the_same_scheme():
    """The FP64 run differs from FP32 only by rounding over a short horizon."""
    n = 12
    obst, u = O.c1_inputs(seed=3, n=n)
    p = O.derive_params(O.c1_config())
    a = O.Oracle((n, n, n), p, "f32")
    b = O.Oracle((n, n, n), p, "f64")
    for o in (a, b):
        o.set_fields(obst, *u)
        o.step(50)
    assert O.rel_err(a.macro()[:, 1:], b.macro()[:, 1:]) < 1e-5


def _thermal_oracle(n, seed, steps, precision="f32"):
    obst, u, temp, src, cfg, preload = O.thermal_case(n, seed)
    o = O.Oracle((n, n, n), O.derive_params(cfg), precision)
    o.set_temperature(preload)
    o.set_fields(obst, *u, temperature=temp)
    o.set_thermal_source(src)
    o.step(steps)
    return o


def test_oracle_thermal_transport_matches_golden():
    """Buoyancy driven by the reference's benchmark-mode temperature transport
    (advection by the previous collision's velocity, diffusion, packet source,
    Dirichlet / Neumann / periodic / adiabatic thermal faces): flow output and
    temperature state bit-identical to the reference library's fixture."""
    g = np.load(GOLDEN / "thermal_12_20.npz")
    o = _thermal_oracle(int(g["n"]), int(g["seed"]), int(g["steps"]))
    assert _bits_equal(o.output(), g["out"])
    assert _bits_equal(o.temperature(), g["temperature"])


@pytest.mark.skipif(not O.REF_LIB.exists(), reason="reference library not built here")
@pytest.mark.parametrize("preload,source", [(False, False), (True, True)])
def test_oracle_thermal_transport_matches_reference_live(preload, source):
    n, steps = 10, 15
    obst, u, temp, src, cfg, pre = O.thermal_case(n, seed=23)
    cfg = dict(cfg, thermal_source=source)
    pk = O.packet_from(obst, *u, temperature=temp, source=src)
    ref = O.RefLib()
    out = ref.run((n, n, n), cfg, pk, steps, temperature_state=pre if preload else None)
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    if preload:
        o.set_temperature(pre)
    o.set_fields(obst, *u, temperature=temp)
    o.set_thermal_source(src)
    o.step(steps)
    assert _bits_equal(o.output(), out)
    assert _bits_equal(o.temperature(), ref.temperature)


def test_oracle_bfecc_transport_matches_golden():
    """Heated-cavity preset: its BFECC temperature transport (forward and
    backward advection, error correction, local limiter, diffusion) and the
    preset's derived Rayleigh/Prandtl/Mach parameters, bit-identical to the
    reference library's fixture."""
    g = np.load(GOLDEN / "cavity_12_25.npz")
    n = int(g["n"])
    obst, u, temp, cfg, preload = O.heated_cavity_case(n, int(g["seed"]))
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    o.set_temperature(preload)
    o.set_fields(obst, *u, temperature=temp)
    o.step(int(g["steps"]))
    assert _bits_equal(o.output(), g["out"])
    assert _bits_equal(o.temperature(), g["temperature"])


@pytest.mark.skipif(not O.REF_LIB.exists(), reason="reference library not built here")
@pytest.mark.parametrize("preset", [O.PRESET_HEATED_CAVITY_2D, O.PRESET_HEATED_CAVITY_3D])
def test_oracle_bfecc_transport_matches_reference_live(preset):
    n, steps = 10, 15
    obst, u, temp, cfg, pre = O.heated_cavity_case(n, seed=9, preset=preset)
    pk = O.packet_from(obst, *u, temperature=temp)
    ref = O.RefLib()
    out = ref.run((n, n, n), cfg, pk, steps, temperature_state=pre)
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    o.set_temperature(pre)
    o.set_fields(obst, *u, temperature=temp)
    o.step(steps)
    assert _bits_equal(o.output(), out)
    assert _bits_equal(o.temperature(), ref.temperature)


def _halo_oracles(cfg, pks, pre, steps, offset, halo, every, precision="f32"):
    n = int(round(pks[0].shape[0] ** (1 / 3)))
    os_ = [O.Oracle((n, n, n), O.derive_params(cfg), precision) for _ in pks]
    for o, pk in zip(os_, pks):
        o.set_temperature(pre)
        o.set_fields(pk[:, 0].reshape(n, n, n).astype(np.uint8), *(pk[:, 5 + a].reshape(n, n, n) for a in range(3)),
                     temperature=pk[:, 10].reshape(n, n, n))
    for s in range(steps):
        for o in os_:
            o.step(1)
        if s + 1 < steps and (s + 1) % every == 0:
            os_[0].exchange_halo(os_[1], offset, halo)
    return os_


def test_oracle_halo_exchange_matches_golden():
    """Two overlapping bricks with the reference's halo exchange between calls
    (populations and temperature of the slabs), bit-identical to the
    reference library's fixture."""
    g = np.load(GOLDEN / "halo_12_12.npz")
    cfg, pks, pre = O.halo_case(int(g["n"]))
    os_ = _halo_oracles(cfg, pks, pre, int(g["steps"]), tuple(int(v) for v in g["offset"]), int(g["halo"]), int(g["every"]))
    assert _bits_equal(os_[0].output(), g["out1"]) and _bits_equal(os_[1].output(), g["out2"])
    assert _bits_equal(os_[0].temperature(), g["t1"]) and _bits_equal(os_[1].temperature(), g["t2"])


@pytest.mark.skipif(not O.REF_LIB.exists(), reason="reference library not built here")
@pytest.mark.parametrize("offset,halo,buoy", [((1, 0, 0), 2, False), ((0, -1, 1), 3, True), ((1, 1, 1), 1, True)])
def test_oracle_halo_exchange_matches_reference_live(offset, halo, buoy):
    n, steps, every = 12, 9, 2
    cfg, pks, pre = O.halo_case(n, buoyancy=buoy)
    ref = O.RefLib()
    outs = ref.run_pair((n, n, n), cfg, pks, steps, offset, halo, exchange_every=every, temperature_states=(pre, pre))
    os_ = _halo_oracles(cfg, pks, pre, steps, offset, halo, every)
    for o, out, t in zip(os_, outs, ref.temperatures):
        assert _bits_equal(o.output(), out)
        assert _bits_equal(o.temperature(), t)


def _ctxops_oracle(n, seed, script=None):
    obst, u, temp, src, cfg, pre = O.thermal_case(n, seed)
    pk = O.packet_from(obst, *u, temperature=temp, source=src)
    o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
    o.set_temperature(pre)
    return O.run_script_oracle(o, cfg, pk, script or O.context_ops_script(n)), (cfg, pk, pre)


def test_oracle_context_ops_match_golden():
    """Shifts, sparse overlays, point and sub-box reads around the step
    (fixture ctxops_12.npz from the reference library), bit for bit."""
    g = np.load(GOLDEN / "ctxops_12.npz")
    res, _ = _ctxops_oracle(int(g["n"]), int(g["seed"]))
    ref = O.load_results(GOLDEN / "ctxops_12.npz")
    assert len(res) == len(ref) and all(O.results_equal(res, ref))


def test_oracle_cylinder_force_matches_golden():
    """The cylinder preset: parabolic inflow and the momentum-exchange force
    after each call (fixture cylinder_44x20x3.npz), bit for bit."""
    dims = (44, 20, 3)
    cfg, pk = O.cylinder_case(*dims)
    o = O.Oracle(dims, O.derive_params(cfg), "f32")
    res = O.run_script_oracle(o, cfg, pk, O.CYLINDER_SCRIPT)
    ref = O.load_results(GOLDEN / "cylinder_44x20x3.npz")
    assert all(O.results_equal(res, ref))
    assert abs(float(res[0][0])) > 0.0  # the disc does feel a force


@pytest.mark.skipif(not O.REF_LIB.exists(), reason="reference library not built here")
@pytest.mark.parametrize("seed,script", [(31, None),
                                         (32, [("step",)] * 3 + [("shift", 0, 0, -5), ("point", 11, 11, 11),
                                                                 ("subrect", 0, 0, 0, 12, 12, 12), ("step",),
                                                                 ("shift", 11, 0, 0), ("flow",), ("temp",)])])
def test_oracle_context_ops_match_reference_live(seed, script):
    n = 12
    res, (cfg, pk, pre) = _ctxops_oracle(n, seed, script)
    ref = O.RefLib().run_script((n, n, n), cfg, pk, script or O.context_ops_script(n), temperature_state=pre)
    assert all(O.results_equal(res, ref))


@pytest.mark.skipif(not O.REF_LIB.exists(), reason="reference library not built here")
def test_oracle_cylinder_force_matches_reference_live():
    dims = (30, 16, 2)
    cfg, pk = O.cylinder_case(*dims, sgs=False)
    script = [("step",), ("force",)] * 3 + [("flow",)]
    o = O.Oracle(dims, O.derive_params(cfg), "f32")
    res = O.run_script_oracle(o, cfg, pk, script)
    ref = O.RefLib().run_script(dims, cfg, pk, script)
    assert all(O.results_equal(res, ref))


def test_oracle_block_edits_and_shell_behaviour():
    """Block edits and the boundary shell have no CPU twin in the reference
    (its CPU build answers "OpenCL disabled"), so the oracle's restatement is
    their specification: a patched cell restarts at rest with the new mask,
    and the shell pulls the shell cells' velocity toward the target, more
    strongly in the outer layer, while a cleared shell leaves the step as it
    was."""
    n = 12
    obst, u, temp, src, cfg, pre = O.thermal_case(n, 41)
    pk = O.packet_from(obst, *u, temperature=temp, source=src)

    def run(script):
        o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
        o.set_temperature(pre)
        return o, O.run_script_oracle(o, cfg, pk, script)

    cell = int(np.flatnonzero(obst.reshape(-1) == 0)[100])
    o, res = run([("step",)] * 2 + [("patch", [cell], [0]), ("flow",)])
    f = o.populations()[:, cell]
    w = np.array([O.feq_rest(q) for q in range(27)])
    assert np.allclose(f, w, rtol=0, atol=1e-7)
    assert abs(res[0][cell]).max() == 0.0  # at rest: no velocity, no pressure
    o, _ = run([("step",)] * 2 + [("patch", [cell], [1])])
    assert o.mask()[cell] == 1

    target = np.zeros((n ** 3, 4), np.float32)
    target[:, 1] = 0.05
    base = [("step",)] * 2
    _, plain = run(base + [("cached",)] * 6 + [("flow",)])
    _, shelled = run(base + [("shell", target, 0b000001, 3, 0.4)] + [("cached",)] * 6 + [("flow",)])
    _, cleared = run(base + [("shell", target, 0b000001, 3, 0.4), ("shell", target, 0, 3, 0.4)] + [("cached",)] * 6
                     + [("flow",)])
    uy_plain = plain[0].reshape(n, n, n, 4)[..., 1]
    uy_shell = shelled[0].reshape(n, n, n, 4)[..., 1]
    fluid = obst == 0
    gain = [float(np.mean((uy_shell - uy_plain)[x][fluid[x]])) for x in range(4)]
    assert gain[0] > gain[1] > gain[2] > 0.0 and gain[0] > 1e-3, gain
    assert _bits_equal(cleared[0], plain[0])


def test_oracle_fans_and_sponge_match_golden():
    """Fan forcing (with noise) and the sponge of the reference's collide,
    bit for bit against fixture fans_12_12.npz."""
    cfg, pk, pre = O.fan_case(12, 61)
    o = O.Oracle((12, 12, 12), O.derive_params(cfg), "f32")
    o.set_temperature(pre)
    res = O.run_script_oracle(o, cfg, pk, O.FAN_SCRIPT)
    assert all(O.results_equal(res, O.load_results(GOLDEN / "fans_12_12.npz")))


@pytest.mark.skipif(not O.REF_LIB.exists(), reason="reference library not built here")
@pytest.mark.parametrize("noise,sponge,seed", [(True, True, 62), (False, True, 63), (True, False, 64)])
def test_oracle_fans_and_sponge_match_reference_live(noise, sponge, seed):
    cfg, pk, pre = O.fan_case(12, seed, noise, sponge)
    script = [("step",)] * 5 + [("flow",), ("temp",)]
    o = O.Oracle((12, 12, 12), O.derive_params(cfg), "f32")
    o.set_temperature(pre)
    res = O.run_script_oracle(o, cfg, pk, script)
    ref = O.RefLib().run_script((12, 12, 12), cfg, pk, script, temperature_state=pre)
    assert all(O.results_equal(res, ref))


def test_oracle_runtime_mode_matches_golden():
    """Benchmark mode off (the game runtime the brick service uses), bit for
    bit against fixture runtime_12_8.npz."""
    cfg, pk, pre = O.runtime_case(12, 71)
    o = O.Oracle((12, 12, 12), O.derive_params(cfg), "f32")
    o.set_temperature(pre)
    res = O.run_script_oracle(o, cfg, pk, O.RUNTIME_SCRIPT)
    assert all(O.results_equal(res, O.load_results(GOLDEN / "runtime_12_8.npz")))


@pytest.mark.skipif(not O.REF_LIB.exists(), reason="reference library not built here")
@pytest.mark.parametrize("seed,fans", [(72, True), (73, False)])
def test_oracle_runtime_mode_matches_reference_live(seed, fans):
    cfg, pk, pre = O.runtime_case(12, seed, fans)
    script = [("step",)] * 4 + [("flow",), ("temp",)] + [("step",)] * 3 + [("flow",), ("temp",)]
    o = O.Oracle((12, 12, 12), O.derive_params(cfg), "f32")
    o.set_temperature(pre)
    res = O.run_script_oracle(o, cfg, pk, script)
    ref = O.RefLib().run_script((12, 12, 12), cfg, pk, script, temperature_state=pre)
    assert all(O.results_equal(res, ref))


@pytest.mark.skipif(not O.REF_LIB.exists(), reason="reference library not built here")
@pytest.mark.parametrize("every", [1, 2, 3])
def test_oracle_runtime_halo_matches_reference_live(every):
    """Halo exchange in runtime mode: the temperature slabs move only after a
    call that updated the temperature (every other call there)."""
    n, steps, offset, halo = 12, 7, (1, 0, 0), 2
    cfg, pk1, pre = O.runtime_case(n, 74)
    _, pk2, _ = O.runtime_case(n, 75)
    ref = O.RefLib()
    outs = ref.run_pair((n, n, n), cfg, [pk1, pk2], steps, offset, halo, exchange_every=every,
                        temperature_states=(pre, pre))
    os_ = []
    for pk in (pk1, pk2):
        o = O.Oracle((n, n, n), O.derive_params(cfg), "f32")
        o.set_temperature(pre)
        os_.append(o)
    for s in range(steps):
        for o, pk in zip(os_, (pk1, pk2)):
            O.run_script_oracle(o, cfg, pk, [("step",)])
        if s + 1 < steps and (s + 1) % every == 0:
            os_[0].exchange_halo(os_[1], offset, halo)
    for o, out, t in zip(os_, outs, ref.temperatures):
        assert _bits_equal(o.output(), out)
        assert _bits_equal(o.temperature(), t)


@pytest.mark.skipif(not O.REF_LIB.exists(), reason="reference library not built here")
@pytest.mark.parametrize("channels", [9, 10])
def test_oracle_short_packets_match_reference_live(channels):
    """Packets without the temperature channel (10) or also without the source
    channel (9): the reference temperature is 0 and, with 9 channels, the
    transport's source comes from the fan channels, also on cells a sparse
    overlay rewrites (the overlay's source value is ignored then)."""
    cfg, pk, pre = O.runtime_case(12, 77, True, channels)
    script = O.short_packet_script(pk)
    o = O.Oracle((12, 12, 12), O.derive_params(cfg), "f32")
    o.set_temperature(pre)
    res = O.run_script_oracle(o, cfg, pk, script)
    ref = O.RefLib().run_script((12, 12, 12), cfg, pk, script, temperature_state=pre)
    assert all(O.results_equal(res, ref))
