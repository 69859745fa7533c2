"""Generate the golden fixtures in this directory from the reference library.

The reference's own CPU step (compiled from its sources into
oracle/_ref/libaero_lbm_ref.so by `make -C oracle ref`) is driven through its C
ABI on seeded inputs; its write_output results are saved as .npz together with
the seed and a checksum of the inputs. Run from the repository root:

    python tests/golden/make_golden.py

Fixtures:
  c1_32_1000.npz  plain FP32 brick 32^3, periodic x/y, bounce-back z, solid
                  floor z=0 + Bernoulli(0.05) interior, tau 0.55, SGS on,
                  u = (0.05,0,0) + U(-0.005,0.005); 1000 steps.
  c1_16_200.npz   the same set-up at 16^3, 200 steps.
  tunnel_16_60.npz wind-tunnel faces (velocity inlet x-, convective outflow
                  x+, symmetry y/z), sphere obstacle, SGS off; 60 steps.
  meso_12x8x10_30.npz D3Q19 mesoscale step (aero_lbm_mesoscale_step_context),
                  12 x 8 x 10 (y up), seeded 25-channel forcing (seed 5,
                  terrain up to 3 cells, wind (6, 0, 3) m/s), dx 64 m,
                  dt 5 s; the 6-channel state after 30 calls.
  cavity_12_25.npz the differentially heated cavity preset (3-D) with the
                  BFECC temperature transport: oracle.heated_cavity_case(12,
                  seed 3), 25 steps; write_output and the temperature state.
  halo_12_12.npz  two overlapping 12^3 bricks (oracle.halo_case: the thermal
                  case and a second seeded brick, buoyancy on), halo 2 at
                  offset (1, -1, 0), aero_lbm_exchange_halo_layers_rect after
                  every third of 12 calls; both write_output results and
                  temperature states.
  ctxops_12.npz   the per-context entry points around the step
                  (oracle.context_ops_script: steps, shifts, sparse overlays,
                  point and sub-box reads, the last force) on
                  oracle.thermal_case(12, seed 21) with the transport; every
                  recorded result in order (r<i>, or r<i>_0 / r<i>_1 for pairs).
  cylinder_44x20x3.npz the cylinder crossflow preset (oracle.cylinder_case:
                  parabolic inflow, convective outflow, the disc as the mask):
                  the momentum-exchange force after each of 5 calls and the
                  final flow (oracle.CYLINDER_SCRIPT).
  brickworld_16x4_6.npz the reference's brick-world service (its simulation
                  bridge over its CPU step, oracle.BrickService) on
                  oracle.brick_world_case(): four 16^3 bricks, 6 ticks in the
                  classic solver mode; packed atlases, dynamic bricks, status.
  fans_12_12.npz  the fan forcing, fan noise and sponge of the reference's
                  collide switched on in benchmark mode (oracle.fan_case(12,
                  seed 61)): flow and temperature after 6 calls, flow after 12.
  runtime_12_8.npz benchmark mode off (the reference's game runtime:
                  fans, noise, sponge, state nudge, every-other-call BFECC
                  transport with eddy diffusivity, convective outflow faces),
                  oracle.runtime_case(12, seed 71), oracle.RUNTIME_SCRIPT.
  thermal_12_20.npz buoyancy on with the reference's temperature transport:
                  oracle.thermal_case(12, seed 11) (every thermal face kind,
                  packet source channel, state preloaded), 20 steps; the
                  write_output result and the temperature state.

`python tests/golden/make_golden.py thermal` regenerates only the fixtures
whose name contains "thermal" (any substring filter works).
"""
from __future__ import annotations

import hashlib
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def tunnel_case(n: int = 16):
    """Sphere in a wind tunnel (the reference tools' check geometry)."""
    obst = np.zeros((n, n, n), np.uint8)
    c = np.array([n // 3, n // 2, n // 2])
    r = max(1.0, n * 0.12)
    g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1)
    obst[np.sum((g - c) ** 2, -1) <= r * r] = 1
    u_in = 0.1
    ux = np.where(obst == 0, np.float32(u_in), np.float32(0)).astype(np.float32)
    zero = np.zeros_like(ux)
    cfg = {
        "reynolds": u_in / 0.01,
        "initial_velocity": (u_in, 0.0, 0.0),
        "faces": [{"kind": O.VELOCITY, "velocity": (u_in, 0.0, 0.0)}, {"kind": O.CONVECTIVE},
                  {"kind": O.SYMMETRY}, {"kind": O.SYMMETRY}, {"kind": O.SYMMETRY}, {"kind": O.SYMMETRY}],
        "sgs": False,
        "buoyancy": False,
    }
    return obst, (ux, zero, zero.copy()), cfg


def thermal_fixture(ref) -> None:
    n, seed, steps = 12, 11, 20
    obst, u, temp, src, cfg, preload = O.thermal_case(n, seed)
    pk = O.packet_from(obst, *u, temperature=temp, source=src)
    out = ref.run((n, n, n), cfg, pk, steps, temperature_state=preload)
    np.savez_compressed(OUT / "thermal_12_20.npz", out=out, temperature=ref.temperature, seed=seed, n=n, steps=steps,
                        input_sha256=digest(pk, preload))
    print("thermal_12_20 written")


def cavity_fixture(ref) -> None:
    n, seed, steps = 12, 3, 25
    obst, u, temp, cfg, preload = O.heated_cavity_case(n, seed)
    pk = O.packet_from(obst, *u, temperature=temp)
    out = ref.run((n, n, n), cfg, pk, steps, temperature_state=preload)
    np.savez_compressed(OUT / "cavity_12_25.npz", out=out, temperature=ref.temperature, seed=seed, n=n, steps=steps,
                        input_sha256=digest(pk, preload))
    print("cavity_12_25 written")


def halo_fixture(ref) -> None:
    n, steps, offset, halo, every = 12, 12, (1, -1, 0), 2, 3
    cfg, pks, pre = O.halo_case(n)
    outs = ref.run_pair((n, n, n), cfg, pks, steps, offset, halo, exchange_every=every, temperature_states=(pre, pre))
    np.savez_compressed(OUT / "halo_12_12.npz", out1=outs[0], out2=outs[1], t1=ref.temperatures[0], t2=ref.temperatures[1],
                        n=n, steps=steps, offset=np.array(offset), halo=halo, every=every,
                        input_sha256=digest(pks[0], pks[1], pre))
    print("halo_12_12 written")


def save_results(path, results, **meta) -> None:
    arrays = {}
    for i, r in enumerate(results):
        if isinstance(r, tuple):
            for j, a in enumerate(r):
                arrays[f"r{i}_{j}"] = a
        else:
            arrays[f"r{i}"] = r
    np.savez_compressed(path, count=len(results), **arrays, **meta)


def ctxops_fixture(ref) -> None:
    n, seed = 12, 21
    obst, u, temp, src, cfg, pre = O.thermal_case(n, seed)
    pk = O.packet_from(obst, *u, temperature=temp, source=src)
    res = ref.run_script((n, n, n), cfg, pk, O.context_ops_script(n), temperature_state=pre)
    save_results(OUT / "ctxops_12.npz", res, n=n, seed=seed, input_sha256=digest(pk, pre))
    print("ctxops_12 written")


def cylinder_fixture(ref) -> None:
    dims = (44, 20, 3)
    cfg, pk = O.cylinder_case(*dims)
    res = ref.run_script(dims, cfg, pk, O.CYLINDER_SCRIPT)
    save_results(OUT / "cylinder_44x20x3.npz", res, dims=np.array(dims), input_sha256=digest(pk))
    print("cylinder_44x20x3 written")


def brickworld_fixture() -> None:
    w = O.brick_world_case()
    r = O.BrickService(O.SIM_REF_LIB).run(w)
    np.savez_compressed(OUT / "brickworld_16x4_6.npz", atlas=np.stack(r["atlas"]), flow=np.stack(r["flow"]),
                        air_t=np.stack(r["air_t"]), status=r["status"], steps=w["steps"], n=w["n"],
                        input_sha256=digest(*w["obstacle"], *w["flow"], *w["air_t"]))
    print("brickworld_16x4_6 written")


def fans_fixture(ref) -> None:
    cfg, pk, pre = O.fan_case(12, 61)
    res = ref.run_script((12, 12, 12), cfg, pk, O.FAN_SCRIPT, temperature_state=pre)
    save_results(OUT / "fans_12_12.npz", res, input_sha256=digest(pk, pre))
    print("fans_12_12 written")


def runtime_fixture(ref) -> None:
    cfg, pk, pre = O.runtime_case(12, 71)
    res = ref.run_script((12, 12, 12), cfg, pk, O.RUNTIME_SCRIPT, temperature_state=pre)
    save_results(OUT / "runtime_12_8.npz", res, input_sha256=digest(pk, pre))
    print("runtime_12_8 written")


def main() -> int:
    O.build(ref=True)
    ref = O.RefLib()
    only = sys.argv[1] if len(sys.argv) > 1 else ""
    if only:
        if only in "thermal_12_20":
            thermal_fixture(ref)
        if only in "cavity_12_25":
            cavity_fixture(ref)
        if only in "halo_12_12":
            halo_fixture(ref)
        if only in "ctxops_12":
            ctxops_fixture(ref)
        if only in "cylinder_44x20x3":
            cylinder_fixture(ref)
        if only in "brickworld_16x4_6":
            brickworld_fixture()
        if only in "fans_12_12":
            fans_fixture(ref)
        if only in "runtime_12_8":
            runtime_fixture(ref)
        return 0
    for name, n, steps in (("c1_16_200", 16, 200), ("c1_32_1000", 32, 1000)):
        seed = 1234
        obst, u = O.c1_inputs(seed=seed, n=n)
        cfg = O.c1_config()
        pk = O.packet_from(obst, *u)
        t0 = time.time()
        out = ref.run((n, n, n), cfg, pk, steps)
        print(f"{name}: reference {steps} steps in {time.time() - t0:.1f}s")
        np.savez_compressed(OUT / f"{name}.npz", out=out, seed=seed, n=n, steps=steps,
                            input_sha256=digest(pk))
    obst, u, cfg = tunnel_case(16)
    pk = O.packet_from(obst, *u)
    out = ref.run((16, 16, 16), cfg, pk, 60)
    np.savez_compressed(OUT / "tunnel_16_60.npz", out=out, obstacle=obst, steps=60, input_sha256=digest(pk))
    print("tunnel_16_60 written")
    dims, seed, steps = (12, 8, 10), 5, 30
    forcing = O.meso_forcing(dims, seed=seed)
    out = O.meso_ref_run(dims, forcing, steps)
    np.savez_compressed(OUT / "meso_12x8x10_30.npz", out=out, seed=seed, dims=np.array(dims), steps=steps,
                        input_sha256=digest(forcing))
    print("meso_12x8x10_30 written")
    thermal_fixture(ref)
    cavity_fixture(ref)
    halo_fixture(ref)
    ctxops_fixture(ref)
    cylinder_fixture(ref)
    brickworld_fixture()
    fans_fixture(ref)
    runtime_fixture(ref)
    return 0


if __name__ == "__main__":
    sys.exit(main())
