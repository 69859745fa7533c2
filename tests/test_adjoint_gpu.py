"""Discrete adjoint of the brick step on the GPU (the inverse problem of the
64^3 differentiation set-up: gradients of a sparse-probe velocity-mismatch
loss with respect to the body-force field and the inflow vector).

* gradient of the FP32 forward vs central finite differences (eps = 1e-3
  relative) of the FP64 run of the same model, on 32 random force components
  and the 3 inflow components: relative error <= 1e-3;
* the same against central finite differences of the oracle (the reference
  scheme restated on the CPU, FP64) on a small brick;
* checkpointing every 20 calls gives the same gradient as storing every state;
* a torch.autograd.Function over the C ABI (this harness only) returns the
  gradient through backward(), checked by a directional derivative.
"""
from __future__ import annotations

import numpy as np
import pytest

import aero_b200
import oracle as O
from test_inplace_gpu import load_cases

pytestmark = pytest.mark.gpu
cases = load_cases()


def make_brick(c, **over):
    cfg = {**c.config, **over}
    b = aero_b200.AdjointBrick(c.obstacle, c.temperature, **cfg)
    return b


def targets_of(c, b):
    _, u = b.forward(c.force_true, c.inflow_true, precision=1)
    return u


def relerr(a, b):
    return abs(a - b) / max(abs(b), 1e-30)


@pytest.fixture(scope="module")
def c5(gpu):
    c = cases.c5_adjoint()
    b = make_brick(c)
    b.set_probes(c.probes, np.zeros((len(c.probes), 3), np.float32))
    t = targets_of(c, b)
    b.set_probes(c.probes, t)
    loss, gf, gu = b.gradient(c.force0, c.inflow0)
    yield c, b, loss, gf, gu
    b.close()


def loss64(b, force, inflow):
    return b.forward(force, inflow, precision=1)[0]


def test_loss_consistent(c5):
    c, b, loss, gf, gu = c5
    l32 = b.forward(c.force0, c.inflow0, precision=0)[0]
    l64 = loss64(b, c.force0, c.inflow0)
    assert loss > 0 and abs(loss - l32) <= 1e-12 * loss
    assert relerr(l32, l64) < 1e-4


def test_force_gradient_vs_finite_differences(c5):
    c, b, loss, gf, gu = c5
    rng = np.random.default_rng(7)
    flat = np.abs(gf).reshape(-1)
    # components whose gradient is not negligible (probe neighbourhoods)
    pool = np.flatnonzero(flat >= 1e-2 * flat.max())
    picks = rng.choice(pool, size=32, replace=False)
    worst = 0.0
    for k in picks:
        a, cell = divmod(int(k), b.cells)
        idx = (a,) + np.unravel_index(cell, b.dims)
        x0 = float(c.force0[idx])
        eps = 1e-3 * abs(x0) if x0 != 0 else 1e-9
        fp, fm = c.force0.copy(), c.force0.copy()
        fp[idx] = x0 + eps
        fm[idx] = x0 - eps
        # the perturbation actually stored in float32
        h = (float(np.float32(fp[idx])) - float(np.float32(fm[idx]))) / 2
        fd = (loss64(b, fp, c.inflow0) - loss64(b, fm, c.inflow0)) / (2 * h)
        worst = max(worst, relerr(float(gf[idx]), fd))
    assert worst <= 1e-3, worst


def test_inflow_gradient_vs_finite_differences(c5):
    c, b, loss, gf, gu = c5
    for a in range(3):
        x0 = c.inflow0[a]
        eps = 1e-3 * abs(x0) if x0 != 0 else 1e-6
        up, um = list(c.inflow0), list(c.inflow0)
        up[a] = x0 + eps
        um[a] = x0 - eps
        h = (float(np.float32(up[a])) - float(np.float32(um[a]))) / 2
        fd = (loss64(b, c.force0, up) - loss64(b, c.force0, um)) / (2 * h)
        assert relerr(gu[a], fd) <= 1e-3, (a, gu[a], fd)


def test_checkpointing_matches_store_all(c5):
    c, b, loss, gf, gu = c5
    t = targets_of(c, b)
    full = make_brick(c, checkpoint_every=1)
    full.set_probes(c.probes, t)
    l2, gf2, gu2 = full.gradient(c.force0, c.inflow0)
    full.close()
    assert l2 == loss
    assert np.array_equal(gf2, gf)
    assert np.array_equal(gu2, gu)


def test_gradient_vs_oracle_finite_differences(gpu):
    """Small brick: the adjoint gradient against central differences of the
    oracle's FP64 forward (the reference scheme restated on the CPU)."""
    c = cases.c5_adjoint(n=14, steps=24, checkpoint_every=5, seed=9, nprobe=12)
    b = make_brick(c)
    b.set_probes(c.probes, np.zeros((len(c.probes), 3), np.float32))
    t = targets_of(c, b)
    b.set_probes(c.probes, t)
    loss, gf, gu = b.gradient(c.force0, c.inflow0)
    b.close()

    def oracle_loss(force, inflow):
        p = O.OracleParams()
        p.tau_shear = p.tau_normal = np.float32(0.55)
        p.nu0 = np.float32(0.05) / np.float32(3.0)
        p.sgs_c2 = np.float32(0.1) * np.float32(0.1)
        p.sgs_nut_max_ratio, p.sgs_bulk_coupling = 5.0, np.float32(0.3)
        p.buoyancy_beta, p.buoyancy_force_max = np.float32(1e-4), np.float32(0.02)
        p.max_speed = np.float32(0.57735026919) * np.float32(0.6)
        p.enable_sgs, p.enable_buoyancy, p.gravity_axis = 1, 1, 2
        for f, k in enumerate(c.config["face_kind"]):
            p.face_kind[f] = k
            for a in range(3):
                p.face_velocity[f][a] = float(np.float32(inflow[a]))
        o = O.Oracle(c.dims, p, "f64")
        fluid = c.obstacle == 0
        u = [np.where(fluid, np.float32(inflow[a]), np.float32(0)).astype(np.float32) for a in range(3)]
        o.set_fields(c.obstacle, *u, np.zeros(c.dims, np.float32), c.temperature)
        o.set_force_field(*[np.ascontiguousarray(force[a]) for a in range(3)])
        o.step(c.config["steps"])
        f = o.populations()[:, c.probes]
        cx = np.array([q // 9 - 1 for q in range(27)], float)
        cy = np.array([(q // 3) % 3 - 1 for q in range(27)], float)
        cz = np.array([q % 3 - 1 for q in range(27)], float)
        rho = np.clip(f.sum(0), 0.97, 1.03)
        uu = np.stack([cx @ f, cy @ f, cz @ f], 1) / rho[:, None]
        return float(np.sum((uu - t.astype(np.float64)) ** 2))

    rng = np.random.default_rng(3)
    flat = np.abs(gf).reshape(-1)
    pool = np.flatnonzero(flat >= 1e-2 * flat.max())
    for k in rng.choice(pool, size=6, replace=False):
        a, cell = divmod(int(k), int(np.prod(c.dims)))
        idx = (a,) + np.unravel_index(cell, c.dims)
        x0 = float(c.force0[idx])
        fp, fm = c.force0.copy(), c.force0.copy()
        fp[idx] = x0 * (1 + 1e-3)
        fm[idx] = x0 * (1 - 1e-3)
        h = (float(np.float32(fp[idx])) - float(np.float32(fm[idx]))) / 2
        fd = (oracle_loss(fp, c.inflow0) - oracle_loss(fm, c.inflow0)) / (2 * h)
        assert relerr(float(gf[idx]), fd) <= 1e-3, (idx, gf[idx], fd)
    for a in (0, 1):
        x0 = c.inflow0[a]
        up, um = list(c.inflow0), list(c.inflow0)
        up[a], um[a] = x0 * (1 + 1e-3), x0 * (1 - 1e-3)
        h = (float(np.float32(up[a])) - float(np.float32(um[a]))) / 2
        fd = (oracle_loss(c.force0, up) - oracle_loss(c.force0, um)) / (2 * h)
        assert relerr(gu[a], fd) <= 1e-3, (a, gu[a], fd)


def test_torch_autograd_function(c5):
    torch = pytest.importorskip("torch")
    c, b, loss, gf, gu = c5

    class ProbeLoss(torch.autograd.Function):
        """Loss of the brick through the C ABI; backward = the adjoint sweep."""

        @staticmethod
        def forward(ctx, force, inflow):
            l, g_f, g_u = b.gradient(force.detach().cpu().numpy().astype(np.float32),
                                     inflow.detach().cpu().numpy().astype(np.float32))
            ctx.save_for_backward(torch.from_numpy(g_f), torch.from_numpy(g_u))
            return torch.tensor(l, dtype=torch.float64)

        @staticmethod
        def backward(ctx, grad_out):
            g_f, g_u = ctx.saved_tensors
            return grad_out * g_f, grad_out * g_u

    force = torch.tensor(c.force0, dtype=torch.float64, requires_grad=True)
    inflow = torch.tensor(c.inflow0, dtype=torch.float64, requires_grad=True)
    out = ProbeLoss.apply(force, inflow)
    out.backward()
    assert float(out.detach()) == pytest.approx(loss, rel=1e-12)
    # directional derivative along a smooth direction vs central differences
    rng = np.random.default_rng(1)
    d_f = cases.smooth_force_field(c.dims, 1e-6, 4.0, 99)
    d_u = rng.normal(size=3) * 1e-3
    h = 1e-3
    fp, fm = (c.force0 + h * d_f).astype(np.float32), (c.force0 - h * d_f).astype(np.float32)
    up = (np.asarray(c.inflow0) + h * d_u).astype(np.float32)
    um = (np.asarray(c.inflow0) - h * d_u).astype(np.float32)
    # the step actually taken (the brick reads float32 inputs)
    dfa = fp.astype(np.float64) - fm.astype(np.float64)
    dua = up.astype(np.float64) - um.astype(np.float64)
    ad = float((force.grad.numpy() * dfa).sum() + (inflow.grad.numpy() * dua).sum())
    fd = loss64(b, fp, up) - loss64(b, fm, um)
    assert relerr(ad, fd) <= 1e-3, (ad, fd)


def test_adjoint_cost_per_step(c5):
    """The gradient (segment recomputation + reverse launch) costs at most
    3 forward steps per step at the configured checkpoint interval (K = 20),
    timed on the device on warm calls (the lowest of three)."""
    c, b, loss, gf, gu = c5
    ratios = []
    for _ in range(3):
        b.gradient(c.force0, c.inflow0)
        t = b.timing()
        assert t["forward_ms_per_step"] > 0 and t["reverse_ms_per_step"] > 0
        ratios.append((t["recompute_ms_per_step"] + t["reverse_ms_per_step"]) / t["forward_ms_per_step"])
    print(f"adjoint step / forward step at K = {c.config.get('checkpoint_every')}: {min(ratios):.3f}")
    assert min(ratios) <= 3.0, ratios
