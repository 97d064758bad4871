"""The differentiable operator (autograd.py) on a small case with the
reconstruction configuration's laws (10 MHz, Moon occultation, 10 satellites):
the gradient w.r.t. the sky and the 30 satellite coordinates against central
finite differences (h = 1e-3) and against the FP64 operator's gradient; the
adjoint identity; and L-BFGS improving on the dirty image."""
import numpy as np
import pytest
import torch

from viss_optimize_3d_b200 import reconstruct, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small(viss, cuda_device):
    cfg = synth.scaled(synth.CONFIGS["c5"], nside=8, n_snap=24)
    return reconstruct.make_problem(cfg, device=cuda_device, seed=1), \
        reconstruct.make_problem(cfg, device=cuda_device, seed=1, fp64=True)


def _grads(p, x, d):
    x = x.clone().requires_grad_(True)
    d = d.clone().requires_grad_(True)
    L = reconstruct.loss(p, x, d)
    L.backward()
    return float(L.detach()), x.grad.double(), d.grad.double()


def _oracle_loss(oracle, p, lmn, occ, x, d):
    """The same weighted least-squares loss with the FP64 CPU oracle's forward."""
    u = reconstruct.baselines(p.P0, d, p.pairs, p.lam).cpu().numpy()
    V = oracle.forward(u, lmn, (x.double() * p.omega).cpu().numpy(), p.model.refs.cpu().numpy(), occ)
    r = (V - p.V_obs.cpu().numpy().astype(np.complex128)) * p.w.double().cpu().numpy()
    return float((r.real ** 2 + r.imag ** 2).sum() / p.sigma ** 2)


def test_gradient_vs_finite_differences_and_fp64(small, oracle):
    p, p64 = small
    gen = torch.Generator(device="cpu").manual_seed(0)
    x = (p.x_true.cpu() * (1 + 0.3 * torch.randn(p.x_true.shape, generator=gen))).to(p.x_true.device)
    d = torch.randn(p.delta_true.shape, generator=gen, dtype=torch.float64).to(x.device) * 3.0
    L, gx, gd = _grads(p64, x, d)
    lmn = p.model.lmn.cpu().numpy()
    occ = p.model.occ.cpu().numpy()
    assert abs(_oracle_loss(oracle, p, lmn, occ, x, d) - L) < 1e-5 * L
    # central differences of the FP64 oracle's loss, h = 1e-3 (sky units; metres)
    h = 1e-3
    for j in (0, 17, 301, 700):
        e = torch.zeros_like(x)
        e[j] = h
        fd = (_oracle_loss(oracle, p, lmn, occ, x + e, d) - _oracle_loss(oracle, p, lmn, occ, x - e, d)) / (2 * h)
        assert abs(fd - float(gx[j])) <= 1e-3 * float(gx.abs().max()), (j, fd, float(gx[j]))
    fd_d = torch.zeros_like(gd)
    for s_ in range(d.shape[0]):
        for c in range(3):
            e = torch.zeros_like(d)
            e[s_, c] = h
            fd_d[s_, c] = (_oracle_loss(oracle, p, lmn, occ, x, d + e)
                           - _oracle_loss(oracle, p, lmn, occ, x, d - e)) / (2 * h)
    assert float((fd_d - gd).norm() / gd.norm()) < 1e-3
    # the split-precision operator's gradient against the FP64 one
    _, gx32, gd32 = _grads(p, x, d)
    assert float((gx32 - gx).norm() / gx.norm()) < 1e-4
    assert float((gd32 - gd).norm() / gd.norm()) < 1e-3


def test_lbfgs_beats_dirty_image(small):
    p, _ = small
    dirty = reconstruct.dirty_image(p)
    x, delta, hist = reconstruct.reconstruct(p, iters=60)
    assert hist[-1] < 0.05 * hist[0]
    e_rec = reconstruct.rel_l2(x, p.x_true)
    e_dirty = reconstruct.rel_l2(dirty, p.x_true)
    assert e_rec < e_dirty, (e_rec, e_dirty)
    # position offsets move toward the truth (a common translation of every
    # satellite leaves the baselines unchanged, so compare centred offsets)
    c = lambda t: t - t.mean(dim=0, keepdim=True)
    assert float((c(delta) - c(p.delta_true)).norm()) < 0.5 * float(c(p.delta_true).norm())


def test_formation_operator_gradients(small, cuda_device):
    """The formation operator (satellite vectors in, autograd.FormationModel):
    loss and gradients against the FP64 direct operator, within the split
    path's own tolerances, and closer still to the split direct operator."""
    p, p64 = small
    pf = reconstruct.make_problem(p.cfg, device=cuda_device, seed=1, formation=True)
    assert torch.equal(pf.V_obs, p.V_obs)
    gen = torch.Generator(device="cpu").manual_seed(3)
    x = (p.x_true.cpu() * (1 + 0.3 * torch.randn(p.x_true.shape, generator=gen))).to(p.x_true.device)
    d = torch.randn(p.delta_true.shape, generator=gen, dtype=torch.float64).to(x.device) * 3.0
    L64, gx64, gd64 = _grads(p64, x, d)
    L32, gx32, gd32 = _grads(p, x, d)
    Lf, gxf, gdf = _grads(pf, x, d)
    assert abs(Lf - L64) < 1e-5 * L64
    assert float((gxf - gx64).norm() / gx64.norm()) < 1e-4
    assert float((gdf - gd64).norm() / gd64.norm()) < 1e-3
    assert float((gxf - gx32).norm() / gx32.norm()) < 1e-4
    dirty = reconstruct.dirty_image(pf)
    xr, _dr, hist = reconstruct.reconstruct(pf, iters=40)
    assert hist[-1] < 0.1 * hist[0]
    assert reconstruct.rel_l2(xr, pf.x_true) < reconstruct.rel_l2(dirty, pf.x_true)
