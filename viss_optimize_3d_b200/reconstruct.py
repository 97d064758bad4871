"""Differentiable sky reconstruction beside the reference's dirty image.

The reference images by density-compensated back-projection only
(computeC, vissgen3d_blockage.cu:167-192).  Here the same geometry is solved
as weighted least squares,

    L(x, delta) = || w (A(Omega x, u(delta)) - V_obs) ||^2 / sigma^2,

for the sky x (per-pixel intensity, Omega = 4 pi / npix) and a constant
position offset delta per satellite (the 30 coordinates of 10 satellites),
with u(delta) = (P_a + delta_a - P_b - delta_b) / lambda, using
torch.optim.LBFGS on the GPU operator of autograd.py (exponentials recomputed
in every pass, never stored).  w are the shell-histogram DCF weights.  With
formation=True the operator is FormationModel: the same A through the
formation entry points, its input the satellite vectors
U = (P0 + delta - c) / lambda (c: each snapshot's nominal centroid).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
import torch

from . import api, synth
from .autograd import FormationModel, VisibilityModel
from .pipeline import build_occulters


@dataclasses.dataclass
class Problem:
    cfg: synth.ObsConfig
    lam: float
    omega: float
    P0: torch.Tensor          # (T, S, 3) nominal positions (m)
    pairs: torch.Tensor       # (B, 2)
    delta_true: torch.Tensor  # (S, 3) true position offsets (m)
    x_true: torch.Tensor      # (J,) true sky
    V_obs: torch.Tensor       # (K,) observed visibilities
    sigma: float
    w: torch.Tensor           # (K,) weights
    model: VisibilityModel | FormationModel
    centre: torch.Tensor | None = None  # (T, 1, 3) per-snapshot origin of U (formation model)


def baselines(P0: torch.Tensor, delta: torch.Tensor, pairs: torch.Tensor, lam: float) -> torch.Tensor:
    """u (T*B, 3) in wavelengths, sample order (snapshot, baseline)."""
    P = P0 + delta[None, :, :]
    d = P[:, pairs[:, 0], :] - P[:, pairs[:, 1], :]
    return (d / lam).reshape(-1, 3)


def formation_vectors(P0: torch.Tensor, delta: torch.Tensor, centre: torch.Tensor, lam: float) -> torch.Tensor:
    """U (T, S, 3) in wavelengths: U_a - U_b is baselines()' u of pair (a, b)."""
    return (P0 + delta[None, :, :] - centre) / lam


def make_problem(cfg: synth.ObsConfig, device="cuda", seed: int = 0, snr: float = 20.0,
                 pos_sigma_m: float = 5.0, fp64: bool = False, formation: bool = False) -> Problem:
    obs = synth.make_observation(cfg)
    f = cfg.freqs_hz[0]
    lam = synth.C_LIGHT / f
    omega = 4 * math.pi / cfg.npix
    lmn = api.pix2lmn(cfg.nside, "ring", device=device)
    occ = build_occulters(obs, device)
    model = VisibilityModel(lmn, obs.refs, occ, fp64=fp64)
    g = torch.Generator(device="cpu").manual_seed(seed + 77)
    P0 = torch.as_tensor(obs.positions, device=device)
    pairs = torch.as_tensor(obs.pairs, device=device, dtype=torch.long)
    delta_true = (torch.randn((cfg.n_sat, 3), generator=g, dtype=torch.float64) * pos_sigma_m).to(device)
    x_true = torch.as_tensor(obs.sky, dtype=torch.float32, device=device)
    with torch.no_grad():
        V = model.forward_raw(x_true * omega, baselines(P0, delta_true, pairs, lam))
    sigma = float(V.abs().pow(2).mean().sqrt()) / snr
    noise = torch.complex(torch.randn(V.shape, generator=g), torch.randn(V.shape, generator=g))
    V_obs = V + (noise * (sigma / math.sqrt(2))).to(device=device, dtype=torch.complex64)
    bll = torch.as_tensor(obs.bll(f), dtype=torch.float32, device=device)
    w_np = obs.uvw(f)[:, 2]
    gs, _c, dcf = api.dcf(bll, obs.nr(f), multiplicity=2)
    _dg, wt = api.weights(torch.as_tensor(w_np, dtype=torch.float32, device=device), bll, gs, dcf,
                          obs.nr(f))
    w = wt / wt.mean()
    centre = None
    if formation:
        if fp64:
            raise ValueError("the formation entry points are split precision only")
        T, S = cfg.n_snap, cfg.n_sat
        occ_sat = occ[:T * S].reshape(T, S, 4) if cfg.moon else None
        occ_snap = occ[T * S:T * S + T] if obs.earth_rows is not None else None
        model = FormationModel(lmn, occ_sat, occ_snap)
        centre = P0.mean(dim=1, keepdim=True)
    return Problem(cfg, lam, omega, P0, pairs, delta_true, x_true, V_obs, sigma, w, model, centre)


def operator_input(p: Problem, delta: torch.Tensor) -> torch.Tensor:
    """What the problem's model takes: u (K, 3) or, for the formation model, U (T, S, 3)."""
    if p.centre is not None:
        return formation_vectors(p.P0, delta, p.centre, p.lam)
    return baselines(p.P0, delta, p.pairs, p.lam)


def loss(p: Problem, x: torch.Tensor, delta: torch.Tensor) -> torch.Tensor:
    V = p.model(x * p.omega, operator_input(p, delta))
    r = (V - p.V_obs).to(torch.complex128) * p.w.to(torch.float64)
    return (r.real.square() + r.imag.square()).sum() / (p.sigma ** 2)


def dirty_image(p: Problem) -> torch.Tensor:
    """The reference's density-compensated back-projection of V_obs at the
    nominal positions, scaled by the least-squares factor onto the true sky
    (the dirty image has arbitrary units)."""
    with torch.no_grad():
        u0 = operator_input(p, torch.zeros_like(p.delta_true))
        img = p.model.adjoint_raw((p.V_obs * p.w).contiguous(), u0).to(torch.float64)
        t = p.x_true.to(torch.float64)
        a = float((img * t).sum() / (img * img).sum())
    return (a * img).to(torch.float32)


def rel_l2(a: torch.Tensor, b: torch.Tensor) -> float:
    a, b = a.to(torch.float64), b.to(torch.float64)
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def reconstruct(p: Problem, iters: int = 200, positions: bool = True, x0=None,
                history_size: int = 20):
    """L-BFGS over (x, delta); returns (x, delta, loss history)."""
    x = (x0.clone() if x0 is not None else torch.zeros_like(p.x_true)).requires_grad_(True)
    delta = torch.zeros_like(p.delta_true).requires_grad_(positions)
    params = [x] + ([delta] if positions else [])
    opt = torch.optim.LBFGS(params, lr=1.0, max_iter=iters, max_eval=int(iters * 1.5),
                            history_size=history_size, tolerance_grad=0.0,
                            tolerance_change=0.0, line_search_fn="strong_wolfe")
    hist = []

    def closure():
        opt.zero_grad()
        L = loss(p, x, delta)
        L.backward()
        hist.append(float(L.detach()))
        return L

    opt.step(closure)
    return x.detach(), delta.detach(), hist
