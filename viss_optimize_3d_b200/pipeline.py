"""One observation through the hot path, on the GPU: the stage order of the
reference's host function vissGen (vissgen3d_blockage.cu:195-563) without its
text I/O:

  pix2ang -> (l, m, n)          pix2ang.cu:92-160, vissgen3d_blockage.cu:53-74
  sky * 4 pi / npix             vissgen3d_blockage.cu:72, :242
  forward V (+ occultation)     vissgen3d_blockage.cu:76-102
  shells + DCF                  vissgen3d_blockage.cu:105-141 (un-shifted)
  dg, weights                   vissgen3d_blockage.cu:144-164, :178, :187
  adjoint image (+ occultation) vissgen3d_blockage.cu:167-192

The reference evaluates every sample twice, once as itself and once as its
conjugate mirror (V[i+amount] = conj(V[i]), :100).  Here only the unique
samples are evaluated: the histogram counts each one twice (multiplicity 2)
and the adjoint's real part is doubled (scale 2), which is the reference's
sum over both halves whenever the mirror rows are exact negatives.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
import torch

from . import api
from .synth import C_LIGHT, Observation, R_MOON


@dataclasses.dataclass
class GpuObservation:
    """Device-resident inputs of one observation at one frequency."""
    obs: Observation
    f_hz: float
    lmn: torch.Tensor       # (J, 3) FP64, RING order
    sky: torch.Tensor       # (J,) FP32, already scaled by 4 pi / npix
    uvw: torch.Tensor       # (K, 3) FP64
    w: torch.Tensor         # (K,) FP32
    bll: torch.Tensor       # (K,) FP32
    refs: torch.Tensor | None
    occ: torch.Tensor | None
    nr: int
    plan: api.Plan


def build_occulters(obs: Observation, device) -> torch.Tensor | None:
    if obs.refs is None:
        return None
    P = torch.as_tensor(obs.occ_sat_positions, dtype=torch.float64, device=device)
    occ = api.occulters(P, R=R_MOON, mode=0)
    if obs.earth_rows is not None:
        occ = torch.cat([occ, torch.as_tensor(obs.earth_rows, dtype=torch.float64, device=device)])
    return occ.contiguous()


def formation_inputs(obs: Observation, f_hz: float, device="cuda", occ: torch.Tensor | None = None):
    """(U, occ_sat, occ_snap) of viss_plan_set_formation for a synthetic
    observation: U = (P - formation centre) / lambda per snapshot (the pair
    differences are the observation's uvw), and the occulter rows split into
    the satellites' (T*S first rows of build_occulters) and the snapshots'."""
    cfg = obs.cfg
    P = np.asarray(obs.positions, dtype=np.float64)
    U = (P - P.mean(axis=1, keepdims=True)) / (C_LIGHT / f_hz)
    occ_sat = occ_snap = None
    if obs.refs is not None:
        occ = build_occulters(obs, device) if occ is None else occ
        T, S = cfg.n_snap, cfg.n_sat
        if cfg.moon:
            occ_sat = occ[:T * S].reshape(T, S, 4)
        if obs.earth_rows is not None:
            occ_snap = occ[T * S:T * S + T]
    return torch.as_tensor(U, device=device), occ_sat, occ_snap


def upload(obs: Observation, f_hz: float, device="cuda", lmn: torch.Tensor | None = None,
           occ: torch.Tensor | None = None) -> GpuObservation:
    cfg = obs.cfg
    if lmn is None:
        lmn = api.pix2lmn(cfg.nside, "ring", device=device)
    uvw_np = obs.uvw(f_hz)
    uvw = torch.as_tensor(uvw_np, dtype=torch.float64, device=device)
    w = torch.as_tensor(uvw_np[:, 2], dtype=torch.float32, device=device)
    bll = torch.as_tensor(np.linalg.norm(uvw_np, axis=1), dtype=torch.float32, device=device)
    omega = 4.0 * math.pi / cfg.npix
    sky = torch.as_tensor(obs.sky_at(f_hz) * omega, dtype=torch.float32, device=device)
    refs = None if obs.refs is None else torch.as_tensor(obs.refs, dtype=torch.int32, device=device)
    if occ is None:
        occ = build_occulters(obs, device)
    plan = api.Plan(lmn, uvw, None, refs, occ)
    return GpuObservation(obs, f_hz, lmn, sky, uvw, w, bll, refs, occ, obs.nr(f_hz), plan)


def dirty_image(g: GpuObservation, V: torch.Tensor, fp64: bool = False, gridded: bool = False) -> torch.Tensor:
    """DCF weights and the imaging adjoint for visibilities V; gridded: through
    viss_adjoint_gridded (per-facet NUFFTs; split precision only)."""
    gs, _counts, dcf = api.dcf(g.bll, g.nr, multiplicity=2)
    _dg, wt = api.weights(g.w, g.bll, gs, dcf, g.nr)
    coef = api.scale_coef(wt, V)
    if gridded:
        if fp64:
            raise ValueError("the gridded adjoint is split precision only")
        return g.plan.adjoint_gridded(coef, scale=2.0, mask=g.obs.cfg.imaging_mask)
    return g.plan.adjoint(coef, scale=2.0, fp64=fp64, mask=g.obs.cfg.imaging_mask)


def observe(g: GpuObservation, fp64: bool = False, gridded: bool = False):
    """Forward visibilities and the density-compensated dirty image."""
    V = g.plan.forward(g.sky, fp64=fp64)
    img = dirty_image(g, V, fp64=fp64, gridded=gridded)
    return V, img
