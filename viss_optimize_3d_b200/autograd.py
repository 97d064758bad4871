"""Differentiable visibility operator for sky reconstruction.

V = A(I, u):  V_k = sum_j I_j vis_kj exp(-2 pi i u_k . s_j)   (viss_forward)

is exposed as a torch.autograd.Function of the sky I (J, FP32) and the
baselines u (K x 3, FP64, in wavelengths).  Nothing of A is stored: the
backward pass recomputes the exponentials in the GPU kernels.

  dL/dI_j    = Re( sum_k conj(A_kj) g_k )                 -- viss_adjoint with
               coef = g, the weighted back-projection (the dirty image's kernel)
  dL/du_kc   = Re( g_k conj(dV_k/du_kc) ) = -2 pi Im( g_k conj(D_kc) ),
               D_kc = sum_j I_j vis_kj s_jc exp(-2 pi i u_k . s_j)

where g = dL/dV in PyTorch's convention for complex tensors (for a real loss,
the gradient of V is 2 dL/dconj(V)).  D is the phase derivative: three extra
visibility sums with the sky weighted by l, m and n, computed as one
three-channel viss_forward.  The occultation mask is held fixed (it is not
differentiable in u).  Gradients w.r.t. satellite positions follow from u's
torch graph (u = (P_a - P_b) / lambda).

FormationModel is the same operator on the formation entry points
(viss_forward_formation / viss_adjoint_formation): its input is the satellite
vectors U (T x S x 3) instead of u, with u_ab = U_a - U_b, so
dL/dU_a = sum_b dL/du_ab - sum_b' dL/du_b'a, and D is three formation
forwards of the weighted sky.
"""
from __future__ import annotations

import math

import torch

from .api import Plan


class VisibilityModel:
    """A(I, u) on a fixed pixel grid with fixed occultation rows.

    lmn (J, 3) FP64 sky directions; refs (K, 3) / occ (G, 4) the occultation
    (None: no mask); fp64 selects the plain FP64 kernels.
    """

    def __init__(self, lmn: torch.Tensor, refs=None, occ=None, fp64: bool = False):
        self.lmn = lmn.to(torch.float64).contiguous()
        self.refs = None if refs is None else torch.as_tensor(refs, device=self.lmn.device)
        self.occ = occ
        self.fp64 = fp64
        self.plan = Plan(self.lmn)
        self.dplan = Plan(self.lmn)
        self._u = None
        self._du = None

    def _stage(self, uvw: torch.Tensor):
        if self._u is None or self._u.shape != uvw.shape or not torch.equal(self._u, uvw):
            self.plan.set_samples(uvw, None, self.refs, self.occ)
            self._u = uvw.detach().clone()

    def _stage_d(self, uvw: torch.Tensor):
        if self._du is None or self._du.shape != uvw.shape or not torch.equal(self._du, uvw):
            refs3 = None if self.refs is None else self.refs.repeat(3, 1)
            self.dplan.set_samples(uvw.repeat(3, 1), None, refs3, self.occ)
            self.dplan.set_channels(3)
            self._du = uvw.detach().clone()

    def forward_raw(self, sky: torch.Tensor, uvw: torch.Tensor) -> torch.Tensor:
        self._stage(uvw)
        return self.plan.forward(sky.contiguous(), fp64=self.fp64)

    def adjoint_raw(self, coef: torch.Tensor, uvw: torch.Tensor) -> torch.Tensor:
        self._stage(uvw)
        return self.plan.adjoint(coef.contiguous(), fp64=self.fp64)

    def dphase(self, sky: torch.Tensor, uvw: torch.Tensor) -> torch.Tensor:
        """D (K, 3) complex: sum_j I_j vis_kj s_jc exp(-2 pi i u_k . s_j)."""
        self._stage_d(uvw)
        sky3 = (sky.to(torch.float64)[None, :] * self.lmn.T).to(torch.float32).contiguous()
        D = self.dplan.forward(sky3, fp64=self.fp64)
        return D.view(3, -1).T

    def __call__(self, sky: torch.Tensor, uvw: torch.Tensor) -> torch.Tensor:
        return _Visibility.apply(sky, uvw, self)


class _Visibility(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sky, uvw, model: VisibilityModel):
        ctx.model = model
        ctx.save_for_backward(sky, uvw)
        return model.forward_raw(sky.detach().to(torch.float32), uvw.detach().to(torch.float64))

    @staticmethod
    def backward(ctx, g):
        sky, uvw = ctx.saved_tensors
        m = ctx.model
        g = g.to(torch.complex64).contiguous()
        u = uvw.detach().to(torch.float64)
        grad_sky = grad_uvw = None
        if ctx.needs_input_grad[0]:
            grad_sky = m.adjoint_raw(g, u).to(sky.dtype)
        if ctx.needs_input_grad[1]:
            D = m.dphase(sky.detach().to(torch.float32), u)
            grad_uvw = (-2.0 * math.pi) * (g.to(torch.complex128)[:, None] * D.conj().to(torch.complex128)).imag
            grad_uvw = grad_uvw.to(uvw.dtype)
        return grad_sky, grad_uvw, None


class FormationModel:
    """A(I, U) for a satellite formation on a fixed pixel grid.

    lmn (J, 3) FP64; occ_sat (T, S, 4) / occ_snap (T, 4) fixed occulter rows
    (None: no mask).  Sample order t * S(S-1)/2 + pair, pairs a < b in
    lexicographic order.
    """

    def __init__(self, lmn: torch.Tensor, occ_sat=None, occ_snap=None):
        self.lmn = lmn.to(torch.float64).contiguous()
        self.occ_sat = occ_sat
        self.occ_snap = occ_snap
        self.plan = Plan(self.lmn)
        self._U = None
        self._pairs = None

    def _stage(self, U: torch.Tensor):
        if self._U is None or self._U.shape != U.shape or not torch.equal(self._U, U):
            self.plan.set_formation(U, None, self.occ_sat, self.occ_snap)
            self._U = U.detach().clone()
            S = U.shape[1]
            if self._pairs is None or self._pairs.shape[0] != S * (S - 1) // 2:
                self._pairs = torch.tensor([(a, b) for a in range(S) for b in range(a + 1, S)],
                                           dtype=torch.long, device=U.device)

    def forward_raw(self, sky: torch.Tensor, U: torch.Tensor) -> torch.Tensor:
        self._stage(U)
        return self.plan.forward_formation(sky.contiguous())

    def adjoint_raw(self, coef: torch.Tensor, U: torch.Tensor) -> torch.Tensor:
        self._stage(U)
        return self.plan.adjoint_formation(coef.contiguous())

    def dphase(self, sky: torch.Tensor, U: torch.Tensor) -> torch.Tensor:
        """D (K, 3) complex: sum_j I_j vis_kj s_jc exp(-2 pi i u_k . s_j)."""
        self._stage(U)
        sky64 = sky.to(torch.float64)
        return torch.stack([self.plan.forward_formation((sky64 * self.lmn[:, c]).to(torch.float32).contiguous())
                            for c in range(3)], dim=1)

    def pair_to_satellites(self, grad_u: torch.Tensor, T: int, S: int) -> torch.Tensor:
        """(T*B, 3) gradient w.r.t. u_ab = U_a - U_b -> (T, S, 3) w.r.t. U."""
        gu = grad_u.view(T, -1, 3)
        gU = torch.zeros((T, S, 3), dtype=gu.dtype, device=gu.device)
        gU.index_add_(1, self._pairs[:, 0], gu)
        gU.index_add_(1, self._pairs[:, 1], -gu)
        return gU

    def __call__(self, sky: torch.Tensor, U: torch.Tensor) -> torch.Tensor:
        return _FormationVisibility.apply(sky, U, self)


class _FormationVisibility(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sky, U, model: FormationModel):
        ctx.model = model
        ctx.save_for_backward(sky, U)
        return model.forward_raw(sky.detach().to(torch.float32), U.detach().to(torch.float64))

    @staticmethod
    def backward(ctx, g):
        sky, U = ctx.saved_tensors
        m = ctx.model
        g = g.to(torch.complex64).contiguous()
        Ud = U.detach().to(torch.float64)
        grad_sky = grad_U = None
        if ctx.needs_input_grad[0]:
            grad_sky = m.adjoint_raw(g, Ud).to(sky.dtype)
        if ctx.needs_input_grad[1]:
            D = m.dphase(sky.detach().to(torch.float32), Ud)
            grad_u = (-2.0 * math.pi) * (g.to(torch.complex128)[:, None] * D.conj().to(torch.complex128)).imag
            grad_U = m.pair_to_satellites(grad_u, U.shape[0], U.shape[1]).to(U.dtype)
        return grad_sky, grad_U, None
