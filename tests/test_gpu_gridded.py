"""The gridded (per-facet type-3 NUFFT) imaging adjoint, viss_adjoint_gridded.

It evaluates the unmasked adjoint of the reference's noblockage programs
(computeC, vissgen3d_noblockage.cu:167-182),

  image_j = scale * sum_k Re(coef_k exp(+2 pi i (u_k.s_j + off_k))),

and must equal viss_adjoint with VISS_NO_MASK (the direct sum) to rel-L2
<= 1e-5, the split path's bound, for every facet size, with phase offsets and
VISS_ACCUMULATE; the gridded image is also checked against the FP64 oracle on
a pixel subset.  The occulted adjoint has no gridded form: a plan with
occulter refs is refused unless VISS_NO_MASK is passed, and so are grids
beyond the size limit.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from viss_optimize_3d_b200 import api, pipeline, synth

pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel(a, b):
    a, b = a.double(), b.double()
    return (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()


@pytest.fixture(scope="module")
def c1(viss, cuda_device):
    obs = synth.make_observation(synth.CONFIGS["c1"])            # Nside 32, 1 MHz, 10,080 samples
    return obs, pipeline.upload(obs, 1e6, device=cuda_device)


def _coef(K, dev, seed=3):
    g = torch.Generator(device=dev).manual_seed(seed)
    return torch.complex(torch.randn(K, device=dev, generator=g), torch.randn(K, device=dev, generator=g))


@pytest.mark.parametrize("facet", [16, 64, 0])
def test_gridded_matches_direct_unmasked(c1, cuda_device, facet):
    """C1 (Nside 32, |u| up to 422 wavelengths): facets of up to 64 records
    keep the grid under its limit; 0 lets the library choose."""
    obs, g = c1
    a = _coef(g.plan.K, cuda_device)
    direct = g.plan.adjoint(a, scale=2.0, mask=False)
    grid = g.plan.adjoint_gridded(a, scale=2.0, facet_pixels=facet)
    info = g.plan.gridded_info()
    assert rel(grid, direct) <= TOL, (facet, rel(grid, direct), info)
    assert info["facet_pixels"] == (facet or info["facet_pixels"]) and min(info["grid"]) >= 16


def test_gridded_against_the_fp64_oracle(c1, oracle, cuda_device):
    obs, g = c1
    a = _coef(g.plan.K, cuda_device, seed=5)
    grid = g.plan.adjoint_gridded(a).cpu().numpy().astype(np.float64)
    js = np.sort(np.random.default_rng(2).choice(g.plan.J, 64, replace=False))
    lmn, uvw = g.lmn.cpu().numpy(), g.uvw.cpu().numpy()
    Co = oracle.adjoint(uvw, a.cpu().numpy().astype(np.complex128), lmn[js])
    assert np.linalg.norm(grid[js] - Co) / np.linalg.norm(Co) <= TOL


def test_gridded_offsets_accumulate_and_a_finer_grid(viss, cuda_device):
    """Phase offsets and VISS_ACCUMULATE on a finer grid (Nside 128 at 1 MHz,
    45 baselines x 1,080 snapshots), facets of 256 and 1,024 records and the
    library's choice."""
    cfg = synth.scaled(synth.CONFIGS["c3_1mhz"], nside=128, n_snap=1080)
    obs = synth.make_observation(cfg)
    lmn = api.pix2lmn(cfg.nside, "ring", device=cuda_device)
    uvw = torch.as_tensor(obs.uvw(1e6), device=cuda_device)
    gen = torch.Generator(device=cuda_device).manual_seed(7)
    off = torch.rand(uvw.shape[0], dtype=torch.float64, device=cuda_device, generator=gen) * 4 - 2
    plan = api.Plan(lmn, uvw, off)
    a = _coef(plan.K, cuda_device, seed=9)
    direct = plan.adjoint(a, scale=0.5)
    for facet in (256, 1024, 0):
        grid = plan.adjoint_gridded(a, scale=0.5, facet_pixels=facet)
        assert rel(grid, direct) <= TOL, (facet, rel(grid, direct), plan.gridded_info())
    base = torch.rand(plan.J, device=cuda_device, generator=gen)
    acc = base.clone()
    plan.adjoint_gridded(a, scale=0.5, out=acc, accumulate=True)
    assert rel(acc - base, direct) <= TOL
    no_off = plan.adjoint_gridded(a, scale=0.5, use_offset=False)
    assert rel(no_off, plan.adjoint(a, scale=0.5, use_offset=False)) <= TOL


def test_gridded_refusals(viss, cuda_device):
    """A plan with occulter refs is imaged through the gridded path only with
    VISS_NO_MASK; without it the call returns VISS_ERR_ARG.  So does a sky
    too coarse for its baselines (Nside 8 at 10 MHz: no facet, down to 64
    records, keeps the grid under its limit) and an explicit facet too large
    for the grid.  At 0.1 MHz the same occulted plan images with VISS_NO_MASK;
    a NaN coefficient returns VISS_ERR_NOTFINITE."""
    from viss_optimize_3d_b200 import _capi
    cfg = synth.scaled(synth.CONFIGS["c2"], nside=8, n_snap=16)
    obs = synth.make_observation(cfg)
    g = pipeline.upload(obs, 1e7, device=cuda_device)
    a = _coef(g.plan.K, cuda_device)
    img = torch.empty(g.plan.J, dtype=torch.float32, device=cuda_device)
    st = _capi.lib.viss_adjoint_gridded(g.plan._h, C.c_void_p(a.data_ptr()), C.c_void_p(img.data_ptr()), 1.0,
                                        0, 0, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _capi.VISS_ERR_ARG and "unmasked" in _capi.last_error()
    with pytest.raises(_capi.VissError, match="no facet size") as ei:
        g.plan.adjoint_gridded(a)                          # VISS_NO_MASK
    assert ei.value.status == _capi.VISS_ERR_ARG
    # one facet over the whole C1 sky (Nside 32, |u| to 422 wavelengths) would
    # need a grid of ~3e11 points
    c1obs = synth.make_observation(synth.CONFIGS["c1"])
    plan1 = api.Plan(api.pix2lmn(32, "ring", device=cuda_device),
                     torch.as_tensor(c1obs.uvw(1e6), device=cuda_device))
    with pytest.raises(_capi.VissError, match="above the limit") as ei:
        plan1.adjoint_gridded(_coef(plan1.K, cuda_device), facet_pixels=12288)
    assert ei.value.status == _capi.VISS_ERR_ARG
    g = pipeline.upload(obs, 1e5, device=cuda_device)
    grid = g.plan.adjoint_gridded(a)                       # VISS_NO_MASK
    assert rel(grid, g.plan.adjoint(a, mask=False)) <= TOL
    # a non-finite coefficient is reported, not spread
    bad = a.clone()
    bad[5] = complex(float("nan"), 0.0)
    with pytest.raises(_capi.VissError, match="non-finite") as ei:
        g.plan.adjoint_gridded(bad)
    assert ei.value.status == _capi.VISS_ERR_NOTFINITE
    grid = g.plan.adjoint_gridded(a)                       # the plan is usable again
    assert rel(grid, g.plan.adjoint(a, mask=False)) <= TOL
