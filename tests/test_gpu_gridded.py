"""The gridded (per-facet type-3 NUFFT) imaging adjoint, viss_adjoint_gridded.

It evaluates the unmasked adjoint of the reference's noblockage programs
(computeC, vissgen3d_noblockage.cu:167-182),

  image_j = scale * sum_k Re(coef_k exp(+2 pi i (u_k.s_j + off_k))),

and must equal viss_adjoint with VISS_NO_MASK (the direct sum) to rel-L2
<= 1e-5, the split path's bound, for every facet size, with phase offsets and
VISS_ACCUMULATE; the gridded image is also checked against the FP64 oracle on
a pixel subset.  The occulted adjoint (computeC of the blockage programs,
vissgen3d_blockage.cu:167-192) is a hybrid: pairs whose facet the sample sees
wholly are gridded, the rest go through the direct kernel.  It must equal
viss_adjoint to the same bound, and with zero baselines and unit
coefficients round(image_j) must be exactly the number of samples that see
pixel j (the popcounts of viss_mask_bits): a pair counted by both parts, or
by neither, would show.  Grids beyond the size limit are refused.
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
    grid = g.plan.adjoint_gridded(a, scale=2.0, mask=False, facet_pixels=facet)
    info = g.plan.gridded_info()
    assert rel(grid, direct) <= TOL, (facet, rel(grid, direct), info)
    assert info["facet_pixels"] == (facet or info["facet_pixels"]) and min(info["grid"]) >= 16


def test_gridded_against_the_fp64_oracle(c1, oracle, cuda_device):
    obs, g = c1
    a = _coef(g.plan.K, cuda_device, seed=5)
    grid = g.plan.adjoint_gridded(a, mask=False).cpu().numpy().astype(np.float64)
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
    """A sky too coarse for its baselines (Nside 8 at 10 MHz: no facet keeps
    the grid under its limit) returns VISS_ERR_ARG, occulted or not; so do an
    explicit facet too large for the grid and, on an occulted plan, a facet
    that is not a multiple of 256 records.  At 0.1 MHz the same plan images;
    a NaN coefficient returns VISS_ERR_NOTFINITE."""
    from viss_optimize_3d_b200 import _capi
    cfg = synth.scaled(synth.CONFIGS["c2"], nside=8, n_snap=16)
    obs = synth.make_observation(cfg)
    g = pipeline.upload(obs, 1e7, device=cuda_device)
    a = _coef(g.plan.K, cuda_device)
    img = torch.empty(g.plan.J, dtype=torch.float32, device=cuda_device)
    for flags in (0, _capi.VISS_NO_MASK):                   # occulted (hybrid) and unmasked
        st = _capi.lib.viss_adjoint_gridded(g.plan._h, C.c_void_p(a.data_ptr()), C.c_void_p(img.data_ptr()),
                                            1.0, flags, 0, C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert st == _capi.VISS_ERR_ARG and "no facet size" in _capi.last_error()
    # occulted plans take facets of whole direct-kernel warp tiles
    with pytest.raises(_capi.VissError, match="multiple of 256") as ei:
        g.plan.adjoint_gridded(a, facet_pixels=64)
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
    grid = g.plan.adjoint_gridded(a, mask=False)
    assert rel(grid, g.plan.adjoint(a, mask=False)) <= TOL
    # a non-finite coefficient is reported, not spread
    bad = a.clone()
    bad[5] = complex(float("nan"), 0.0)
    with pytest.raises(_capi.VissError, match="non-finite") as ei:
        g.plan.adjoint_gridded(bad, mask=False)
    assert ei.value.status == _capi.VISS_ERR_NOTFINITE
    grid = g.plan.adjoint_gridded(a, mask=False)           # the plan is usable again
    assert rel(grid, g.plan.adjoint(a, mask=False)) <= TOL


@pytest.fixture(scope="module")
def c3_small(viss, cuda_device):
    """The C3 geometry at 1 MHz, scaled: Nside 128 (196,608 px) x 48,600
    samples (45 baselines x 1,080 snapshots), Moon + Earth occultation."""
    cfg = synth.scaled(synth.CONFIGS["c3_1mhz"], nside=128, n_snap=1080)
    obs = synth.make_observation(cfg)
    return obs, pipeline.upload(obs, 1e6, device=cuda_device)


def test_gridded_occulted_matches_direct(c3_small, cuda_device):
    obs, g = c3_small
    a = _coef(g.plan.K, cuda_device, seed=13)
    direct = g.plan.adjoint(a, scale=2.0)
    for facet in (256, 1024, 0):
        grid = g.plan.adjoint_gridded(a, scale=2.0, facet_pixels=facet)
        assert rel(grid, direct) <= TOL, (facet, rel(grid, direct), g.plan.gridded_info())
        g.plan.last_stats()                                  # no bounded wait of the direct part gave up
    # with phase offsets and VISS_ACCUMULATE
    gen = torch.Generator(device=cuda_device).manual_seed(17)
    off = torch.rand(g.plan.K, dtype=torch.float64, device=cuda_device, generator=gen) * 4 - 2
    plan = api.Plan(g.lmn, g.uvw, off, g.refs, g.occ)
    direct = plan.adjoint(a)
    base = torch.rand(plan.J, device=cuda_device, generator=gen)
    acc = base.clone()
    plan.adjoint_gridded(a, out=acc, accumulate=True)
    assert rel(acc - base, direct) <= TOL


def test_gridded_occulted_counts_exact(c3_small, viss, cuda_device):
    """Zero baselines, unit coefficients: every pixel's count of the samples
    that see it, exactly, for each facet size."""
    obs, g = c3_small
    K, J = g.plan.K, g.plan.J
    cols = torch.zeros(J, dtype=torch.int64, device=cuda_device)
    for k0 in range(0, K, 8192):
        by = viss.mask_bits(g.lmn, g.refs[k0:k0 + 8192], g.occ).view(torch.uint8)
        for b in range(8):
            plane = torch.bitwise_and(torch.bitwise_right_shift(by, b), 1)
            cols[b::8] += plane.sum(dim=0, dtype=torch.int64)[: (J - b + 7) // 8]
    assert 0 < int((cols < K).sum()) < J and int(cols.max()) == K   # occulted for part of the samples
    plan0 = api.Plan(g.lmn, torch.zeros_like(g.uvw), None, g.refs, g.occ)
    ones = torch.ones(K, dtype=torch.complex64, device=cuda_device)
    for facet in (256, 1024, 4096):
        img = plan0.adjoint_gridded(ones, facet_pixels=facet)
        n = torch.round(img.double()).long()
        bad = torch.nonzero(n != cols).flatten()
        assert bad.numel() == 0, (facet, bad[:10].tolist(), img[bad[:10]].tolist(), cols[bad[:10]].tolist())
        assert float((img.double() - cols.double()).abs().max()) < 0.3


def test_pipeline_observe_gridded(c3_small):
    """pipeline.observe(gridded=True): the same visibilities, the dirty image
    through the gridded adjoint within 1e-5 of the direct one."""
    obs, g = c3_small
    V, img = pipeline.observe(g)
    V2, img2 = pipeline.observe(g, gridded=True)
    assert torch.equal(V, V2)
    assert rel(img2, img) <= TOL
    with pytest.raises(ValueError):
        pipeline.observe(g, fp64=True, gridded=True)


def test_gridded_repeated_calls_and_restaged_samples(c3_small, cuda_device):
    """What a call derives from the geometry alone (facet size, |u| bound,
    sample order, mixed-pair bits) is kept for the next call on the same plan:
    repeated calls with new coefficients, and a call after the samples were
    staged again (other baselines), all match the direct adjoint."""
    obs, g = c3_small
    plan = api.Plan(g.lmn, g.uvw, None, g.refs, g.occ)
    for seed in (21, 22, 23):
        a = _coef(plan.K, cuda_device, seed=seed)
        for mask in (True, False, True):
            grid = plan.adjoint_gridded(a, mask=mask)
            assert rel(grid, plan.adjoint(a, mask=mask)) <= TOL, (seed, mask)
    first = plan.gridded_info()
    plan.set_samples(g.uvw * 0.5, None, g.refs, g.occ)        # shorter baselines: another grid
    a = _coef(plan.K, cuda_device, seed=24)
    grid = plan.adjoint_gridded(a)
    assert rel(grid, plan.adjoint(a)) <= TOL
    assert plan.gridded_info()["grid"] != first["grid"]
