"""The reference's production operating point at 1 MHz: HEALPix Nside 512
(3,145,728 pixels, healpix3d_blockage.ipynb:29) and one day of up to
4,000,000 rows (vissgen3d_blockage.cu:28), i.e. 2,000,160 unique samples once
the mirror rows are folded (45 baselines x 44,448 snapshots), Moon + Earth.

At this size the pixel records (100 MB) no longer fit the 126 MB L2 beside
the samples, and the launch grids reach their largest shapes (thousands of
sample blocks, the adjoint's channel x chunk grid).  Checked here:
  - the plan builds and both kernels launch at this size (no grid or
    workspace limit is hit), and no bounded device-side wait gives up;
  - the integer identity of the culling (zero baselines, unit sky):
    round(Re V_k) = visible pixels of sample k on a seeded subset of 8,192
    samples, and round(image_j) = samples that see pixel j on a seeded subset
    of 4,096 pixels (over all 2,000,160 samples), against viss_mask_bits;
  - the split path against the FP64 oracle (rel-L2 <= 1e-5) on a seeded
    subset of samples (forward, all pixels) and of pixels (adjoint, all
    samples).
"""
import numpy as np
import pytest
import torch

from viss_optimize_3d_b200 import api, pipeline, synth

pytestmark = pytest.mark.gpu

TOL_SPLIT = 1e-5


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def np64(t):
    t = t.detach().cpu()
    return t.numpy().astype(np.complex128) if t.is_complex() else t.numpy().astype(np.float64)


def _popcount_rows(bits_u8):
    r = torch.zeros(bits_u8.shape[0], dtype=torch.int64, device=bits_u8.device)
    for b in range(8):
        r += torch.bitwise_and(torch.bitwise_right_shift(bits_u8, b), 1).sum(dim=1, dtype=torch.int64)
    return r


def _popcount_cols(bits_u8, J):
    cols = torch.zeros(J, dtype=torch.int64, device=bits_u8.device)
    for b in range(8):
        cols[b::8] += torch.bitwise_and(torch.bitwise_right_shift(bits_u8, b), 1).sum(
            dim=0, dtype=torch.int64)[: (J - b + 7) // 8]
    return cols


@pytest.fixture(scope="module")
def prod(viss, cuda_device):
    cfg = synth.CONFIGS["prod_1mhz"]
    obs = synth.make_observation(cfg)
    return obs, pipeline.upload(obs, cfg.freqs_hz[0], device=cuda_device)


def test_production_size_counts_exact(prod, viss, cuda_device):
    obs, g = prod
    K, J = g.plan.K, g.plan.J
    assert (K, J) == (2000160, 3145728)
    plan0 = api.Plan(g.lmn, torch.zeros_like(g.uvw), None, g.refs, g.occ)
    V = plan0.forward(torch.ones(J, dtype=torch.float32, device=cuda_device))
    plan0.last_stats()
    img = plan0.adjoint(torch.ones(K, dtype=torch.complex64, device=cuda_device))
    plan0.last_stats()
    rng = np.random.default_rng(31)
    ks = torch.as_tensor(np.sort(rng.choice(K, 8192, replace=False)), device=cuda_device)
    rows = _popcount_rows(viss.mask_bits(g.lmn, g.refs[ks], g.occ).view(torch.uint8))
    n_fwd = torch.round(V.real.double()[ks]).long()
    assert torch.equal(n_fwd, rows), int((n_fwd != rows).sum())
    js = torch.as_tensor(np.sort(rng.choice(J, 4096, replace=False)), device=cuda_device)
    cols = torch.zeros(js.numel(), dtype=torch.int64, device=cuda_device)
    lmn_sel = g.lmn[js].contiguous()
    for k0 in range(0, K, 262144):
        bits = viss.mask_bits(lmn_sel, g.refs[k0:k0 + 262144], g.occ).view(torch.uint8)
        cols += _popcount_cols(bits, js.numel())
    n_adj = torch.round(img.double()[js]).long()
    assert torch.equal(n_adj, cols), int((n_adj != cols).sum())
    assert 0 < int(rows.min()) and int(rows.max()) < J


def test_production_size_split_accuracy(prod, oracle):
    obs, g = prod
    lmn, uvw, sky = np64(g.lmn), np64(g.uvw), np64(g.sky)
    occ = oracle.occulters(obs.occ_sat_positions, synth.R_MOON, 0)
    occ = np.concatenate([occ, obs.earth_rows])
    np.testing.assert_array_equal(np64(g.occ), occ)
    rng = np.random.default_rng(32)
    ks = np.sort(rng.choice(obs.cfg.n_samples, 48, replace=False))
    Vs = np64(g.plan.forward(g.sky))[ks]
    g.plan.last_stats()
    Vo = oracle.forward(uvw[ks], lmn, sky, obs.refs[ks], occ)
    assert rel_l2(Vs, Vo) <= TOL_SPLIT, rel_l2(Vs, Vo)
    js = np.sort(rng.choice(obs.cfg.npix, 24, replace=False))
    a = (rng.standard_normal(g.plan.K) + 1j * rng.standard_normal(g.plan.K)).astype(np.complex64)
    Cs = np64(g.plan.adjoint(torch.as_tensor(a, device=g.lmn.device)))[js]
    g.plan.last_stats()
    Co = oracle.adjoint(uvw, a.astype(np.complex128), lmn[js], obs.refs, occ)
    assert rel_l2(Cs, Co) <= TOL_SPLIT, rel_l2(Cs, Co)


# ------------------------------------------- the 10 MHz production limits
# The reference's 10 MHz operating point is HEALPix Nside 4096 (201,326,592
# pixels, healpix3d_blockage_10Mhz.ipynb:29) and up to 40,000,000 rows a day
# (vissgen3d_blockage_10m.cu:28), i.e. 2e7 unique samples.  One full pass is
# 4e15 terms (about half an hour on one B200), so each axis is exercised at its
# full length separately: all 201,326,592 pixels with 2,048 samples, and
# 20,000,025 samples with Nside 64.  Both run the plan set-up, the largest
# grids (196,608 adjoint CTAs; 19,532 forward sample blocks) and the culling,
# and check the integer visible-count identity (zero baselines, unit sky)
# against viss_mask_bits.

def _counts_identity(viss, lmn, refs, occ, dev, k_check, j_check):
    """The visible-count identity along both axes.  V and the image are FP32,
    which holds integers exactly only below 2^24, so the unit sky (and the
    unit coefficients) are split into slices of fewer than 2^24 pixels
    (samples); each slice's count is then exact and the slices are summed."""
    K, J = refs.shape[0], lmn.shape[0]
    lim = (1 << 24) - 1
    plan0 = api.Plan(lmn, torch.zeros((K, 3), dtype=torch.float64, device=dev), None, refs, occ)
    n_fwd = torch.zeros(K, dtype=torch.int64, device=dev)
    for j0 in range(0, J, lim):
        sky = torch.zeros(J, dtype=torch.float32, device=dev)
        sky[j0:j0 + lim] = 1.0
        n_fwd += torch.round(plan0.forward(sky).real.double()).long()
        plan0.last_stats()
    n_adj = torch.zeros(J, dtype=torch.int64, device=dev)
    for k0 in range(0, K, lim):
        coef = torch.zeros(K, dtype=torch.complex64, device=dev)
        coef[k0:k0 + lim] = 1.0
        n_adj += torch.round(plan0.adjoint(coef).double()).long()
        plan0.last_stats()
    # samples: popcounts of their full rows, 64 at a time
    n_rows = []
    for i in range(0, k_check.numel(), 64):
        sel = k_check[i:i + 64]
        n_rows.append(_popcount_rows(viss.mask_bits(lmn, refs[sel], occ).view(torch.uint8)))
    rows = torch.cat(n_rows)
    assert torch.equal(n_fwd[k_check], rows), int((n_fwd[k_check] != rows).sum())
    # pixels: popcounts over all samples of the checked pixels
    lmn_sel = lmn[j_check].contiguous()
    cols = torch.zeros(j_check.numel(), dtype=torch.int64, device=dev)
    for k0 in range(0, K, 1 << 20):
        cols += _popcount_cols(viss.mask_bits(lmn_sel, refs[k0:k0 + (1 << 20)], occ).view(torch.uint8),
                               j_check.numel())
    assert torch.equal(n_adj[j_check], cols), int((n_adj[j_check] != cols).sum())
    del plan0


def test_10mhz_production_pixel_axis(viss, cuda_device):
    import dataclasses
    cfg = dataclasses.replace(synth.CONFIGS["c3_10mhz"], n_snap=8640)
    obs = synth.make_observation(cfg)
    # 2,048 samples spread over the orbit (every 190th): many occultation states
    ks = np.arange(0, cfg.n_samples, 190)[:2048]
    refs = torch.as_tensor(obs.refs[ks], device=cuda_device)
    occ = pipeline.build_occulters(obs, cuda_device)
    lmn = viss.pix2lmn(4096, "ring", device=cuda_device)
    assert lmn.shape[0] == 201326592
    rng = np.random.default_rng(41)
    k_check = torch.as_tensor(np.sort(rng.choice(len(ks), 256, replace=False)), device=cuda_device)
    j_check = torch.as_tensor(np.sort(rng.choice(lmn.shape[0], 8192, replace=False)), device=cuda_device)
    _counts_identity(viss, lmn, refs, occ, cuda_device, k_check, j_check)


def test_10mhz_production_sample_axis(viss, cuda_device):
    import dataclasses
    cfg = dataclasses.replace(synth.CONFIGS["c3_10mhz"], nside=64, n_snap=444445)
    obs = synth.make_observation(cfg)
    assert cfg.n_samples == 20000025
    refs = torch.as_tensor(obs.refs, device=cuda_device)
    occ = pipeline.build_occulters(obs, cuda_device)
    lmn = viss.pix2lmn(64, "ring", device=cuda_device)
    rng = np.random.default_rng(42)
    k_check = torch.as_tensor(np.sort(rng.choice(cfg.n_samples, 4096, replace=False)), device=cuda_device)
    j_check = torch.as_tensor(np.sort(rng.choice(lmn.shape[0], 1024, replace=False)), device=cuda_device)
    _counts_identity(viss, lmn, refs, occ, cuda_device, k_check, j_check)
