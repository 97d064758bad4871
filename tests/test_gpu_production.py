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
