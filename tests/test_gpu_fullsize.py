"""Mask exactness at the headline size, through the culling kernels.

The forward and adjoint kernels never evaluate the occultation predicate for
most terms: they classify 128-pixel tiles (and 8-tile super-tiles, 32-pixel
sub-tiles) against each sample's occulter rows in FP32 with a conservative
margin, skip hidden tiles, run visible ones without a test, and apply the
exact FP64 predicate (vissgen3d_blockage.cu:88-94, :180-186) only where the
classification is undecided.  A wrongly culled pixel moves one visibility by
~1/J relative, far inside the 1e-5 accuracy bound, so accuracy tests cannot
see it.  An integer identity can: with every baseline zero and a unit sky,

  forward   round(Re V_k)   = number of pixels sample k sees
  adjoint   round(image_j)  = number of samples that see pixel j  (coef = 1)

exactly, for all 388,800 samples and all 786,432 pixels of the C3
configuration (Nside 256, 45 baselines x 8,640 snapshots, Moon + Earth), and
both must equal the popcounts of viss_mask_bits (the plain predicate, pinned
to the FP64 oracle on a seeded subset here).  The occultation geometry does
not depend on the frequency, so one pass covers the 1 MHz and the 10 MHz
configurations (asserted: their occulter tables are identical); their
frequency-dependent accuracy is checked against the oracle on subsets.
"""
import numpy as np
import pytest
import torch

from viss_optimize_3d_b200 import pipeline, synth

pytestmark = pytest.mark.gpu

TOL_SPLIT = 1e-5


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def np64(t):
    t = t.detach().cpu()
    return t.numpy().astype(np.complex128) if t.is_complex() else t.numpy().astype(np.float64)


def _oracle_occ(obs, oracle):
    occ = oracle.occulters(obs.occ_sat_positions, synth.R_MOON, 0)
    if obs.earth_rows is not None:
        occ = np.concatenate([occ, obs.earth_rows])
    return occ


@pytest.fixture(scope="module")
def c3_pair(viss, cuda_device):
    """Both C3 configurations on the device."""
    out = {}
    for name, f in (("c3_10mhz", 1e7), ("c3_1mhz", 1e6)):
        obs = synth.make_observation(synth.CONFIGS[name])
        out[name] = (obs, pipeline.upload(obs, f, device=cuda_device))
    return out


def _mask_popcounts(viss, lmn, refs, occ, chunk=8192):
    """(visible pixels per sample, visible samples per pixel) from
    viss_mask_bits, in chunks of samples; bit j of a row is pixel j."""
    K, J = refs.shape[0], lmn.shape[0]
    rows = torch.empty(K, dtype=torch.int64, device=lmn.device)
    cols = torch.zeros(J, dtype=torch.int64, device=lmn.device)
    for k0 in range(0, K, chunk):
        k1 = min(K, k0 + chunk)
        by = viss.mask_bits(lmn, refs[k0:k1], occ).view(torch.uint8)      # (k, J/8) bytes
        r = torch.zeros(k1 - k0, dtype=torch.int64, device=lmn.device)
        for b in range(8):
            plane = torch.bitwise_and(torch.bitwise_right_shift(by, b), 1)
            r += plane.sum(dim=1, dtype=torch.int64)
            cols[b::8] += plane.sum(dim=0, dtype=torch.int64)[: (J - b + 7) // 8]
        rows[k0:k1] = r
    return rows, cols


def test_c3_visible_counts_exact(c3_pair, viss, oracle, cuda_device):
    obs10, g = c3_pair["c3_10mhz"]
    obs1, g1 = c3_pair["c3_1mhz"]
    # the geometry of the two frequencies is the same
    assert torch.equal(g.refs, g1.refs) and torch.equal(g.occ, g1.occ)
    K, J = g.plan.K, g.plan.J
    assert (K, J) == (388800, 786432)

    # viss_mask_bits pinned to the FP64 oracle on a seeded subset of samples
    occ_o = _oracle_occ(obs10, oracle)
    np.testing.assert_array_equal(np64(g.occ), occ_o)
    sel = np.sort(np.random.default_rng(11).choice(K, 24, replace=False))
    bits = viss.mask_bits(g.lmn, g.refs[sel], g.occ).cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(bits, oracle.mask_bits(np64(g.lmn), obs10.refs[sel], occ_o))

    rows, cols = _mask_popcounts(viss, g.lmn, g.refs, g.occ)
    assert 0 < int(rows.min()) and int(rows.max()) < J     # partly occulted samples
    assert int((cols == 0).sum()) < J // 2                   # most of the sky is seen at some time

    from viss_optimize_3d_b200 import api
    plan0 = api.Plan(g.lmn, torch.zeros_like(g.uvw), None, g.refs, g.occ)
    ones = torch.ones(J, dtype=torch.float32, device=cuda_device)
    for shape in range(4):          # every launch shape of both kernels
        plan0.set_shapes(shape, shape)
        V = plan0.forward(ones)
        n_fwd = torch.round(V.real.double()).long()
        bad = torch.nonzero(n_fwd != rows).flatten()
        assert bad.numel() == 0, (shape, bad[:10].tolist(), n_fwd[bad[:10]].tolist(), rows[bad[:10]].tolist())
        img = plan0.adjoint(torch.ones(K, dtype=torch.complex64, device=cuda_device))
        n_adj = torch.round(img.double()).long()
        bad = torch.nonzero(n_adj != cols).flatten()
        assert bad.numel() == 0, (shape, bad[:10].tolist(), n_adj[bad[:10]].tolist(), cols[bad[:10]].tolist())
        plan0.last_stats()          # no bounded wait gave up

    # the formation entry points (per-satellite factoring, their own per-snapshot
    # tile classification): all satellites at one point, so every pair's
    # baseline is zero, and the same sample order as the direct entry points
    U, occ_sat, occ_snap = pipeline.formation_inputs(obs10, 1e7, device=cuda_device, occ=g.occ)
    plan0.set_formation(torch.zeros_like(U), None, occ_sat, occ_snap)
    V = plan0.forward_formation(ones)
    n_fwd = torch.round(V.real.double()).long()
    bad = torch.nonzero(n_fwd != rows).flatten()
    assert bad.numel() == 0, ("formation", bad[:10].tolist(), n_fwd[bad[:10]].tolist(), rows[bad[:10]].tolist())
    img = plan0.adjoint_formation(torch.ones(K, dtype=torch.complex64, device=cuda_device))
    n_adj = torch.round(img.double()).long()
    bad = torch.nonzero(n_adj != cols).flatten()
    assert bad.numel() == 0, ("formation", bad[:10].tolist(), n_adj[bad[:10]].tolist(), cols[bad[:10]].tolist())
    plan0.last_stats()


@pytest.mark.parametrize("name", ["c3_10mhz", "c3_1mhz"])
def test_c3_split_accuracy_on_subsets_both_frequencies(c3_pair, oracle, name):
    """Split path vs the FP64 oracle at both C3 frequencies, on a seeded
    subset of samples (forward) and of pixels (adjoint): the oracle cannot
    afford the full 3e11 terms."""
    obs, g = c3_pair[name]
    lmn, uvw, sky = np64(g.lmn), np64(g.uvw), np64(g.sky)
    occ = _oracle_occ(obs, oracle)
    rng = np.random.default_rng(21)
    ks = np.sort(rng.choice(obs.cfg.n_samples, 96, replace=False))
    Vs = np64(g.plan.forward(g.sky))[ks]
    Vo = oracle.forward(uvw[ks], lmn, sky, obs.refs[ks], occ)
    assert rel_l2(Vs, Vo) <= TOL_SPLIT, rel_l2(Vs, Vo)
    js = np.sort(rng.choice(obs.cfg.npix, 48, replace=False))
    a = (rng.standard_normal(g.plan.K) + 1j * rng.standard_normal(g.plan.K)).astype(np.complex64)
    Cs = np64(g.plan.adjoint(torch.as_tensor(a, device=g.lmn.device)))[js]
    Co = oracle.adjoint(uvw, a.astype(np.complex128), lmn[js], obs.refs, occ)
    assert rel_l2(Cs, Co) <= TOL_SPLIT, rel_l2(Cs, Co)
