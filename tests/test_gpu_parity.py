"""GPU path vs the FP64 oracle on the benchmark configurations.

Tolerances (written here, per path):
  split path (FP64 phase + turn reduction, FP32 sincos, compensated FP32
  sums, FP64 cross-block sum):  rel-L2 <= 1e-5 vs the FP64 oracle
  plain FP64 path (complex64 output): rel-L2 <= 1e-7
  masks, shell indices, histogram counts, DCF table, dg, weights,
  occulter rows: bit-exact.
Replaces / checks: healpix_moonback_viss (vissgen3d_blockage.cu:76-102),
computeC (:167-192), the occultation predicate (:88-94, :180-186), the shell
pipeline (:105-141, vissgen3d_noblockage.cu:132-141) and the weights
(:144-164, :178, :187).
"""
import math

import numpy as np
import pytest
import torch

from viss_optimize_3d_b200 import pipeline, synth

pytestmark = pytest.mark.gpu

TOL_SPLIT = 1e-5
TOL_FP64 = 1e-7


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def np64(t):
    return t.detach().cpu().numpy().astype(np.float64) if t.dtype != torch.complex64 else \
        t.detach().cpu().numpy().astype(np.complex128)


def _oracle_occ(obs, oracle):
    if obs.refs is None:
        return None
    occ = oracle.occulters(obs.occ_sat_positions, synth.R_MOON, 0)
    if obs.earth_rows is not None:
        occ = np.concatenate([occ, obs.earth_rows])
    return occ


@pytest.fixture(scope="module")
def c1(viss, cuda_device):
    obs = synth.make_observation(synth.CONFIGS["c1"])
    return obs, pipeline.upload(obs, 1e6, device=cuda_device)


@pytest.fixture(scope="module")
def c2(viss, cuda_device):
    obs = synth.make_observation(synth.CONFIGS["c2"])
    return obs, pipeline.upload(obs, 1e7, device=cuda_device)


# ----------------------------------------------------------------- C1
def test_c1_forward(c1, oracle):
    obs, g = c1
    lmn, uvw, sky = np64(g.lmn), np64(g.uvw), np64(g.sky)
    Vo = oracle.forward(uvw, lmn, sky)
    Vs = np64(g.plan.forward(g.sky))
    Vd = np64(g.plan.forward(g.sky, fp64=True))
    e_s, e_d = rel_l2(Vs, Vo), rel_l2(Vd, Vo)
    assert e_s <= TOL_SPLIT, e_s
    assert e_d <= TOL_FP64, e_d
    ev, tot = g.plan.last_counts()
    assert tot == obs.cfg.n_samples * obs.cfg.npix and ev == tot   # no occultation in C1


def test_c1_adjoint_and_dirty_image(c1, oracle):
    obs, g = c1
    lmn, uvw = np64(g.lmn), np64(g.uvw)
    rng = np.random.default_rng(4)
    a = (rng.standard_normal(g.plan.K) + 1j * rng.standard_normal(g.plan.K)).astype(np.complex64)
    Co = oracle.adjoint(uvw, a.astype(np.complex128), lmn)
    Cs = np64(g.plan.adjoint(torch.as_tensor(a, device=g.lmn.device)))
    Cd = np64(g.plan.adjoint(torch.as_tensor(a, device=g.lmn.device), fp64=True))
    assert rel_l2(Cs, Co) <= TOL_SPLIT, rel_l2(Cs, Co)
    assert rel_l2(Cd, Co) <= TOL_FP64, rel_l2(Cd, Co)
    # the whole observation: forward, DCF (x2 mirror rows), weights, 2 Re adjoint
    V, img = pipeline.observe(g)
    Vo = oracle.forward(uvw, lmn, np64(g.sky))
    bll, w = np64(g.bll).astype(np.float32), np64(g.w).astype(np.float32)
    gs, counts, dcf = oracle.dcf(bll, g.nr, 2)
    wt = oracle.weights(gs, oracle.gamma_dg(w, bll), dcf, g.nr)
    img_o = 2.0 * oracle.adjoint(uvw, wt.astype(np.float64) * Vo, lmn)
    assert rel_l2(np64(img), img_o) <= TOL_SPLIT, rel_l2(np64(img), img_o)


# ----------------------------------------------------------------- C2
def test_c2_masks_bit_exact(c2, viss, oracle):
    obs, g = c2
    occ_o = _oracle_occ(obs, oracle)
    np.testing.assert_array_equal(np64(g.occ), occ_o)        # occulter rows, bit for bit
    sel = np.arange(0, obs.cfg.n_samples, 17)
    refs = obs.refs[sel]
    bits = viss.mask_bits(g.lmn, torch.as_tensor(refs, device=g.lmn.device), g.occ).cpu().numpy()
    bits_o = oracle.mask_bits(np64(g.lmn), refs, occ_o)
    np.testing.assert_array_equal(bits.view(np.uint32), bits_o)
    vis_frac = np.unpackbits(bits_o.view(np.uint8)).mean()
    assert 0.4 < vis_frac < 0.95        # the Moon does hide a good part of the sky


def test_c2_forward_with_occultation(c2, oracle):
    obs, g = c2
    lmn, uvw, sky = np64(g.lmn), np64(g.uvw), np64(g.sky)
    occ = _oracle_occ(obs, oracle)
    sel = np.arange(0, obs.cfg.n_samples, 7)
    Vo = oracle.forward(uvw[sel], lmn, sky, obs.refs[sel], occ)
    Vs = np64(g.plan.forward(g.sky))[sel]
    Vd = np64(g.plan.forward(g.sky, fp64=True))[sel]
    assert rel_l2(Vs, Vo) <= TOL_SPLIT, rel_l2(Vs, Vo)
    assert rel_l2(Vd, Vo) <= TOL_FP64, rel_l2(Vd, Vo)
    # a single wrong mask bit moves one V_k by ~1/sqrt(J) relative: per-sample check
    per = np.abs(Vs - Vo) / np.abs(Vo)
    assert per.max() < 1e-3, per.max()
    ev, tot = g.plan.last_counts()
    assert ev < tot          # culled tiles were skipped


def test_c2_adjoint_with_occultation(c2, oracle):
    obs, g = c2
    lmn, uvw = np64(g.lmn), np64(g.uvw)
    occ = _oracle_occ(obs, oracle)
    rng = np.random.default_rng(8)
    a = (rng.standard_normal(g.plan.K) + 1j * rng.standard_normal(g.plan.K)).astype(np.complex64)
    pix = np.arange(3, obs.cfg.npix, 13)
    Co = oracle.adjoint(uvw, a.astype(np.complex128), lmn[pix], obs.refs, occ)
    at = torch.as_tensor(a, device=g.lmn.device)
    Cs = np64(g.plan.adjoint(at))[pix]
    Cd = np64(g.plan.adjoint(at, fp64=True))[pix]
    assert rel_l2(Cs, Co) <= TOL_SPLIT, rel_l2(Cs, Co)
    assert rel_l2(Cd, Co) <= TOL_FP64, rel_l2(Cd, Co)


def test_cone_boundary_pixels(viss, oracle, cuda_device):
    """Occulters whose threshold is exactly a pixel's dot product (visible,
    >=) or one ulp above it (hidden): the GPU must agree bit for bit, also
    through the forward kernel's tile classification."""
    nside = 16
    lmn = viss.pix2lmn(nside, "nest", device=cuda_device)
    L = np64(lmn)
    rng = np.random.default_rng(12)
    rows = []
    for j in rng.choice(L.shape[0], 24, replace=False):
        q = rng.standard_normal(3)
        q /= np.linalg.norm(q)
        d = oracle.dots(L[j:j + 1], np.append(q, 0.0))[0]
        rows.append(np.append(q, d))
        rows.append(np.append(q, np.nextafter(d, np.inf)))
    occ = np.array(rows)
    G = occ.shape[0]
    refs = np.stack([np.arange(G), -np.ones(G), -np.ones(G)], axis=1).astype(np.int32)
    bits = viss.mask_bits(lmn, torch.as_tensor(refs, device=cuda_device),
                          torch.as_tensor(occ, device=cuda_device)).cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(bits, oracle.mask_bits(L, refs, occ))
    # through the forward: one sample per occulter, u = 0 so V_k = sum of visible sky
    uvw = np.zeros((G, 3))
    sky = rng.uniform(1, 2, L.shape[0]).astype(np.float32)
    plan = viss.Plan(lmn, uvw, None, refs, occ)
    for fp64 in (False, True):
        V = np64(plan.forward(torch.as_tensor(sky, device=cuda_device), fp64=fp64))
        Vo = oracle.forward(uvw, L, sky.astype(np.float64), refs, occ)
        np.testing.assert_allclose(V.real, Vo.real, rtol=2e-6)


# ---------------------------------------------------- DCF / weights (C3 size)
def test_dcf_and_weights_bit_exact(viss, oracle, cuda_device):
    obs = synth.make_observation(synth.CONFIGS["c3_10mhz"])
    f = 1e7
    uvw = obs.uvw(f)
    bll = np.linalg.norm(uvw, axis=1).astype(np.float32)
    w = uvw[:, 2].astype(np.float32)
    nr = obs.nr(f)
    bt = torch.as_tensor(bll, device=cuda_device)
    gs, counts, dcf = viss.dcf(bt, nr, multiplicity=2)
    ogs, ocounts, odcf = oracle.dcf(bll, nr, 2)
    np.testing.assert_array_equal(gs.cpu().numpy(), ogs)
    np.testing.assert_array_equal(counts.cpu().numpy().view(np.uint32), ocounts)
    np.testing.assert_array_equal(dcf.cpu().numpy().view(np.uint32), odcf.view(np.uint32))
    dg, wt = viss.weights(torch.as_tensor(w, device=cuda_device), bt, gs, dcf, nr)
    odg = oracle.gamma_dg(w, bll)
    np.testing.assert_array_equal(dg.cpu().numpy().view(np.uint32), odg.view(np.uint32))
    np.testing.assert_array_equal(wt.cpu().numpy().view(np.uint32),
                                  oracle.weights(ogs, odg, odcf, nr).view(np.uint32))
    # nr beyond the shared-memory histogram (global atomics path), small bll too
    gs2, c2, d2 = viss.dcf(bt, 40000)
    np.testing.assert_array_equal(c2.cpu().numpy().view(np.uint32), oracle.dcf(bll, 40000)[1])


def test_dcf_and_weights_adversarial_values(viss, oracle, cuda_device):
    """Shell edges, NaN/inf/negative/huge bll, |w| > bll, w = bll: the shell
    index, counts, DCF, dg and clamped weight stay bit-equal to the oracle
    (gs = -1 for NaN, saturated for huge values, clamped into [0, nr] when
    indexing; dg = inf where |w/bll| >= 1, capped at 1/8 by the weight)."""
    rng = np.random.default_rng(12)
    bll = rng.uniform(0.0, 40.0, 4000).astype(np.float32)
    w = (rng.uniform(-1, 1, 4000) * bll * 0.9).astype(np.float32)
    edge = np.array([0.25, 0.75, 0.7500001, 1.25, np.nan, np.inf, -np.inf, -3.0, 0.0, 1e30,
                     np.float32(2.0 ** 31), 5.0, 5.0, 5.0, 33.0], dtype=np.float32)
    wedge = np.array([0.1, 0.5, 0.2, 1.25, 0.3, 1.0, 0.0, 1.0, 0.0, 2.0, 1.0, 5.0, -6.0, np.nan,
                      -33.0], dtype=np.float32)
    bll[:edge.size], w[:edge.size] = edge, wedge
    nr = 70
    for mult in (1, 2):
        bt = torch.as_tensor(bll, device=cuda_device)
        gs, counts, dcf = viss.dcf(bt, nr, multiplicity=mult)
        ogs, ocounts, odcf = oracle.dcf(bll, nr, mult)
        np.testing.assert_array_equal(gs.cpu().numpy(), ogs)
        np.testing.assert_array_equal(counts.cpu().numpy().view(np.uint32), ocounts)
        np.testing.assert_array_equal(dcf.cpu().numpy().view(np.uint32), odcf.view(np.uint32))
        dg, wt = viss.weights(torch.as_tensor(w, device=cuda_device), bt, gs, dcf, nr)
        odg = oracle.gamma_dg(w, bll)
        np.testing.assert_array_equal(dg.cpu().numpy().view(np.uint32), odg.view(np.uint32))
        np.testing.assert_array_equal(wt.cpu().numpy().view(np.uint32),
                                      oracle.weights(ogs, odg, odcf, nr).view(np.uint32))
    assert ogs[4] == -1


def test_wrot_and_mirror(viss, oracle, cuda_device):
    rng = np.random.default_rng(6)
    n = 5000
    w = rng.uniform(-3000, 3000, n).astype(np.float32)
    V = (rng.standard_normal(2 * n) + 1j * rng.standard_normal(2 * n)).astype(np.complex64)
    Vt = torch.as_tensor(V, device=cuda_device)
    viss.wrot_(torch.as_tensor(w, device=cuda_device), Vt[:n])
    Vo = oracle.wrot(w.astype(np.float64), V[:n].astype(np.complex128))
    assert rel_l2(np64(Vt[:n]), Vo) < 1e-7
    viss.conj_mirror_(Vt, n)
    np.testing.assert_array_equal(np64(Vt[n:]), np.conj(np64(Vt[:n])))


# -------------------------------------------------------- C3, full size
@pytest.fixture(scope="module")
def c3(viss, cuda_device):
    obs = synth.make_observation(synth.CONFIGS["c3_10mhz"])
    return obs, pipeline.upload(obs, 1e7, device=cuda_device)


def test_c3_split_accuracy_on_subsets(c3, oracle):
    """Headline configuration (Nside 256, 388,800 samples, Moon + Earth):
    split path vs FP64 oracle on a seeded subset of samples (forward) and of
    pixels (adjoint) -- the oracle cannot afford the full 3e11 terms."""
    obs, g = c3
    lmn, uvw, sky = np64(g.lmn), np64(g.uvw), np64(g.sky)
    occ = _oracle_occ(obs, oracle)
    rng = np.random.default_rng(0)
    ks = np.sort(rng.choice(obs.cfg.n_samples, 96, replace=False))
    Vs = np64(g.plan.forward(g.sky))[ks]
    Vo = oracle.forward(uvw[ks], lmn, sky, obs.refs[ks], occ)
    assert rel_l2(Vs, Vo) <= TOL_SPLIT, rel_l2(Vs, Vo)
    js = np.sort(rng.choice(obs.cfg.npix, 48, replace=False))
    a = (rng.standard_normal(g.plan.K) + 1j * rng.standard_normal(g.plan.K)).astype(np.complex64)
    Cs = np64(g.plan.adjoint(torch.as_tensor(a, device=g.lmn.device)))[js]
    Co = oracle.adjoint(uvw, a.astype(np.complex128), lmn[js], obs.refs, occ)
    assert rel_l2(Cs, Co) <= TOL_SPLIT, rel_l2(Cs, Co)


def test_c3_adjoint_identity_and_linearity(c3):
    """Size-independent properties at full size: <x, A^H a> = Re <A x, a> and
    A(x + 2y) = A x + 2 A y."""
    obs, g = c3
    dev = g.lmn.device
    gen = torch.Generator(device=dev).manual_seed(1)
    a = torch.complex(torch.randn(g.plan.K, device=dev, generator=gen),
                      torch.randn(g.plan.K, device=dev, generator=gen))
    x = g.sky
    Ax = g.plan.forward(x).to(torch.complex128)
    AHa = g.plan.adjoint(a).double()
    lhs = torch.dot(x.double(), AHa).item()
    rhs = torch.real(torch.sum(a.to(torch.complex128) * torch.conj(Ax))).item()
    scale = (torch.linalg.norm(x.double()) * torch.linalg.norm(AHa)).item()   # Cauchy-Schwarz
    assert abs(lhs - rhs) <= 1e-5 * scale, (lhs, rhs, scale)
    y = torch.rand(g.plan.J, device=dev, generator=gen) * x.mean()
    lin = g.plan.forward(x + 2 * y).to(torch.complex128)
    ref = Ax + 2 * g.plan.forward(y).to(torch.complex128)
    assert (torch.linalg.norm(lin - ref) / torch.linalg.norm(ref)).item() < 1e-5
