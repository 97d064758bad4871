"""Oracle pins for the visibility / imaging arithmetic (CPU).

The C oracle (oracle/viss_oracle.c) is checked against an independent numpy
restatement of the reference kernels on small seeded cases:
forward (vissgen3d_blockage.cu:76-102), adjoint (:167-192), the shell
histogram and DCF (:105-130, vissgen3d_noblockage.cu:132-141), dg and the
weight clamp (:144-164, :178, :187), the w-rotation (:150-151) and the
occultation predicate (:88-94, constants :249-252).
"""
import math

import numpy as np
import pytest


def _rand_unit(rng, n):
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _np_forward(uvw, lmn, I, vis, off):
    ph = uvw @ lmn.T + off[:, None]
    return ((I[None, :] * vis) * np.exp(-2j * np.pi * ph)).sum(axis=1)


def _np_adjoint(uvw, a, lmn, vis, off):
    ph = uvw @ lmn.T + off[:, None]
    return np.real(a[:, None] * vis * np.exp(2j * np.pi * ph)).sum(axis=0)


@pytest.fixture(scope="module")
def case():
    rng = np.random.default_rng(7)
    K, J, G = 37, 53, 6
    lmn = _rand_unit(rng, J)
    uvw = rng.uniform(-300, 300, (K, 3))
    off = rng.uniform(-2, 2, K)
    I = rng.uniform(0, 2, J)
    occ = np.concatenate([_rand_unit(rng, G), rng.uniform(-0.6, 0.2, (G, 1))], axis=1)
    refs = rng.integers(-1, G, (K, 3)).astype(np.int32)
    return dict(K=K, J=J, lmn=lmn, uvw=uvw, off=off, I=I, occ=occ, refs=refs)


def _np_vis(case):
    d = case["lmn"] @ case["occ"][:, :3].T          # (J, G)
    ok = d >= case["occ"][None, :, 3]
    vis = np.ones((case["K"], case["J"]), bool)
    for c in range(3):
        g = case["refs"][:, c]
        sel = g >= 0
        vis[sel] &= ok[:, g[sel]].T
    return vis


def test_mask_matches_numpy_predicate(oracle, case):
    bits = oracle.mask_bits(case["lmn"], case["refs"], case["occ"])
    J = case["J"]
    got = np.unpackbits(bits.view(np.uint8), axis=1, bitorder="little")[:, :J].astype(bool)
    exp = _np_vis(case)
    # numpy's dot has no fma; only exact-boundary pixels could differ
    d = case["lmn"] @ case["occ"][:, :3].T
    margin = np.abs(d - case["occ"][None, :, 3]).min()
    assert margin > 1e-12
    np.testing.assert_array_equal(got, exp)


def test_forward_matches_numpy(oracle, case):
    vis = _np_vis(case)
    V = oracle.forward(case["uvw"], case["lmn"], case["I"], case["refs"], case["occ"], case["off"])
    Vn = _np_forward(case["uvw"], case["lmn"], case["I"], vis, case["off"])
    np.testing.assert_allclose(V, Vn, rtol=1e-11, atol=1e-11)
    # no mask, no offset
    V0 = oracle.forward(case["uvw"], case["lmn"], case["I"])
    np.testing.assert_allclose(V0, _np_forward(case["uvw"], case["lmn"], case["I"], True,
                                               np.zeros(case["K"])), rtol=1e-11, atol=1e-11)


def test_adjoint_matches_numpy_and_is_adjoint(oracle, case):
    rng = np.random.default_rng(3)
    a = rng.standard_normal(case["K"]) + 1j * rng.standard_normal(case["K"])
    vis = _np_vis(case)
    C = oracle.adjoint(case["uvw"], a, case["lmn"], case["refs"], case["occ"], case["off"])
    np.testing.assert_allclose(C, _np_adjoint(case["uvw"], a, case["lmn"], vis, case["off"]),
                               rtol=1e-11, atol=1e-11)
    # <x, A^H a> = Re <A x, a>
    x = case["I"]
    V = oracle.forward(case["uvw"], case["lmn"], x, case["refs"], case["occ"], case["off"])
    lhs = float(np.dot(x, C))
    rhs = float(np.real(np.sum(a * np.conj(V))))
    assert abs(lhs - rhs) <= 1e-11 * max(1.0, abs(lhs))


def test_forward_dphase_is_derivative(oracle, case):
    uvw, lmn, I = case["uvw"], case["lmn"], case["I"]
    D = oracle.forward_dphase(uvw, lmn, I)
    h = 1e-6
    for c in range(3):
        du = np.zeros_like(uvw)
        du[:, c] = h
        Vp = oracle.forward(uvw + du, lmn, I)
        Vm = oracle.forward(uvw - du, lmn, I)
        fd = (Vp - Vm) / (2 * h)
        np.testing.assert_allclose(fd, -2j * np.pi * D[:, c], rtol=1e-6, atol=1e-6)


def test_dcf_matches_numpy(oracle):
    rng = np.random.default_rng(11)
    bll = rng.uniform(0.0, 40.0, 5000).astype(np.float32)
    bll[:5] = [0.25, 0.75, 0.7500001, 1.25, np.nan]
    nr = 70
    for mult in (1, 2):
        gs, counts, dcf = oracle.dcf(bll, nr, mult)
        d = (bll - np.float32(0.25)).astype(np.float32)
        gsn = np.ceil(d * np.float32(2.0))
        gsn = np.where(np.isnan(gsn), -1, gsn).astype(np.int32)
        np.testing.assert_array_equal(gs, gsn)
        assert gs[0] == 0 and gs[1] == 1 and gs[2] == 2 and gs[4] == -1
        cn = np.bincount(gsn[(gsn >= 1) & (gsn <= nr)] - 1, minlength=nr) * mult
        np.testing.assert_array_equal(counts, cn)
        k = np.arange(1, nr + 1, dtype=np.float64)
        R = k * 0.5 + 0.25
        with np.errstate(divide="ignore"):
            exp = ((2 * math.pi / 3) * (R ** 3 - (R - 0.5) ** 3) / cn).astype(np.float32)
        np.testing.assert_allclose(dcf[1:], exp, rtol=1e-7)
        assert dcf[0] == np.float32(1 / (4 * math.pi))


def test_dg_and_weights_match_numpy(oracle):
    rng = np.random.default_rng(5)
    n = 4000
    bll = rng.uniform(0.5, 50, n).astype(np.float32)
    w = (bll * rng.uniform(-1.2, 1.2, n)).astype(np.float32)
    dg = oracle.gamma_dg(w, bll)
    x = w.astype(np.float64) / bll.astype(np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        exp = np.where(np.abs(x) < 1,
                       1.5 * np.sqrt(np.abs(1 - 4 * x * x)) / np.sqrt(1 - x * x), np.inf).astype(np.float32)
    np.testing.assert_allclose(dg, exp, rtol=1e-7)
    # the reference's trig route agrees (FP64 here)
    g = np.arcsin(np.clip(x, -1, 1))
    with np.errstate(divide="ignore"):
        ref = np.abs(np.sqrt((1 - 4 * np.sin(g) ** 2).astype(complex))) / np.abs(np.cos(g)) * 1.5
    fin = np.abs(x) < 0.999
    np.testing.assert_allclose(dg[fin], ref[fin], rtol=2e-6)
    nr = 101
    gs, _, dcf = oracle.dcf(bll, nr)
    wt = oracle.weights(gs, dg, dcf, nr)
    g2 = np.clip(gs, 0, nr)
    np.testing.assert_array_equal(wt, np.fmin(dcf[g2] * dg, np.float32(0.125)))
    assert (wt <= 0.125).all()


def test_wrot_and_cone_threshold(oracle):
    rng = np.random.default_rng(2)
    w = rng.uniform(-500, 500, 300)
    V = rng.standard_normal(300) + 1j * rng.standard_normal(300)
    np.testing.assert_allclose(oracle.wrot(w, V), V * np.exp(-2j * np.pi * w), rtol=1e-9)
    # vissgen3d_blockage.cu:249-252: phi = pi - asin(R/(R+h)); cos(phi) = -sqrt(1-rho^2)
    thr = oracle.cone_threshold(1737.1e3, 300e3)
    rho = 1737.1e3 / 2037.1e3
    assert abs(thr + math.sqrt(1 - rho * rho)) < 1e-6


def test_occulters_ray_sphere(oracle):
    rng = np.random.default_rng(9)
    P = _rand_unit(rng, 50) * rng.uniform(1.9e6, 2.2e6, (50, 1))
    occ = oracle.occulters(P, 1737.4e3, 0)
    r = np.linalg.norm(P, axis=1)
    np.testing.assert_allclose(occ[:, :3], P / r[:, None], rtol=1e-15, atol=1e-16)
    np.testing.assert_allclose(occ[:, 3], -np.sqrt(1 - (1737.4e3 / r) ** 2), rtol=1e-14)
    # the predicate is the ray-sphere test: directions inside the Moon's disc are hidden
    s = _rand_unit(rng, 2000)
    for i in range(5):
        p = P[i]
        tca = s @ p                                     # along-ray distance of closest approach (neg)
        d2 = (p @ p) - tca ** 2
        hits = (tca < 0) & (d2 < 1737.4e3 ** 2)
        vis = (s @ occ[i, :3]) >= occ[i, 3]
        near = np.abs(d2 - 1737.4e3 ** 2) < 1e3
        np.testing.assert_array_equal(vis[~near], ~hits[~near])
