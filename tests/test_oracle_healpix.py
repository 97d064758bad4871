"""HEALPix oracle pins (CPU).

The reference's pix2ang.cu does not produce HEALPix pixel centres (it keeps
1-based MATLAB table indexing, pix2ang.cu:109-123), so the oracle is pinned to
the published HEALPix definition (Gorski et al. 2005): known pixel centres for
Nside 1 and 2, the ring structure and equal-area layout, and the exact
NESTED <-> RING correspondence.
"""
import math

import numpy as np
import pytest


def test_nside1_known_centres(oracle):
    th, ph, xyz = oracle.pix2ang(1)
    z = np.cos(th)
    np.testing.assert_allclose(z, [2 / 3] * 4 + [0] * 4 + [-2 / 3] * 4, atol=1e-15)
    np.testing.assert_allclose(ph[:4], np.pi / 4 * np.array([1, 3, 5, 7]), rtol=1e-15)
    np.testing.assert_allclose(ph[4:8], np.pi / 2 * np.arange(4), atol=1e-15)
    np.testing.assert_allclose(ph[8:], np.pi / 4 * np.array([1, 3, 5, 7]), rtol=1e-15)
    # NESTED and RING coincide at Nside 1 (base pixel = face)
    thn, phn, _ = oracle.pix2ang(1, nest=True)
    np.testing.assert_array_equal(thn, th)
    np.testing.assert_array_equal(phn, ph)


def test_nside2_known_centres(oracle):
    th, ph, _ = oracle.pix2ang(2)
    z = np.cos(th)
    # ring 1: z = 11/12, 4 pixels at (2k+1) pi/4
    np.testing.assert_allclose(z[:4], 11 / 12, rtol=1e-15)
    np.testing.assert_allclose(ph[:4], np.pi / 4 * np.array([1, 3, 5, 7]), rtol=1e-15)
    # ring 2: z = 2/3, 8 pixels at (2k+1) pi/8
    np.testing.assert_allclose(z[4:12], 2 / 3, rtol=1e-15)
    np.testing.assert_allclose(ph[4:12], np.pi / 8 * (2 * np.arange(8) + 1), rtol=1e-15)
    # ring 3: z = 1/3, 8 pixels at k pi/4 (shifted ring)
    np.testing.assert_allclose(z[12:20], 1 / 3, rtol=1e-15)
    np.testing.assert_allclose(ph[12:20], np.pi / 4 * np.arange(8), atol=1e-15)
    # equator: z = 0, unshifted
    np.testing.assert_allclose(z[20:28], 0, atol=1e-15)
    np.testing.assert_allclose(ph[20:28], np.pi / 8 * (2 * np.arange(8) + 1), rtol=1e-15)


@pytest.mark.parametrize("nside", [1, 2, 4, 8, 16, 64])
def test_ring_structure_and_equal_area(oracle, nside):
    N = nside
    npix = 12 * N * N
    th, ph, xyz = oracle.pix2ang(N)
    z = xyz[:, 2]
    rings = [oracle.pix2ring(N, p)[0] for p in range(0, npix, max(1, npix // 997))]
    assert min(rings) >= 1 and max(rings) <= 4 * N - 1
    # pixel count per ring: 4i (caps), 4N (belt); z constant in a ring and
    # stepping so that every pixel covers 4 pi / npix (equal area)
    start = 0
    for i in range(1, 4 * N):
        n = 4 * min(i, 4 * N - i, N)
        zr = z[start:start + n]
        assert np.ptp(zr) < 1e-15
        if i < N:
            zexp = 1 - i * i / (3 * N * N)
        elif i <= 3 * N:
            zexp = (2 * N - i) * 2 / (3 * N)
        else:
            zexp = -1 + (4 * N - i) ** 2 / (3 * N * N)
        assert abs(zr[0] - zexp) < 2e-16
        d = np.diff(ph[start:start + n])
        np.testing.assert_allclose(d, 2 * np.pi / n, rtol=1e-12)
        start += n
    assert start == npix
    np.testing.assert_allclose(np.linalg.norm(xyz, axis=1), 1.0, atol=3e-16)
    # fraction of pixels north of z0 equals the cap area fraction (equal area)
    for z0 in (2 / 3, 0.0):
        assert abs((z > z0 + 1e-12).sum() / npix - (1 - z0) / 2) <= 4 * N / npix + 1e-12


@pytest.mark.parametrize("nside", [1, 2, 4, 8, 32])
def test_nest_ring_bijection(oracle, nside):
    npix = 12 * nside * nside
    n2r = oracle.nest2ring(nside, np.arange(npix))
    r2n = oracle.ring2nest(nside, np.arange(npix))
    np.testing.assert_array_equal(np.sort(n2r), np.arange(npix))
    np.testing.assert_array_equal(r2n[n2r], np.arange(npix))
    thr, phr, xr = oracle.pix2ang(nside)
    thn, phn, xn = oracle.pix2ang(nside, nest=True)
    # same pixel, same centre, bit for bit
    np.testing.assert_array_equal(thn, thr[n2r])
    np.testing.assert_array_equal(phn, phr[n2r])
    np.testing.assert_array_equal(xn, xr[n2r])


@pytest.mark.parametrize("nside", [1, 2, 8, 32])
def test_vec2pix_inverts_pix2ang(oracle, nside):
    npix = 12 * nside * nside
    _, _, xr = oracle.pix2ang(nside)
    _, _, xn = oracle.pix2ang(nside, nest=True)
    np.testing.assert_array_equal(oracle.vec2pix(nside, xr), np.arange(npix))
    np.testing.assert_array_equal(oracle.vec2pix(nside, xn, nest=True), np.arange(npix))


def test_nested_faces_are_compact(oracle):
    # a NESTED sub-block of 4^k pixels is a square patch: its extent shrinks by
    # 2 per level (the property the tile cones rely on)
    nside = 64
    _, _, xn = oracle.pix2ang(nside, nest=True)
    for block in (16, 64, 256):
        blocks = xn.reshape(-1, block, 3)
        c = blocks.mean(axis=1)
        c /= np.linalg.norm(c, axis=1, keepdims=True)
        rho = np.linalg.norm(blocks - c[:, None, :], axis=2).max()
        assert rho < 2.5 * math.sqrt(block) * math.sqrt(4 * math.pi / (12 * nside * nside))


def test_mk_pix2xy(oracle):
    x, y = oracle.mk_pix2xy()
    k = np.arange(1024)
    rebuilt = np.zeros(1024, dtype=np.int64)
    for b in range(5):
        rebuilt |= ((x >> b) & 1) << (2 * b)
        rebuilt |= ((y >> b) & 1) << (2 * b + 1)
    np.testing.assert_array_equal(rebuilt, k)
    assert x.max() == 31 and y.max() == 31
