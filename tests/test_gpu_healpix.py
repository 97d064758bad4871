"""GPU HEALPix tables vs the oracle: bit-exact indices, <= 1 ulp of FP64 for
theta, phi and the unit vector (replaces pix2ang.cu:61-160)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def ulp_diff(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)

    def ordered(x):
        i = x.view(np.int64)
        return np.where(i < 0, np.int64(-0x8000000000000000) - i, i)

    return np.abs(ordered(a) - ordered(b))


@pytest.mark.parametrize("nside", [1, 2, 16, 64, 256])
@pytest.mark.parametrize("scheme", ["ring", "nest"])
def test_pix2ang_within_one_ulp(viss, oracle, cuda_device, nside, scheme):
    th, ph, xyz = viss.pix2ang(nside, scheme, device=cuda_device)
    oth, oph, oxyz = oracle.pix2ang(nside, nest=(scheme == "nest"))
    d_th = ulp_diff(th.cpu().numpy(), oth).max()
    d_ph = ulp_diff(ph.cpu().numpy(), oph).max()
    g = xyz.cpu().numpy()
    # components that are tiny (|x| < 1e-300 e.g. exact zeros) compare absolutely
    d_xyz = ulp_diff(g, oxyz)
    d_xyz = np.where(np.abs(oxyz) < 1e-300, np.abs(g - oxyz) > 0, d_xyz).max()
    assert d_th <= 1 and d_ph <= 1 and d_xyz <= 1, (d_th, d_ph, d_xyz)


@pytest.mark.parametrize("nside", [1, 4, 32, 128])
def test_scheme_conversion_exact(viss, oracle, cuda_device, nside):
    npix = 12 * nside * nside
    n2r = viss.pix_convert(nside, "nest", "ring", device=cuda_device).cpu().numpy()
    r2n = viss.pix_convert(nside, "ring", "nest", device=cuda_device).cpu().numpy()
    sel = np.arange(npix) if npix <= 50000 else np.random.default_rng(0).choice(npix, 50000, replace=False)
    np.testing.assert_array_equal(n2r[sel], oracle.nest2ring(nside, sel))
    np.testing.assert_array_equal(r2n[sel], oracle.ring2nest(nside, sel))
    np.testing.assert_array_equal(r2n[n2r], np.arange(npix))
    # the same pixel centre through either scheme, bit for bit
    _, _, xr = viss.pix2ang(nside, "ring", device=cuda_device)
    _, _, xn = viss.pix2ang(nside, "nest", device=cuda_device)
    assert torch.equal(xn, xr[torch.as_tensor(n2r, device=cuda_device)])


def test_mk_pix2xy_and_lmn(viss, oracle, cuda_device):
    x, y = viss.mk_pix2xy(device=cuda_device)
    ox, oy = oracle.mk_pix2xy()
    np.testing.assert_array_equal(x.cpu().numpy(), ox)
    np.testing.assert_array_equal(y.cpu().numpy(), oy)
    _, _, xyz = viss.pix2ang(32, "ring", device=cuda_device)
    lmn = viss.pix2lmn(32, "ring", device=cuda_device)
    # (l, m, n) = (x, -y, z): the reference's convention, vissgen3d_blockage.cu:53-74
    assert torch.equal(lmn[:, 0], xyz[:, 0]) and torch.equal(lmn[:, 1], -xyz[:, 1])
    assert torch.equal(lmn[:, 2], xyz[:, 2])


def test_sky_pre_matches_oracle(viss, oracle, cuda_device):
    th, ph, _ = oracle.pix2ang(16, nest=True)
    th32, ph32 = th.astype(np.float32), ph.astype(np.float32)
    B = np.random.default_rng(1).uniform(0, 5, th.size).astype(np.float32)
    s = np.float32(4 * np.pi / th.size)
    lmn, Bo = viss.healpix_moonback_pre(torch.as_tensor(th32, device=cuda_device),
                                        torch.as_tensor(ph32, device=cuda_device),
                                        torch.as_tensor(B, device=cuda_device), float(s))
    olmn, oB = oracle.sky_pre_f32(th32, ph32, B, s)
    np.testing.assert_array_equal(Bo.cpu().numpy(), oB)
    assert np.abs(lmn.cpu().numpy() - olmn).max() < 4e-16
