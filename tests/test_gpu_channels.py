"""Frequency channels in one launch (viss_plan_set_channels) against one plan
per channel, and both against the FP64 oracle on a small multi-channel case
(the batched benchmark configuration's laws: spectral index per pixel,
Moon + Earth occultation)."""
import numpy as np
import pytest
import torch

from viss_optimize_3d_b200 import pipeline, synth

pytestmark = pytest.mark.gpu


def test_batched_channels_match_per_channel_plans(viss, oracle, cuda_device):
    freqs = (1e6, 4e6, 7e6, 1e7)
    cfg = synth.scaled(synth.CONFIGS["c4"], nside=16, n_snap=40, freqs_hz=freqs)
    obs = synth.make_observation(cfg)
    lmn = viss.pix2lmn(cfg.nside, "ring", device=cuda_device)
    occ = pipeline.build_occulters(obs, cuda_device)
    refs = torch.as_tensor(obs.refs, device=cuda_device)
    C, K, J = len(freqs), cfg.n_samples, cfg.npix
    uvw_all = torch.cat([torch.as_tensor(obs.uvw(f), device=cuda_device) for f in freqs])
    sky_all = torch.stack([torch.as_tensor(obs.sky_at(f) * 4 * np.pi / J, dtype=torch.float32,
                                           device=cuda_device) for f in freqs])
    plan = viss.Plan(lmn, uvw_all, None, refs.repeat(C, 1), occ, channels=C)
    V = plan.forward(sky_all)
    rng = np.random.default_rng(2)
    coef = torch.as_tensor((rng.standard_normal(C * K) + 1j * rng.standard_normal(C * K)).astype(np.complex64),
                           device=cuda_device)
    img = plan.adjoint(coef)
    assert img.shape == (C, J)
    L = lmn.cpu().numpy()
    occ_o = occ.cpu().numpy()
    for c, f in enumerate(freqs):
        single = viss.Plan(lmn, uvw_all[c * K:(c + 1) * K], None, refs, occ)
        Vc = single.forward(sky_all[c])
        Ic = single.adjoint(coef[c * K:(c + 1) * K])
        torch.testing.assert_close(V[c * K:(c + 1) * K], Vc, rtol=1e-5, atol=1e-6 * Vc.abs().max().item())
        torch.testing.assert_close(img[c], Ic, rtol=1e-5, atol=1e-6 * Ic.abs().max().item())
        Vo = oracle.forward(obs.uvw(f), L, sky_all[c].double().cpu().numpy(), obs.refs, occ_o)
        Vb = V[c * K:(c + 1) * K].cpu().numpy()
        assert np.linalg.norm(Vb - Vo) / np.linalg.norm(Vo) < 1e-5
        Io = oracle.adjoint(obs.uvw(f), coef[c * K:(c + 1) * K].cpu().numpy().astype(np.complex128), L,
                            obs.refs, occ_o)
        assert np.linalg.norm(img[c].cpu().numpy() - Io) / np.linalg.norm(Io) < 1e-5


def test_channels_require_a_divisor(viss, cuda_device):
    lmn = viss.pix2lmn(2, "ring", device=cuda_device)
    plan = viss.Plan(lmn, torch.zeros((10, 3), dtype=torch.float64, device=cuda_device))
    with pytest.raises(RuntimeError):
        plan.set_channels(3)
    with pytest.raises(RuntimeError):
        plan.set_channels(2)      # 5 samples per channel: must be even
