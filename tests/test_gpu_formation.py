"""Formation mode (viss_plan_set_formation, csrc/formation.cu): every sample
a pair of one snapshot's satellites, the exponential factored per satellite.
Same arithmetic contract as the direct kernels: the forward and adjoint match
the direct path on the same plan and the FP64 oracle (rel-L2 1e-5; masks from
the same exact predicate), with Moon rows, Earth rows, phase offsets, no mask;
invalid uses are rejected."""
import dataclasses

import numpy as np
import pytest
import torch

from viss_optimize_3d_b200 import api, pipeline, synth

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _case(cfg, f, dev, seed_off=None):
    obs = synth.make_observation(cfg)
    g = pipeline.upload(obs, f, device=dev)
    U, occ_sat, occ_snap = pipeline.formation_inputs(obs, f, device=dev, occ=g.occ)
    off = None
    if seed_off is not None:
        off = np.random.default_rng(seed_off).uniform(-3, 3, cfg.n_samples)
        g.plan.set_samples(g.uvw, torch.as_tensor(off, device=dev), g.refs, g.occ)
    g.plan.set_formation(U, None if off is None else off.reshape(cfg.n_snap, -1), occ_sat, occ_snap)
    return obs, g, off


@pytest.mark.parametrize("cfgname,f,S,nside,T,with_off", [
    ("c2", 1e7, 8, 16, 30, False),
    ("c3_10mhz", 1e7, 10, 16, 24, True),
    ("c3_1mhz", 1e6, 10, 32, 16, False),
    ("c1", 1e6, 4, 16, 200, True),        # no occultation; several adjoint chunks
    ("c2", 1e7, 6, 16, 130, False),       # Moon only, T not a multiple of 8
    ("c3_10mhz", 1e7, 5, 16, 40, False),  # odd S
    ("c3_10mhz", 1e7, 7, 16, 19, True),
    ("c3_10mhz", 1e7, 2, 16, 64, False),
])
def test_formation_matches_direct_and_oracle(oracle, cuda_device, cfgname, f, S, nside, T, with_off):
    cfg = synth.scaled(synth.CONFIGS[cfgname], nside=nside, n_snap=T, n_sat=S)
    obs, g, off = _case(cfg, f, cuda_device, seed_off=3 if with_off else None)
    lmn, uvw = g.lmn.cpu().numpy(), g.uvw.cpu().numpy()
    occ = g.occ.cpu().numpy() if g.occ is not None else None
    Vd = g.plan.forward(g.sky).cpu().numpy().astype(np.complex128)
    Vf = g.plan.forward_formation(g.sky).cpu().numpy().astype(np.complex128)
    Vo = oracle.forward(uvw, lmn, g.sky.cpu().numpy().astype(np.float64), obs.refs, occ, off=off)
    assert rel_l2(Vf, Vo) <= 1e-5, rel_l2(Vf, Vo)
    assert rel_l2(Vf, Vd) <= 1e-5, rel_l2(Vf, Vd)
    rng = np.random.default_rng(5)
    a = (rng.standard_normal(cfg.n_samples) + 1j * rng.standard_normal(cfg.n_samples)).astype(np.complex64)
    at = torch.as_tensor(a, device=cuda_device)
    Cd = g.plan.adjoint(at, scale=2.0).cpu().numpy()
    Cf = g.plan.adjoint_formation(at, scale=2.0).cpu().numpy()
    Co = 2.0 * oracle.adjoint(uvw, a.astype(np.complex128), lmn, obs.refs, occ, off=off)
    assert rel_l2(Cf, Co) <= 1e-5, rel_l2(Cf, Co)
    assert rel_l2(Cf, Cd) <= 1e-5, rel_l2(Cf, Cd)
    # without the mask
    Vn = g.plan.forward_formation(g.sky, mask=False).cpu().numpy().astype(np.complex128)
    Von = oracle.forward(uvw, lmn, g.sky.cpu().numpy().astype(np.float64), off=off)
    assert rel_l2(Vn, Von) <= 1e-5, rel_l2(Vn, Von)
    Cn = g.plan.adjoint_formation(at, mask=False).cpu().numpy()
    Con = oracle.adjoint(uvw, a.astype(np.complex128), lmn, off=off)
    assert rel_l2(Cn, Con) <= 1e-5, rel_l2(Cn, Con)


def test_formation_rejects_invalid_use(cuda_device):
    from viss_optimize_3d_b200._capi import VissError, check, lib
    lmn = api.pix2lmn(4, "ring", device=cuda_device)
    plan = api.Plan(lmn)
    with pytest.raises(VissError, match="formation not set"):
        plan.form_T, plan.form_B = 1, 1
        plan.forward_formation(torch.ones(lmn.shape[0], device=cuda_device))
    with pytest.raises(VissError, match="S must be"):
        plan.set_formation(torch.zeros((3, 11, 3), dtype=torch.float64))
    plan.set_formation(torch.zeros((3, 4, 3), dtype=torch.float64))
    V = torch.empty(18, dtype=torch.complex64, device=cuda_device)
    sky = torch.ones(lmn.shape[0], device=cuda_device)
    with pytest.raises(VissError, match="split precision only"):
        check(lib.viss_forward_formation(plan._h, sky.data_ptr(), V.data_ptr(), 1, None), "fwd")
    U = torch.zeros((3, 4, 3), dtype=torch.float64)
    U[1, 2, 0] = float("nan")
    with pytest.raises(VissError, match="non-finite"):
        plan.set_formation(U)
    # shapes: U must be (T, S, 3) or (C, T, S, 3); occulter rows cover T snapshots
    with pytest.raises(ValueError, match="U must be"):
        plan.set_formation(torch.zeros((3, 4, 2), dtype=torch.float64))
    with pytest.raises(ValueError, match="occulter rows must cover"):
        plan.set_formation(torch.zeros((2, 3, 4, 3), dtype=torch.float64),
                           occ_sat=torch.zeros((4, 4, 4), dtype=torch.float64))
    plan.set_formation(torch.zeros((2, 3, 4, 3), dtype=torch.float64))
    assert plan.form_C == 2 and plan.form_T == 6
    with pytest.raises(ValueError, match="sky must hold"):
        plan.forward_formation(torch.ones(lmn.shape[0], device=cuda_device))
    with pytest.raises(ValueError, match="coef must hold"):
        plan.adjoint_formation(torch.ones(5, dtype=torch.complex64, device=cuda_device))


def test_formation_hidden_snapshots(oracle, cuda_device):
    """A snapshot row that hides the whole sky (thr > 1) zeroes that snapshot's
    samples exactly; a satellite row that hides everything zeroes its pairs."""
    cfg = synth.scaled(synth.CONFIGS["c3_10mhz"], nside=16, n_snap=12, n_sat=6)
    obs = synth.make_observation(cfg)
    g = pipeline.upload(obs, 1e7, device=cuda_device)
    U, occ_sat, occ_snap = pipeline.formation_inputs(obs, 1e7, device=cuda_device, occ=g.occ)
    occ_snap = occ_snap.clone()
    occ_snap[3] = torch.tensor([0.0, 0.0, 1.0, 2.0], dtype=torch.float64)
    occ_sat = occ_sat.clone()
    occ_sat[5, 2] = torch.tensor([0.0, 0.0, 1.0, 2.0], dtype=torch.float64)
    g.plan.set_formation(U, None, occ_sat, occ_snap)
    B = 15
    V = g.plan.forward_formation(g.sky).cpu().numpy().reshape(12, B)
    assert np.all(V[3] == 0)
    pairs_with_2 = [k for k, (a, b) in enumerate(synth.baseline_pairs(6)) if 2 in (a, b)]
    assert np.all(V[5, pairs_with_2] == 0)
    # the rest against the oracle on the same rows
    occ = torch.cat([occ_sat.reshape(-1, 4), occ_snap]).cpu().numpy()
    Vo = oracle.forward(g.uvw.cpu().numpy(), g.lmn.cpu().numpy(), g.sky.cpu().numpy().astype(np.float64),
                        obs.refs, occ).reshape(12, B)
    assert rel_l2(V, Vo) <= 1e-5, rel_l2(V, Vo)


def test_formation_channels(oracle, cuda_device):
    """Frequency channels in one launch per kernel (set_formation with
    U (C, T, S, 3)): every channel's V and image against the oracle on that
    channel's uvw and sky; the occulter rows are shared."""
    cfg = synth.scaled(synth.CONFIGS["c4"], nside=16, n_snap=24, freqs_hz=(1e6, 4.5e6, 1e7))
    obs = synth.make_observation(cfg)
    C, K, J = 3, cfg.n_samples, cfg.npix
    g = pipeline.upload(obs, cfg.freqs_hz[0], device=cuda_device)
    Us, skies = [], []
    for f in cfg.freqs_hz:
        U, occ_sat, occ_snap = pipeline.formation_inputs(obs, f, device=cuda_device, occ=g.occ)
        Us.append(U)
        skies.append(torch.as_tensor(obs.sky_at(f) * 4 * np.pi / J, dtype=torch.float32, device=cuda_device))
    plan = g.plan
    plan.set_formation(torch.stack(Us), None, occ_sat, occ_snap)
    sky = torch.stack(skies)
    V = plan.forward_formation(sky).cpu().numpy().reshape(C, K)
    rng = np.random.default_rng(11)
    a = (rng.standard_normal(C * K) + 1j * rng.standard_normal(C * K)).astype(np.complex64)
    img = plan.adjoint_formation(torch.as_tensor(a, device=cuda_device), scale=2.0).cpu().numpy()
    assert img.shape == (C, J)
    lmn = g.lmn.cpu().numpy()
    occ = g.occ.cpu().numpy()
    for c, f in enumerate(cfg.freqs_hz):
        uvw = obs.uvw(f)
        Vo = oracle.forward(uvw, lmn, skies[c].cpu().numpy().astype(np.float64), obs.refs, occ)
        assert rel_l2(V[c], Vo) <= 1e-5, (c, rel_l2(V[c], Vo))
        Co = 2.0 * oracle.adjoint(uvw, a[c * K:(c + 1) * K].astype(np.complex128), lmn, obs.refs, occ)
        assert rel_l2(img[c], Co) <= 1e-5, (c, rel_l2(img[c], Co))
    # channels must divide the snapshots; set_formation resets to one channel
    from viss_optimize_3d_b200._capi import VissError, check, lib
    with pytest.raises(VissError, match="multiple of channels"):
        check(lib.viss_plan_set_formation_channels(plan._h, 5), "set_formation_channels")
    plan.set_formation(Us[0], None, occ_sat, occ_snap)
    V0 = plan.forward_formation(skies[0]).cpu().numpy()
    assert rel_l2(V0, V[0]) <= 1e-6


def test_formation_flags(oracle, cuda_device):
    """VISS_NO_OFFSET drops the phase offsets, VISS_ACCUMULATE adds into out,
    as in the direct entry points."""
    cfg = synth.scaled(synth.CONFIGS["c3_10mhz"], nside=16, n_snap=16, n_sat=6)
    obs, g, off = _case(cfg, 1e7, cuda_device, seed_off=9)
    lmn, uvw, occ = g.lmn.cpu().numpy(), g.uvw.cpu().numpy(), g.occ.cpu().numpy()
    sky64 = g.sky.cpu().numpy().astype(np.float64)
    Vn = g.plan.forward_formation(g.sky, use_offset=False).cpu().numpy()
    assert rel_l2(Vn, oracle.forward(uvw, lmn, sky64, obs.refs, occ)) <= 1e-5
    V = g.plan.forward_formation(g.sky)
    out = V.clone()
    g.plan.forward_formation(g.sky, out=out, accumulate=True)
    assert rel_l2(out.cpu().numpy(), 2 * V.cpu().numpy()) <= 1e-6
    a = torch.ones(cfg.n_samples, dtype=torch.complex64, device=cuda_device)
    Cn = g.plan.adjoint_formation(a, use_offset=False).cpu().numpy()
    assert rel_l2(Cn, oracle.adjoint(uvw, np.ones(cfg.n_samples, np.complex128), lmn, obs.refs, occ)) <= 1e-5
    img = g.plan.adjoint_formation(a)
    img2 = img.clone()
    g.plan.adjoint_formation(a, out=img2, accumulate=True)
    assert rel_l2(img2.cpu().numpy(), 2 * img.cpu().numpy()) <= 1e-6
