"""Host side of the formation mode (no GPU): the satellite vectors and
occulter rows pipeline.formation_inputs builds reproduce, pair by pair, the
per-sample layout the direct entry points take: u_ab = U_a - U_b in the
samples' lexicographic pair order, and each sample's occulter references
pointing at its two satellites' rows and its snapshot's row."""
import numpy as np
import torch

from viss_optimize_3d_b200 import pipeline, synth


def test_formation_inputs_match_sample_layout(oracle):
    cfg = synth.scaled(synth.CONFIGS["c3_10mhz"], nside=8, n_snap=12)
    obs = synth.make_observation(cfg)
    f = cfg.freqs_hz[0]
    occ = np.concatenate([oracle.occulters(obs.occ_sat_positions, synth.R_MOON, 0), obs.earth_rows])
    U, occ_sat, occ_snap = pipeline.formation_inputs(obs, f, device="cpu", occ=torch.as_tensor(occ))
    T, S = cfg.n_snap, cfg.n_sat
    assert U.shape == (T, S, 3) and occ_sat.shape == (T, S, 4) and occ_snap.shape == (T, 4)
    pairs = synth.baseline_pairs(S)
    B = len(pairs)
    assert [tuple(p) for p in pairs] == [(a, b) for a in range(S) for b in range(a + 1, S)]
    U = U.numpy()
    uvw = obs.uvw(f).reshape(T, B, 3)
    diff = U[:, pairs[:, 0], :] - U[:, pairs[:, 1], :]
    # the same baselines to FP64 rounding: far below the 2^-23-turn phase resolution
    assert np.abs(diff - uvw).max() <= 1e-9
    refs = obs.refs.reshape(T, B, 3)
    np.testing.assert_array_equal(occ_sat.numpy()[np.arange(T)[:, None], pairs[None, :, 0]], occ[refs[..., 0]])
    np.testing.assert_array_equal(occ_sat.numpy()[np.arange(T)[:, None], pairs[None, :, 1]], occ[refs[..., 1]])
    np.testing.assert_array_equal(np.broadcast_to(occ_snap.numpy()[:, None, :], (T, B, 4)), occ[refs[..., 2]])


def test_formation_inputs_without_occultation():
    cfg = synth.scaled(synth.CONFIGS["c1"], nside=8, n_snap=5)
    obs = synth.make_observation(cfg)
    U, occ_sat, occ_snap = pipeline.formation_inputs(obs, cfg.freqs_hz[0], device="cpu")
    assert occ_sat is None and occ_snap is None
    pairs = synth.baseline_pairs(cfg.n_sat)
    d = U.numpy()[:, pairs[:, 0], :] - U.numpy()[:, pairs[:, 1], :]
    assert np.abs(d.reshape(-1, 3) - obs.uvw(cfg.freqs_hz[0])).max() <= 1e-9
