"""The seeded synthetic generator (CPU): shapes, determinism, geometry laws."""
import math

import numpy as np

from viss_optimize_3d_b200 import synth


def test_config_sizes_match_the_benchmark_table():
    c = synth.CONFIGS
    assert c["c1"].npix == 12288 and c["c1"].n_samples == 28 * 360
    assert c["c2"].npix == 49152 and c["c2"].n_samples == 28 * 720
    assert c["c3_10mhz"].npix == 786432 and c["c3_10mhz"].n_samples == 388800
    assert c["c4"].npix == 196608 and c["c4"].n_samples == 129600 and len(c["c4"].freqs_hz) == 64
    assert c["c5"].n_samples == 45 * 4320


def test_observation_is_deterministic_and_lawful():
    cfg = synth.scaled(synth.CONFIGS["c3_10mhz"], nside=8, n_snap=48)
    a = synth.make_observation(cfg)
    b = synth.make_observation(cfg)
    np.testing.assert_array_equal(a.baselines_m, b.baselines_m)
    np.testing.assert_array_equal(a.sky, b.sky)
    r = np.linalg.norm(a.positions, axis=2)
    assert abs(r.mean() - (synth.R_MOON + synth.ALTITUDE)) < 2e3
    # consecutive along-track spacings in [1, 30] km
    d = np.linalg.norm(a.positions[0, 1:] - a.positions[0, :-1], axis=1)
    assert (d > 0.9e3).all() and (d < 31e3).all()
    # inclination 30 deg: orbit normal tilted 30 deg from z
    p0, p1 = a.positions[0, 0], a.positions[cfg.n_snap // 4, 0]
    nrm = np.cross(p0, p1)
    nrm /= np.linalg.norm(nrm)
    assert abs(math.degrees(math.acos(abs(nrm[2]))) - 30.0) < 0.2
    # sample order (snapshot, baseline) and refs pointing at its satellites
    B = cfg.n_baselines
    k = 5 * B + 7
    pa, pb = a.pairs[7]
    np.testing.assert_allclose(a.baselines_m[k], a.positions[5, pa] - a.positions[5, pb])
    assert tuple(a.refs[k]) == (5 * cfg.n_sat + pa, 5 * cfg.n_sat + pb, cfg.n_snap * cfg.n_sat + 5)
    # earth rows: cap of 0.95 deg, q = -e
    assert a.earth_rows.shape == (cfg.n_snap, 4)
    np.testing.assert_allclose(a.earth_rows[:, 3], -math.cos(math.radians(0.95)))
    # sky law: 20 bright sources, diffuse log-normal
    assert (a.sky > 10).sum() >= 20


def test_uvw_scales_with_frequency():
    obs = synth.make_observation(synth.scaled(synth.CONFIGS["c1"], nside=4, n_snap=10))
    np.testing.assert_allclose(obs.uvw(1e7), 10 * obs.uvw(1e6))
    assert abs(synth.C_LIGHT / 1e6 - 299.79) < 0.01
    assert obs.nr(1e6) >= 2 * obs.bll(1e6).max()
