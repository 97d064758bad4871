"""Seeded synthetic observations for the benchmark configurations.

The reference's inputs (sky map B, satellite tracks, uvw, bll) were made
outside its repository and never shipped (vissgen3d_blockage.cu:312,334,355,
376 name the files only).  This module generates inputs of the same kind:

* sky: I_j = exp(N(0,1)) per pixel plus 20 point sources U(10, 100) at
  random pixels (seed 0), on a HEALPix RING grid; per-channel spectral index
  N(-2.5, 0.1) per pixel for multi-channel runs;
* satellites: one circular lunar orbit, radius 1737.4 + 300 km, inclination
  30 deg; consecutive along-track spacings U(1, 30) km, constant radial and
  cross-track offsets N(0, 0.5) km per satellite;
* snapshots evenly spaced over one orbital period;
* baselines u = (P_a - P_b) / lambda (FP64, lambda = c / f), all pairs a < b,
  sample k = snapshot * n_baselines + baseline;
* occulters: one ray-sphere row per (snapshot, satellite) against the Moon,
  and optionally one Earth-cap row per snapshot (radius 0.95 deg, direction
  advancing 13.2 deg/day in the orbital plane of the Moon).

Everything is numpy FP64 and deterministic for a given seed.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

C_LIGHT = 299792458.0
GM_MOON = 4.9048695e12          # m^3 s^-2
R_MOON = 1737.4e3               # m
ALTITUDE = 300e3                # m
EARTH_CAP_DEG = 0.95
EARTH_RATE_DEG_PER_DAY = 13.2


@dataclasses.dataclass(frozen=True)
class ObsConfig:
    name: str
    nside: int
    n_sat: int
    n_snap: int
    freqs_hz: tuple
    moon: bool = False
    earth: bool = False
    imaging_mask: bool = True     # apply the occultation mask in imaging too
    seed: int = 0
    inclination_deg: float = 30.0
    day: float = 0.0              # epoch of the first snapshot, days

    @property
    def npix(self) -> int:
        return 12 * self.nside * self.nside

    @property
    def n_baselines(self) -> int:
        return self.n_sat * (self.n_sat - 1) // 2

    @property
    def n_samples(self) -> int:
        return self.n_baselines * self.n_snap


CONFIGS = {
    # plain method, CPU-runnable
    "c1": ObsConfig("c1", nside=32, n_sat=8, n_snap=360, freqs_hz=(1e6,)),
    # 10 MHz with Moon occultation
    "c2": ObsConfig("c2", nside=64, n_sat=8, n_snap=720, freqs_hz=(1e7,), moon=True),
    # headline: Nside 256, 45 baselines x 8640 snapshots, Moon + Earth
    "c3_1mhz": ObsConfig("c3_1mhz", nside=256, n_sat=10, n_snap=8640, freqs_hz=(1e6,),
                         moon=True, earth=True),
    "c3_10mhz": ObsConfig("c3_10mhz", nside=256, n_sat=10, n_snap=8640, freqs_hz=(1e7,),
                          moon=True, earth=True),
    # the reference's production operating point at 1 MHz: Nside 512 and one
    # day of up to 4,000,000 rows (vissgen3d_blockage.cu:28), i.e. 2,000,160
    # unique samples once the mirror rows are folded (45 baselines x 44,448
    # snapshots), Moon + Earth
    "prod_1mhz": ObsConfig("prod_1mhz", nside=512, n_sat=10, n_snap=44448, freqs_hz=(1e6,),
                           moon=True, earth=True),
    # batched: 64 channels 1-10 MHz
    "c4": ObsConfig("c4", nside=128, n_sat=10, n_snap=2880,
                    freqs_hz=tuple(np.linspace(1e6, 1e7, 64)), moon=True, earth=True),
    # differentiable reconstruction
    "c5": ObsConfig("c5", nside=128, n_sat=10, n_snap=4320, freqs_hz=(1e7,), moon=True),
}


def scaled(cfg: ObsConfig, nside: int | None = None, n_snap: int | None = None,
           n_sat: int | None = None, freqs_hz=None) -> ObsConfig:
    """A smaller copy of a configuration (same laws, fewer pixels/samples)."""
    return dataclasses.replace(cfg, name=cfg.name + "_small",
                               nside=nside or cfg.nside, n_snap=n_snap or cfg.n_snap,
                               n_sat=n_sat or cfg.n_sat,
                               freqs_hz=tuple(freqs_hz) if freqs_hz is not None else cfg.freqs_hz)


def sky_map(npix: int, seed: int = 0) -> np.ndarray:
    """I_j = exp(N(0,1)) + 20 point sources U(10,100) at random pixels (RING order)."""
    rng = np.random.default_rng(seed)
    I = np.exp(rng.standard_normal(npix))
    idx = rng.choice(npix, size=min(20, npix), replace=False)
    I[idx] += rng.uniform(10.0, 100.0, size=idx.size)
    return I


def spectral_index(npix: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed + 1000)
    return rng.normal(-2.5, 0.1, size=npix)


def channel_sky(I0: np.ndarray, alpha: np.ndarray, f_hz: float, f0_hz: float = 1e6) -> np.ndarray:
    return I0 * (f_hz / f0_hz) ** alpha


def orbit_period(radius: float = R_MOON + ALTITUDE) -> float:
    return 2.0 * math.pi * math.sqrt(radius ** 3 / GM_MOON)


def satellite_positions(cfg: ObsConfig) -> np.ndarray:
    """P[t, s, :] in metres, Moon-centred frame (the (l, m, n) frame)."""
    rng = np.random.default_rng(cfg.seed + 1)
    r0 = R_MOON + ALTITUDE
    spacing = rng.uniform(1e3, 30e3, size=cfg.n_sat - 1)
    along = np.concatenate([[0.0], np.cumsum(spacing)])
    radial = rng.normal(0.0, 500.0, size=cfg.n_sat)
    cross = rng.normal(0.0, 500.0, size=cfg.n_sat)
    inc = math.radians(cfg.inclination_deg)
    e1 = np.array([1.0, 0.0, 0.0])
    e2 = np.array([0.0, math.cos(inc), math.sin(inc)])
    nrm = np.cross(e1, e2)
    T = orbit_period(r0)
    t = np.arange(cfg.n_snap) * (T / cfg.n_snap)
    omega = 2.0 * math.pi / T
    ang = omega * t[:, None] + along[None, :] / r0            # (T, S)
    rad = (r0 + radial)[None, :, None]
    P = rad * (np.cos(ang)[..., None] * e1 + np.sin(ang)[..., None] * e2) \
        + cross[None, :, None] * nrm
    return P


def earth_direction(cfg: ObsConfig) -> np.ndarray:
    """Unit vector toward the Earth per snapshot, advancing 13.2 deg/day."""
    T = orbit_period()
    t_days = cfg.day + np.arange(cfg.n_snap) * (T / cfg.n_snap) / 86400.0
    a = np.radians(EARTH_RATE_DEG_PER_DAY * t_days)
    return np.stack([np.cos(a), np.sin(a), np.zeros_like(a)], axis=-1)


def baseline_pairs(n_sat: int) -> np.ndarray:
    return np.array([(a, b) for a in range(n_sat) for b in range(a + 1, n_sat)], dtype=np.int32)


@dataclasses.dataclass
class Observation:
    cfg: ObsConfig
    positions: np.ndarray      # (T, S, 3) metres
    pairs: np.ndarray          # (B, 2)
    baselines_m: np.ndarray    # (K, 3) metres, sample order (t, b)
    refs: np.ndarray | None    # (K, 3) int32 occulter rows
    occ_sat_positions: np.ndarray  # (T*S, 3) positions whose rows come first in the table
    earth_rows: np.ndarray | None  # (T, 4) (q, thr) rows appended after the satellites
    sky: np.ndarray            # (J,) RING order, FP64
    alpha: np.ndarray | None

    def uvw(self, f_hz: float) -> np.ndarray:
        return self.baselines_m / (C_LIGHT / f_hz)

    def bll(self, f_hz: float) -> np.ndarray:
        return np.linalg.norm(self.uvw(f_hz), axis=1)

    def nr(self, f_hz: float) -> int:
        """Number of half-wavelength shells that covers every sample."""
        return int(math.ceil(2.0 * float(self.bll(f_hz).max()) + 1.0))

    def sky_at(self, f_hz: float) -> np.ndarray:
        if self.alpha is None:
            return self.sky
        return channel_sky(self.sky, self.alpha, f_hz)


def make_observation(cfg: ObsConfig) -> Observation:
    P = satellite_positions(cfg)
    pairs = baseline_pairs(cfg.n_sat)
    T, S, B = cfg.n_snap, cfg.n_sat, pairs.shape[0]
    bl = (P[:, pairs[:, 0], :] - P[:, pairs[:, 1], :]).reshape(T * B, 3)
    refs = None
    earth_rows = None
    if cfg.moon or cfg.earth:
        t_idx = np.repeat(np.arange(T), B)
        b_idx = np.tile(np.arange(B), T)
        refs = np.full((T * B, 3), -1, dtype=np.int32)
        if cfg.moon:
            refs[:, 0] = t_idx * S + pairs[b_idx, 0]
            refs[:, 1] = t_idx * S + pairs[b_idx, 1]
        if cfg.earth:
            e = earth_direction(cfg)
            earth_rows = np.concatenate([-e, np.full((T, 1), -math.cos(math.radians(EARTH_CAP_DEG)))],
                                        axis=1)
            refs[:, 2] = T * S + t_idx
    npix = cfg.npix
    sky = sky_map(npix, cfg.seed)
    alpha = spectral_index(npix, cfg.seed) if len(cfg.freqs_hz) > 1 else None
    return Observation(cfg=cfg, positions=P, pairs=pairs, baselines_m=bl, refs=refs,
                       occ_sat_positions=P.reshape(T * S, 3), earth_rows=earth_rows,
                       sky=sky, alpha=alpha)
