"""A small observation in the reference programs' text formats, and the FP64
oracle's restatement of their host function vissGen on it.

Used by make_reference_fixtures.py (which runs the reference executable on
these inputs to produce golden outputs) and by the tests that compare the
oracle and the drop-in executables with those outputs.

The case: HEALPix Nside 4 NESTED pixel centres (192 pixels, FP32 text), a
log-normal sky, 4 satellites on a 2037.1 km lunar orbit in a compact
formation (so |u| <= ~30 wavelengths at 10 MHz and the reference's FP32
phases stay accurate), 10 snapshots -> 60 unique rows plus their 60 conjugate
mirror rows (u -> -u, same positions and bll), day 1.  The generator rejects
geometries where any (row, pixel) lies within 1e-4 of the occultation cone, so
an FP32 acosf and an FP64 dot product cannot disagree on a mask bit.
"""
from __future__ import annotations

import math
import os

import numpy as np

LAMBDA_10M = np.float32(3e8 / 1e7)   # the reference's lamda = 3e8 / frequency (FP32)


def _fmt(x) -> str:
    return repr(float(np.float32(x)))


def make_case(seed: int = 5, nside: int = 4, n_sat: int = 4, n_snap: int = 10,
              spacing=(40.0, 250.0), cross_sigma: float = 30.0):
    """spacing: along-track gaps U(lo, hi) m; cross_sigma: cross-track jitter (m)."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    from oracle import oracle as O

    th, ph, _ = O.pix2ang(nside, nest=True)
    npix = th.size
    theta = th.astype(np.float32)
    phi = ph.astype(np.float32)
    rng = np.random.default_rng(seed)
    B = np.exp(rng.standard_normal(npix)).astype(np.float32)
    B[rng.choice(npix, 2, replace=False)] += np.float32(20.0)
    thr = O.cone_threshold(1737.1e3, 300e3)
    lmn, _ = O.sky_pre_f32(theta, phi, B, np.float32(4 * math.pi / npix))
    for attempt in range(200):
        r0 = 1737.1e3 + 300e3
        inc = math.radians(30.0)
        e1 = np.array([1.0, 0.0, 0.0])
        e2 = np.array([0.0, math.cos(inc), math.sin(inc)])
        nrm = np.cross(e1, e2)
        along = np.concatenate([[0.0], np.cumsum(rng.uniform(spacing[0], spacing[1], n_sat - 1))])
        cross = rng.normal(0.0, cross_sigma, n_sat)
        t = np.arange(n_snap) * (2 * math.pi / 40.0) + rng.uniform(0, 2 * math.pi)
        ang = t[:, None] + along[None, :] / r0
        P = r0 * (np.cos(ang)[..., None] * e1 + np.sin(ang)[..., None] * e2) + cross[None, :, None] * nrm
        P = P.astype(np.float32).astype(np.float64)           # the text files hold FP32
        pairs = [(a, b) for a in range(n_sat) for b in range(a + 1, n_sat)]
        rows_a = np.array([P[i, a] for i in range(n_snap) for a, b in pairs])
        rows_b = np.array([P[i, b] for i in range(n_snap) for a, b in pairs])
        # cone margin: every (satellite position, pixel) pair far from the boundary
        q = np.concatenate([rows_a, rows_b])
        q = q / np.linalg.norm(q, axis=1, keepdims=True)
        if np.abs(lmn @ q.T - thr).min() > 1e-4:
            break
    else:
        raise RuntimeError("no geometry with a clear occultation margin")
    u = ((rows_a - rows_b) / float(LAMBDA_10M)).astype(np.float32)
    bll = np.linalg.norm(u.astype(np.float64), axis=1).astype(np.float32)
    uvw = np.concatenate([u, -u])
    xyza = np.concatenate([rows_a, rows_a]).astype(np.float32)
    xyzb = np.concatenate([rows_b, rows_b]).astype(np.float32)
    bll2 = np.concatenate([bll, bll])
    return dict(theta=theta, phi=phi, B=B, uvw=uvw, xyza=xyza, xyzb=xyzb, bll=bll2)


def write_inputs(case, root: str, variant_10m: bool = True, day: int = 1):
    """The reference's input files under root (earth_10Mhz/ or earth_1Mhz/),
    the rows as day `day`."""
    d = os.path.join(root, "earth_10Mhz" if variant_10m else "earth_1Mhz")
    os.makedirs(d, exist_ok=True)
    suffix = "_10Mhz.txt" if variant_10m else ".txt"
    npix = case["B"].size
    with open(os.path.join(d, "B" + suffix), "w") as f:
        f.write(f"{npix}\n")
        f.writelines(_fmt(x) + "\n" for x in case["B"])
    for name in ("theta", "phi"):
        with open(os.path.join(d, name + "_heal" + suffix), "w") as f:
            f.writelines(_fmt(x) + "\n" for x in case[name])
    for name in ("uvw", "xyza", "xyzb"):
        with open(os.path.join(d, f"{name}{day}day1M.txt"), "w") as f:
            f.write("0 0 0\n")                                 # first row, skipped
            f.writelines(" ".join(_fmt(v) for v in row) + "\n" for row in case[name])
    with open(os.path.join(d, f"bll{day}day1M.txt"), "w") as f:
        f.write("0\n")                                         # first token, skipped
        f.writelines(_fmt(x) + "\n" for x in case["bll"])
    return d


def read_inputs(root: str, variant_10m: bool = True):
    d = os.path.join(root, "earth_10Mhz" if variant_10m else "earth_1Mhz")
    suffix = "_10Mhz.txt" if variant_10m else ".txt"
    Bf = np.loadtxt(os.path.join(d, "B" + suffix), dtype=np.float32)
    case = dict(B=Bf[1:], theta=np.loadtxt(os.path.join(d, "theta_heal" + suffix), dtype=np.float32),
                phi=np.loadtxt(os.path.join(d, "phi_heal" + suffix), dtype=np.float32))
    for name in ("uvw", "xyza", "xyzb"):
        case[name] = np.loadtxt(os.path.join(d, name + "1day1M.txt"), dtype=np.float32)[1:]
    case["bll"] = np.loadtxt(os.path.join(d, "bll1day1M.txt"), dtype=np.float32)[1:]
    return case


def oracle_vissgen(case, blockage: bool, frequency: float = 1e7, dcf_shift: bool = False):
    """vissGen (vissgen3d_blockage.cu:195-563) for one day, FP64 oracle:
    returns (V after the w-rotation, complex128 per row; Re C per pixel).
    dcf_shift: the blockage program's shifted DCF (vissgen3d_blockage.cu:133-139,
    dcf[k] from shell k+1 for 1 <= k < nr; dcf[nr] as un-shifted)."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    from oracle import oracle as O

    npix = case["B"].size
    s = np.float32(4 * math.pi / npix)
    lmn, Bs = O.sky_pre_f32(case["theta"], case["phi"], case["B"], s)
    uvw = case["uvw"].astype(np.float64)
    n = uvw.shape[0]
    amount = n // 2
    w = uvw[:, 2]
    thr = O.cone_threshold(np.float32(1737.1e3), np.float32(300e3))
    P = np.concatenate([case["xyza"][:n], case["xyzb"][:n]]).astype(np.float64)
    occ = O.occulters(P, 0.0, 1, thr)
    refs = np.stack([np.arange(n), n + np.arange(n), -np.ones(n)], axis=1).astype(np.int32)
    V = np.zeros(n, np.complex128)
    V[:amount] = O.forward(uvw[:amount], lmn, Bs.astype(np.float64), refs[:amount], occ, off=-w[:amount])
    V[amount:2 * amount] = np.conj(V[:amount])
    V0 = V.copy()
    lam = np.float32(3e8 / np.float32(frequency))
    nr = int(np.ceil(np.float32(100e3) / lam * np.float32(2)))
    gs, _counts, dcf = O.dcf(case["bll"], nr, 1)
    if dcf_shift:
        dcf = dcf.copy()
        dcf[1:nr] = dcf[2:nr + 1]
    V = O.wrot(w, V)
    dg = O.gamma_dg(case["uvw"][:, 2], case["bll"][:n])
    wt = O.weights(gs[:n], dg, dcf, nr)
    C = O.adjoint(uvw, wt.astype(np.float64) * V, lmn, refs if blockage else None,
                  occ if blockage else None)
    return V0, C
