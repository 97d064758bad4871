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
              spacing=(40.0, 250.0), cross_sigma: float = 30.0, frequency: float = 1e7):
    """spacing: along-track gaps U(lo, hi) m; cross_sigma: cross-track jitter (m);
    frequency: the uvw rows are in wavelengths of the reference's FP32
    lamda = 3e8 / frequency."""
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
    lam = np.float32(3e8 / np.float32(frequency))
    u = ((rows_a - rows_b) / float(lam)).astype(np.float32)
    bll = np.linalg.norm(u.astype(np.float64), axis=1).astype(np.float32)
    uvw = np.concatenate([u, -u])
    xyza = np.concatenate([rows_a, rows_a]).astype(np.float32)
    xyzb = np.concatenate([rows_b, rows_b]).astype(np.float32)
    bll2 = np.concatenate([bll, bll])
    return dict(theta=theta, phi=phi, B=B, uvw=uvw, xyza=xyza, xyzb=xyzb, bll=bll2)


def _dir_to_theta_phi(s):
    """HEALPix-style (theta, phi) whose (l, m, n) = (sin t cos p, -sin t sin p,
    cos t) is the unit vector s (the convention of vissgen3d_blockage.cu:53-74)."""
    th = math.acos(max(-1.0, min(1.0, float(s[2]))))
    ph = math.atan2(-float(s[1]), float(s[0])) % (2 * math.pi)
    return th, ph


LIMB_TARGETS = (-2e-6, -6e-7, -2e-7, -6e-8, 0.0, 0.0, 6e-8, 2e-7, 6e-7, 2e-6)


def make_limb_case(seed: int = 7, targets=LIMB_TARGETS, probe_sky: float = 40.0):
    """The small case of make_case (every HEALPix pixel >= 1e-4 from every
    occultation cone), with len(targets) pixels moved onto the cone of one
    (snapshot, satellite) each: their FP64 predicate margin
    s.P/|P| - cos(phi) is the target (as realised after the FP32 rounding of
    the text inputs), and they stay >= 2e-5 from every other satellite's cone.
    For such probes the reference's FP32 acosf predicate
    (vissgen3d_blockage.cu:88-94) and the FP64 dot product may disagree.
    Every probe is seen by another satellite of its snapshot, so its bit
    shows in the reference's forward visibilities and hence in its image."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    from oracle import oracle as O

    case = make_case(seed=seed)
    n = case["uvw"].shape[0] // 2
    npix = case["B"].size
    thr = O.cone_threshold(np.float32(1737.1e3), np.float32(300e3))
    # the distinct satellite positions (snapshot-major), as the rows hold them
    P = np.concatenate([case["xyza"][:n], case["xyzb"][:n]]).astype(np.float64)
    Pu, first = np.unique(P, axis=0, return_index=True)
    Pu = P[np.sort(first)]
    q = Pu / np.linalg.norm(Pu, axis=1, keepdims=True)
    rng = np.random.default_rng(seed + 100)
    theta, phi, B = case["theta"].copy(), case["phi"].copy(), case["B"].copy()
    slots = np.linspace(3, npix - 5, len(targets)).astype(int)
    owners = rng.choice(len(Pu), len(targets), replace=False)
    for slot, g, target in zip(slots, owners, targets):
        qg = q[g]
        # rows (a, b) of this satellite: the partners that must see the probe
        partners = [i for i in range(len(Pu)) if i != g and np.linalg.norm(Pu[i] - Pu[g]) < 5e3]
        for _attempt in range(20000):
            w = rng.standard_normal(3)
            w -= (w @ qg) * qg
            w /= np.linalg.norm(w)
            c = thr + target
            s = c * qg + math.sqrt(1.0 - c * c) * w
            th, ph = _dir_to_theta_phi(s)
            th32, ph32 = np.float32(th), np.float32(ph)
            lmn, _ = O.sky_pre_f32(np.array([th32]), np.array([ph32]), np.array([1.0], np.float32),
                                   np.float32(1.0))
            d = lmn[0] @ q.T - thr
            others = np.delete(np.abs(d), g)
            if (abs(d[g] - target) <= 1.5e-7 and others.min() > 2e-5
                    and any(d[i] > 2e-5 for i in partners)):
                theta[slot], phi[slot] = th32, ph32
                B[slot] = np.float32(probe_sky)
                break
        else:
            raise RuntimeError("no probe direction found")
    case = dict(case, theta=theta, phi=phi, B=B)
    case["probes"] = slots
    return case


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


def make_days_1m(days: int = 3):
    """Three distinct days of the 1 MHz programs (vissgen3d_*, not _10m): the
    same sky, a wider formation (0.4-2.5 km gaps, so |u| reaches ~20
    wavelengths at 300 m) on a new seed each day; every (row, pixel) still
    >= 1e-4 from the occultation cone."""
    cases = [make_case(seed=20 + d, spacing=(400.0, 2500.0), cross_sigma=300.0, frequency=1e6)
             for d in range(days)]
    sky = {k: cases[0][k] for k in ("theta", "phi", "B")}
    return [dict(c, **sky) for c in cases]


def read_inputs(root: str, variant_10m: bool = True, day: int = 1):
    d = os.path.join(root, "earth_10Mhz" if variant_10m else "earth_1Mhz")
    suffix = "_10Mhz.txt" if variant_10m else ".txt"
    Bf = np.loadtxt(os.path.join(d, "B" + suffix), dtype=np.float32)
    case = dict(B=Bf[1:], theta=np.loadtxt(os.path.join(d, "theta_heal" + suffix), dtype=np.float32),
                phi=np.loadtxt(os.path.join(d, "phi_heal" + suffix), dtype=np.float32))
    for name in ("uvw", "xyza", "xyzb"):
        case[name] = np.loadtxt(os.path.join(d, f"{name}{day}day1M.txt"), dtype=np.float32)[1:]
    case["bll"] = np.loadtxt(os.path.join(d, f"bll{day}day1M.txt"), dtype=np.float32)[1:]
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


# ------------------------------------------------- limb: the reference's bits
def satellite_table(case):
    """Distinct satellite positions of the day's unique rows (FP64 from the
    FP32 text), each row's two satellites as indices into them, and the
    unit directions q = P/|P| of the reference's cone test."""
    n = case["uvw"].shape[0] // 2
    P = np.concatenate([case["xyza"][:n], case["xyzb"][:n]]).astype(np.float64)
    Pu, inv = np.unique(P, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    q = Pu / np.linalg.norm(Pu, axis=1, keepdims=True)
    return Pu, q, inv[:n], inv[n:]


def satellite_margins(case):
    """(lmn, margin) with margin[j, g] = s_j . q_g - cos(phi): the FP64
    predicate's distance from the reference's cone (visible iff >= 0) for
    every pixel j and distinct satellite g."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    from oracle import oracle as O
    npix = case["B"].size
    lmn, _ = O.sky_pre_f32(case["theta"], case["phi"], case["B"], np.float32(4 * math.pi / npix))
    _Pu, q, _a, _b = satellite_table(case)
    thr = O.cone_threshold(np.float32(1737.1e3), np.float32(300e3))
    d = np.stack([O.dots(lmn, np.append(qg, 0.0)) for qg in q], axis=1) - thr
    return lmn, d


def vissgen_with_visibility(case, vis, frequency: float = 1e7):
    """The noblockage program's day (vissgen3d_noblockage.cu:195-563) in FP64
    for an explicit per-satellite visibility vis[j, g] (pixel j seen from
    distinct satellite g): the forward's row mask is vis[:, a_i] & vis[:, b_i]
    (:88-94), the imaging adjoint is unmasked (:167-182).  Returns (V of the
    unique rows before the w-rotation, Re C per pixel)."""
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
    _Pu, _q, a, b = satellite_table(case)
    M = (vis[:, a] & vis[:, b]).T                                    # (amount, npix)
    ph = uvw[:amount] @ lmn.T - w[:amount, None]
    V = np.zeros(n, np.complex128)
    V[:amount] = ((Bs.astype(np.float64)[None, :] * M) * np.exp(-2j * np.pi * ph)).sum(axis=1)
    V[amount:] = np.conj(V[:amount])
    V0 = V[:amount].copy()
    lam = np.float32(3e8 / np.float32(frequency))
    nr = int(np.ceil(np.float32(100e3) / lam * np.float32(2)))
    gs, _counts, dcf = O.dcf(case["bll"], nr, 1)
    V = O.wrot(w, V)
    dg = O.gamma_dg(case["uvw"][:, 2], case["bll"][:n])
    wt = O.weights(gs[:n], dg, dcf, nr)
    C = np.real(((wt.astype(np.float64) * V)[:, None] * np.exp(2j * np.pi * (uvw @ lmn.T))).sum(axis=0))
    return V0, C


def infer_limb_bits(case, C_ref, band: float = 5e-6):
    """The reference's visibility bits for the (pixel, satellite) pairs within
    `band` of the cone, recovered from its image C_ref: the image is linear
    in each such bit (the bit only gates that pixel's term in the rows of
    that satellite), so every combination is evaluated and the one whose
    image matches C_ref best is taken.  Every pair outside the band is the
    FP64 predicate's.  Returns (pairs (j, g), margins, reference bits, FP64
    bits, residual of the best combination, of the second best, the image
    of each single-bit flip)."""
    lmn, d = satellite_margins(case)
    vis = d >= 0.0
    pairs = [tuple(x) for x in np.argwhere(np.abs(d) <= band)]
    m = len(pairs)
    base = vis.copy()
    for j, g in pairs:
        base[j, g] = False
    _, C0 = vissgen_with_visibility(case, base)
    dC = []
    for j, g in pairs:
        v = base.copy()
        v[j, g] = True
        dC.append(vissgen_with_visibility(case, v)[1] - C0)
    dC = np.array(dC).reshape(m, -1)
    combos = ((np.arange(2 ** m)[:, None] >> np.arange(m)[None, :]) & 1).astype(np.float64)
    images = C0[None, :] + combos @ dC
    res = np.linalg.norm(images - C_ref[None, :], axis=1) / np.linalg.norm(C_ref)
    order = np.argsort(res)
    best = combos[order[0]].astype(bool)
    ours = np.array([vis[j, g] for j, g in pairs], dtype=bool)
    margins = np.array([d[j, g] for j, g in pairs])
    return pairs, margins, best, ours, float(res[order[0]]), float(res[order[1]]) if m else np.inf, dC
