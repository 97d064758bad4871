#!/usr/bin/env python3
"""Time the reference's own GPU program (vissgen3d_noblockage_10m, built
unmodified by oracle/build_ref.sh into oracle/_ref/) on benchmark-sized
synthetic inputs, on a GPU host.  Measurement infrastructure only: it runs the
reference, never this repository's kernels.

For each config it writes one observation day in the reference's text formats
(earth_10Mhz/{B,theta_heal,phi_heal}_10Mhz.txt, {uvw,xyza,xyzb,bll}1day1M.txt:
the unique rows then their conjugate mirrors, read at
vissgen3d_noblockage_10m.cu:207-225 and :302-380), runs the program in that
directory and reports its wall time.  The per-kernel device times come from an
ncu launch list of this script (one metric, one pass).

The reference sizes its shell table for baselines up to bl_max = 100 km
(vissgen3d_noblockage_10m.cu:248-250) and indexes dcf[gs] without a bound
check, so longer baselines would read past the table.  The synthetic
formations reach 126-156 km; u (and bll) are therefore scaled down to keep
every baseline under 95 km.  The satellite positions (which drive the
forward's occultation test) are unscaled, and the per-term cost of the
reference does not depend on |u|.

    python oracle/time_ref_gpu.py --configs c1,c2,c3_10mhz [--ref PATH]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# run as a script, this directory comes first on sys.path and its oracle.py
# would shadow the oracle/ directory the imports below mean
sys.path[:] = [p for p in sys.path if os.path.abspath(p or ".") != HERE]
sys.path.insert(0, ROOT)

LAMBDA_REF = float(np.float32(3e8 / 1e7))   # the program's lamda = 3e8 / frequency
BL_MAX_SAFE = 95e3                            # metres, under the program's bl_max = 100 km


def write_day(cfg_name: str, root: str) -> dict:
    from oracle import oracle as O
    from viss_optimize_3d_b200 import synth

    cfg = synth.CONFIGS[cfg_name]
    obs = synth.make_observation(cfg)
    th, ph, _ = O.pix2ang(cfg.nside)
    P = np.asarray(obs.positions, dtype=np.float64)          # (T, S, 3) metres
    pairs = np.asarray(obs.pairs)
    Pa = P[:, pairs[:, 0], :].reshape(-1, 3)
    Pb = P[:, pairs[:, 1], :].reshape(-1, 3)
    d = Pa - Pb
    scale = min(1.0, BL_MAX_SAFE / float(np.linalg.norm(d, axis=1).max()))
    u = (d * scale / LAMBDA_REF).astype(np.float32)
    bll = np.linalg.norm(u.astype(np.float64), axis=1).astype(np.float32)
    ddir = os.path.join(root, "earth_10Mhz")
    os.makedirs(ddir)
    os.makedirs(os.path.join(root, "3dnoblockage10M"))
    sky = np.asarray(obs.sky, dtype=np.float32)
    with open(os.path.join(ddir, "B_10Mhz.txt"), "w") as f:
        f.write(f"{sky.size}\n")
        np.savetxt(f, sky, fmt="%.9g")
    np.savetxt(os.path.join(ddir, "theta_heal_10Mhz.txt"), th.astype(np.float32), fmt="%.9g")
    np.savetxt(os.path.join(ddir, "phi_heal_10Mhz.txt"), ph.astype(np.float32), fmt="%.9g")
    rows = {"uvw": np.concatenate([u, -u]),
            "xyza": np.concatenate([Pa, Pa]).astype(np.float32),
            "xyzb": np.concatenate([Pb, Pb]).astype(np.float32)}
    for name, arr in rows.items():
        with open(os.path.join(ddir, name + "1day1M.txt"), "w") as f:
            f.write("0 0 0\n")                                   # first row, skipped
            np.savetxt(f, arr, fmt="%.9g")
    with open(os.path.join(ddir, "bll1day1M.txt"), "w") as f:
        f.write("0\n")                                           # first token, skipped
        np.savetxt(f, np.concatenate([bll, bll]), fmt="%.9g")
    return {"config": cfg_name, "npix": int(sky.size), "unique_rows": int(u.shape[0]),
            "rows": int(2 * u.shape[0]), "u_scale": scale}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--configs", default="c1,c2,c3_10mhz")
    ap.add_argument("--ref", default=os.path.join(HERE, "_ref", "vissgen3d_noblockage_10m"))
    ap.add_argument("--timeout", type=float, default=900.0)
    args = ap.parse_args()
    if not os.path.exists(args.ref):
        sys.exit(f"reference program not built: {args.ref} (run oracle/build_ref.sh)")
    for name in args.configs.split(","):
        with tempfile.TemporaryDirectory() as tmp:
            info = write_day(name, tmp)
            t0 = time.perf_counter()
            r = subprocess.run([args.ref], cwd=tmp, capture_output=True, text=True,
                               timeout=args.timeout)
            info["wall_s"] = round(time.perf_counter() - t0, 3)
            info["returncode"] = r.returncode
            out = os.path.join(tmp, "3dnoblockage10M", "C1day1M.txt")
            info["output_lines"] = sum(1 for _ in open(out)) if os.path.exists(out) else 0
            info["terms_forward"] = info["unique_rows"] * info["npix"]
            info["terms_adjoint_reference"] = info["rows"] * info["npix"]
            print(json.dumps(info), flush=True)
            if r.returncode != 0:
                sys.stderr.write(r.stdout[-2000:] + r.stderr[-2000:])
                sys.exit(r.returncode)


if __name__ == "__main__":
    main()
