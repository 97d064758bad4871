#!/usr/bin/env python3
"""Generate the golden fixtures of tests/golden/ref_noblockage_10m/.

Writes the small synthetic case of refcase.py in the reference's text formats,
runs the reference's own vissgen3d_noblockage_10m program (built unmodified
from its sources by oracle/build_ref.sh) on it -- on a GPU host, since the
reference is CUDA-only -- and keeps its inputs, its output C1day1M.txt and
its stdout (which prints Viss[0..2], the forward visibilities before the
w-rotation).

    python tests/golden/make_reference_fixtures.py --out DIR [--ref PATH] [--case limb]

--case golden (default) writes the case of refcase.make_case (every pixel at
least 1e-4 from every occultation cone); --case limb the case of
refcase.make_limb_case (ten bright probe pixels placed 3e-8 to 2e-6 from one
satellite's cone each), also listing the probes in probes.json.  Both run the
10 MHz program.  --case golden1m runs the 1 MHz vissgen3d_noblockage on the
three days of refcase.make_days_1m; that program loops over 450 days, so days
4-450 are written as copies of day 1 for the run, and only days 1-3 (inputs,
images and the first lines of stdout) are kept.
"""
import argparse
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

import refcase  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--ref", default=os.path.join(ROOT, "oracle", "_ref", "vissgen3d_noblockage_10m"))
    ap.add_argument("--case", choices=["golden", "limb", "golden1m"], default="golden")
    args = ap.parse_args()
    if args.case == "golden1m":
        return golden_1m(args)
    case = refcase.make_case() if args.case == "golden" else refcase.make_limb_case()
    with tempfile.TemporaryDirectory() as tmp:
        refcase.write_inputs(case, tmp, variant_10m=True)
        if "probes" in case:
            import json
            with open(os.path.join(tmp, "probes.json"), "w") as f:
                json.dump({"probe_pixels": [int(x) for x in case["probes"]],
                           "targets": [float(x) for x in refcase.LIMB_TARGETS]}, f)
        os.makedirs(os.path.join(tmp, "3dnoblockage10M"))
        r = subprocess.run([args.ref], cwd=tmp, capture_output=True, text=True, timeout=600)
        with open(os.path.join(tmp, "reference_stdout.txt"), "w") as f:
            f.write(r.stdout)
        if r.returncode != 0:
            sys.stderr.write(r.stdout[-2000:] + r.stderr[-2000:])
            sys.exit(r.returncode)
        out = os.path.abspath(args.out)
        if os.path.exists(out):
            shutil.rmtree(out)
        shutil.copytree(tmp, out)
    print("fixtures in", out)


def golden_1m(args):
    ref = args.ref.replace("vissgen3d_noblockage_10m", "vissgen3d_noblockage")
    days = refcase.make_days_1m()
    with tempfile.TemporaryDirectory() as tmp:
        for d, case in enumerate(days, start=1):
            refcase.write_inputs(case, tmp, variant_10m=False, day=d)
        data = os.path.join(tmp, "earth_1Mhz")
        for d in range(len(days) + 1, 451):       # the program's 450 days
            for name in ("uvw", "xyza", "xyzb", "bll"):
                shutil.copyfile(os.path.join(data, f"{name}1day1M.txt"), os.path.join(data, f"{name}{d}day1M.txt"))
        os.makedirs(os.path.join(tmp, "3dnoblockage"))
        r = subprocess.run([ref], cwd=tmp, capture_output=True, text=True, timeout=1200)
        if r.returncode != 0:
            sys.stderr.write(r.stdout[-2000:] + r.stderr[-2000:])
            sys.exit(r.returncode)
        out = os.path.abspath(args.out)
        if os.path.exists(out):
            shutil.rmtree(out)
        os.makedirs(os.path.join(out, "earth_1Mhz"))
        os.makedirs(os.path.join(out, "3dnoblockage"))
        keep = ["B.txt", "theta_heal.txt", "phi_heal.txt"] + [
            f"{n}{d}day1M.txt" for d in range(1, len(days) + 1) for n in ("uvw", "xyza", "xyzb", "bll")]
        for f in keep:
            shutil.copyfile(os.path.join(data, f), os.path.join(out, "earth_1Mhz", f))
        for d in range(1, len(days) + 1):
            shutil.copyfile(os.path.join(tmp, "3dnoblockage", f"C{d}day1M.txt"),
                            os.path.join(out, "3dnoblockage", f"C{d}day1M.txt"))
        lines = r.stdout.splitlines()
        cut = next((i for i, ln in enumerate(lines) if "Period 4 " in ln), len(lines))
        with open(os.path.join(out, "reference_stdout_days1-3.txt"), "w") as f:
            f.write("\n".join(lines[:cut]) + "\n")
    print("fixtures in", out)


if __name__ == "__main__":
    main()
