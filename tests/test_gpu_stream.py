"""The streaming day loop (bin/vissgen_stream) over binary day files, on the GPU.

* the golden case: the reference program's own image (vissgen3d_noblockage_10m
  run on the case's text inputs, tests/golden/) reproduced through the binary
  files, within the 6-significant-digit text it was written in, and the text
  drop-in executable on the same inputs printing the very same digits;
* three synthetic days with occultation (the vissgen3d_blockage drop-in's
  arithmetic): every day image digit-for-digit equal to the text drop-in's, the
  device day sum (FP64, non-finite as 0) equal to the host sum of the day
  images, --fold-mirrors and --fp64 within 1e-5 (rel-L2) of it;
* errors: a truncated day file, a missing day, non-mirrored rows under
  --fold-mirrors, each a non-zero exit with a message (no GPU fault involved:
  all are found on the host);
* --resume: finished days are taken from their image files, a missing one is
  recomputed bit-identically, the day sum agrees;
* --gridded: the day images through the gridded adjoint (occulted and
  unmasked) within 1e-5 of the direct adjoint's.
"""
import dataclasses
import json
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

from viss_optimize_3d_b200 import dayfile, synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "viss_optimize_3d_b200", "bin")
GOLDEN = os.path.join(ROOT, "tests", "golden", "ref_noblockage_10m")
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import refcase  # noqa: E402


def run(exe, *args, cwd=None, ok=True):
    r = subprocess.run([os.path.join(BIN, exe), *map(str, args)], cwd=cwd, capture_output=True,
                       text=True, timeout=600)
    if ok:
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return r


def text_lines(path):
    with open(path) as f:
        return [line.strip() for line in f if line.strip()]


def g6(img):
    """The default 6-significant-digit ostream form the text images use."""
    return [f"{float(v):g}" for v in img]


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_golden_case_through_binary_files(tmp_path, viss):
    bind, out = tmp_path / "bin", tmp_path / "out"
    bind.mkdir()
    out.mkdir()
    run("vissgen_stream", "--convert-text", os.path.join(GOLDEN, "earth_10Mhz"), "--to", bind, "--text-10m")
    r = run("vissgen_stream", "--sky", bind / "sky.vsky", "--days-dir", bind, "--frequency", "1e7",
            "--blockage", "0", "--out-dir", out)
    info = json.loads(r.stdout.strip().splitlines()[-1])
    assert info["days"] == 1 and info["rows"] == 120 and info["npix"] == 192
    img, day, nd = dayfile.read_image(out / "C1.vimg")
    assert img.dtype == np.float32 and (day, nd) == (1, 1)
    ref = np.loadtxt(os.path.join(GOLDEN, "3dnoblockage10M", "C1day1M.txt"))
    assert img.shape == ref.shape
    assert np.abs(img - ref).max() <= 2e-5 * np.abs(ref).max(), np.abs(img - ref).max()
    # the text drop-in on the same inputs computes the same image
    txt = tmp_path / "text"
    shutil.copytree(os.path.join(GOLDEN, "earth_10Mhz"), txt / "earth_10Mhz")
    (txt / "3dnoblockage10M").mkdir()
    run("vissgen3d_noblockage_10m", cwd=txt)
    assert g6(img) == text_lines(txt / "3dnoblockage10M" / "C1day1M.txt")


@pytest.fixture(scope="module")
def three_days(tmp_path_factory, oracle):
    root = tmp_path_factory.mktemp("days")
    cfg = synth.scaled(synth.CONFIGS["c2"], nside=16, n_snap=40, n_sat=6)
    th, ph, _ = oracle.pix2ang(cfg.nside)
    sky = synth.make_observation(cfg).sky.astype(np.float32)
    (root / "bin").mkdir()
    dayfile.write_sky(root / "bin" / "sky.vsky", sky, th, ph)
    for d in (1, 2, 3):
        obs = synth.make_observation(dataclasses.replace(cfg, day=float(d - 1)))
        rows = dayfile.observation_rows(obs, 1e6)
        dayfile.write_day(dayfile.day_path(root / "bin", d), rows, day=d, frequency=1e6)
        case = dict(theta=th.astype(np.float32), phi=ph.astype(np.float32), B=sky, uvw=rows.uvw,
                    xyza=rows.xyza, xyzb=rows.xyzb, bll=rows.bll)
        refcase.write_inputs(case, str(root / "text"), variant_10m=False, day=d)
    (root / "text" / "3dblockage").mkdir()
    run("vissgen3d_blockage", "--days", "3", cwd=root / "text")
    (root / "out").mkdir()
    r = run("vissgen_stream", "--sky", root / "bin" / "sky.vsky", "--days-dir", root / "bin",
            "--days", "3", "--frequency", "1e6", "--blockage", "1", "--out-dir", root / "out",
            "--sum-out", root / "sum.vimg")
    return root, cfg, json.loads(r.stdout.strip().splitlines()[-1])


def test_days_match_the_text_drop_in(three_days):
    root, cfg, info = three_days
    assert info["days"] == 3 and [d[0] for d in info["per_day"]] == [1, 2, 3]
    assert info["rows"] == 3 * 2 * cfg.n_samples
    for d in (1, 2, 3):
        img, day, _ = dayfile.read_image(root / "out" / f"C{d}.vimg")
        assert day == d and img.size == cfg.npix
        assert g6(img) == text_lines(root / "text" / "3dblockage" / f"C{d}day1M.txt"), d


def test_device_day_sum(three_days):
    root, cfg, _ = three_days
    total, first, nd = dayfile.read_image(root / "sum.vimg")
    assert total.dtype == np.float64 and (first, nd) == (1, 3)
    host = np.zeros(cfg.npix)
    for d in (1, 2, 3):
        img = dayfile.read_image(root / "out" / f"C{d}.vimg")[0].astype(np.float64)
        host += np.where(np.isfinite(img), img, 0.0)
    assert np.array_equal(total, host)


def test_day_sum_through_the_nccl_reduce(three_days):
    """The multi-GPU path of the day sum (one NCCL reduce of the per-GPU FP64
    sums onto GPU 0), forced on one GPU as a one-rank communicator: the same
    sum, bit for bit."""
    root, cfg, _ = three_days
    total = dayfile.read_image(root / "sum.vimg")[0]
    run("vissgen_stream", "--sky", root / "bin" / "sky.vsky", "--days-dir", root / "bin", "--days", "3",
        "--frequency", "1e6", "--blockage", "1", "--nccl-reduce", "--sum-out", root / "sum_nccl.vimg")
    assert np.array_equal(dayfile.read_image(root / "sum_nccl.vimg")[0], total)


def test_fold_mirrors_and_fp64(three_days):
    root, cfg, _ = three_days
    total = dayfile.read_image(root / "sum.vimg")[0]
    base = ["--sky", root / "bin" / "sky.vsky", "--days-dir", root / "bin", "--days", "3",
            "--frequency", "1e6", "--blockage", "1"]
    run("vissgen_stream", *base, "--fold-mirrors", "--sum-out", root / "sum_fold.vimg")
    fold = dayfile.read_image(root / "sum_fold.vimg")[0]
    assert rel_l2(fold, total) <= 1e-5, rel_l2(fold, total)
    run("vissgen_stream", *base, "--fp64", "--sum-out", root / "sum_fp64.vimg")
    f64 = dayfile.read_image(root / "sum_fp64.vimg")[0]
    assert rel_l2(total, f64) <= 1e-5, rel_l2(total, f64)


def test_errors_are_reported(three_days, tmp_path):
    root, cfg, _ = three_days
    bad = tmp_path / "bad"
    shutil.copytree(root / "bin", bad)
    base = ["--sky", bad / "sky.vsky", "--days-dir", bad, "--frequency", "1e6"]
    r = run("vissgen_stream", *base, "--days", "4", ok=False)              # day 4 missing
    assert r.returncode != 0 and "cannot open" in r.stderr
    raw = open(bad / "day2.vday", "rb").read()
    open(bad / "day2.vday", "wb").write(raw[:-8])
    r = run("vissgen_stream", *base, "--days", "3", ok=False)
    assert r.returncode != 0 and "header says" in r.stderr
    rows, _, _ = dayfile.read_day(root / "bin" / "day1.vday")
    rows.uvw = rows.uvw.copy()
    rows.uvw[-1, 0] += 1.0
    dayfile.write_day(bad / "day1.vday", rows, day=1)
    r = run("vissgen_stream", *base, "--days", "1", "--fold-mirrors", ok=False)
    assert r.returncode != 0 and "exact mirrors" in r.stderr


def test_resume_skips_finished_days(three_days, tmp_path):
    """--resume: days whose image an earlier run wrote are not recomputed but
    added to the day sum from their files; a missing day image is recomputed,
    bit-identical to the first run's."""
    root, cfg, _ = three_days
    total = dayfile.read_image(root / "sum.vimg")[0]
    out = tmp_path / "out"
    shutil.copytree(root / "out", out)
    base = ["--sky", root / "bin" / "sky.vsky", "--days-dir", root / "bin", "--days", "3",
            "--frequency", "1e6", "--blockage", "1", "--out-dir", out, "--resume"]
    r = run("vissgen_stream", *base, "--sum-out", tmp_path / "s1.vimg")
    info = json.loads(r.stdout.strip().splitlines()[-1])
    assert info["resumed_days"] == 3 and info["per_day"] == []
    s1 = dayfile.read_image(tmp_path / "s1.vimg")[0]
    np.testing.assert_allclose(s1, total, rtol=1e-12, atol=1e-12 * np.abs(total).max())
    os.remove(out / "C2.vimg")
    r = run("vissgen_stream", *base, "--sum-out", tmp_path / "s2.vimg")
    info = json.loads(r.stdout.strip().splitlines()[-1])
    assert info["resumed_days"] == 2 and [d[0] for d in info["per_day"]] == [2]
    s2 = dayfile.read_image(tmp_path / "s2.vimg")[0]
    np.testing.assert_allclose(s2, total, rtol=1e-12, atol=1e-12 * np.abs(total).max())
    again = dayfile.read_image(out / "C2.vimg")[0]
    assert np.array_equal(again, dayfile.read_image(root / "out" / "C2.vimg")[0])
    r = run("vissgen_stream", "--sky", root / "bin" / "sky.vsky", "--days-dir", root / "bin",
            "--resume", ok=False)
    assert r.returncode != 0 and "--resume needs --out-dir" in r.stderr


@pytest.fixture(scope="module")
def low_freq_days(tmp_path_factory, oracle):
    """Two synthetic days at 0.1 MHz (Nside 16, 6 satellites x 40 snapshots,
    Moon): baselines short enough against the pixels for the gridded adjoint."""
    root = tmp_path_factory.mktemp("lowdays")
    cfg = synth.scaled(synth.CONFIGS["c2"], nside=16, n_snap=40, n_sat=6)
    th, ph, _ = oracle.pix2ang(cfg.nside)
    sky = synth.make_observation(cfg).sky.astype(np.float32)
    dayfile.write_sky(root / "sky.vsky", sky, th, ph)
    for d in (1, 2):
        obs = synth.make_observation(dataclasses.replace(cfg, day=float(d - 1)))
        dayfile.write_day(dayfile.day_path(root, d), dayfile.observation_rows(obs, 1e5), day=d, frequency=1e5)
    return root, cfg


def test_gridded_imaging_in_the_stream(low_freq_days, tmp_path):
    """--gridded images every day through viss_adjoint_gridded: occulted
    (hybrid) and unmasked, each day within 1e-5 (rel-L2) of the direct
    adjoint's image; with --fp64 it is refused before anything runs."""
    root, cfg = low_freq_days
    base = ["--sky", root / "sky.vsky", "--days-dir", root, "--days", "2", "--frequency", "1e5"]
    for blockage in ("1", "0"):
        outs = {}
        for mode in ("direct", "gridded"):
            out = tmp_path / f"{mode}_{blockage}"
            out.mkdir()
            extra = ["--gridded"] if mode == "gridded" else []
            run("vissgen_stream", *base, "--blockage", blockage, "--out-dir", out, *extra)
            outs[mode] = out
        for d in (1, 2):
            a = dayfile.read_image(outs["gridded"] / f"C{d}.vimg")[0].astype(np.float64)
            b = dayfile.read_image(outs["direct"] / f"C{d}.vimg")[0].astype(np.float64)
            assert rel_l2(a, b) <= 1e-5, (blockage, d, rel_l2(a, b))
    r = run("vissgen_stream", *base, "--gridded", "--fp64", ok=False)
    assert r.returncode != 0 and "--gridded" in r.stderr
