"""Binary day / sky / image files of the streaming day loop, on the CPU: the
Python writer and reader, the executable's conversion of the reference's text
day files (vissgen3d_blockage.cu:309-391 formats) and its header checks.  No
GPU: the executable's --convert-text and --info modes make no CUDA call."""
import os
import subprocess
import sys

import numpy as np
import pytest

from viss_optimize_3d_b200 import dayfile, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "viss_optimize_3d_b200", "bin", "vissgen_stream")
GOLDEN = os.path.join(ROOT, "tests", "golden", "ref_noblockage_10m")
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import refcase  # noqa: E402


def _exe(*args, ok=True):
    if not os.path.exists(EXE):
        pytest.fail(f"{EXE} is not built (python -m viss_optimize_3d_b200._build)")
    r = subprocess.run([EXE, *args], capture_output=True, text=True, timeout=120)
    if ok:
        assert r.returncode == 0, r.stdout + r.stderr
    return r


def test_python_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    rows = dayfile.DayRows(rng.standard_normal((10, 3)).astype(np.float32),
                           rng.standard_normal((10, 3)).astype(np.float32),
                           rng.standard_normal((10, 3)).astype(np.float32),
                           rng.random(10).astype(np.float32))
    dayfile.write_day(tmp_path / "d.vday", rows, day=4, frequency=1e7)
    back, day, f = dayfile.read_day(tmp_path / "d.vday")
    assert (day, f) == (4, 1e7)
    for k in ("uvw", "xyza", "xyzb", "bll"):
        assert np.array_equal(getattr(back, k), getattr(rows, k))
    assert os.path.getsize(tmp_path / "d.vday") == 64 + 10 * 10 * 4
    dayfile.write_sky(tmp_path / "s.vsky", np.ones(12), np.zeros(12), np.arange(12))
    B, th, ph = dayfile.read_sky(tmp_path / "s.vsky")
    assert B.dtype == np.float32 and np.array_equal(ph, np.arange(12, dtype=np.float32))
    img = rng.standard_normal(12)
    dayfile.write_image(tmp_path / "i.vimg", img, day=3, days=5)
    back, d0, nd = dayfile.read_image(tmp_path / "i.vimg")
    assert back.dtype == np.float64 and np.array_equal(back, img) and (d0, nd) == (3, 5)
    with pytest.raises(ValueError):
        dayfile.read_sky(tmp_path / "d.vday")          # wrong kind


def test_observation_rows_are_mirrored():
    cfg = synth.scaled(synth.CONFIGS["c2"], nside=4, n_snap=6, n_sat=4)
    rows = dayfile.observation_rows(synth.make_observation(cfg), 1e7)
    m = cfg.n_samples
    assert rows.uvw.shape == (2 * m, 3)
    assert np.array_equal(rows.uvw[m:], -rows.uvw[:m])
    assert np.array_equal(rows.xyza[m:], rows.xyza[:m]) and np.array_equal(rows.bll[m:], rows.bll[:m])


def test_convert_reference_text_files(tmp_path):
    """--convert-text reads the reference's own text inputs (here the golden
    case's) and writes the same FP32 values."""
    _exe("--convert-text", os.path.join(GOLDEN, "earth_10Mhz"), "--to", str(tmp_path), "--text-10m")
    case = refcase.read_inputs(GOLDEN)
    rows, day, _ = dayfile.read_day(tmp_path / "day1.vday")
    assert day == 1
    for k in ("uvw", "xyza", "xyzb", "bll"):
        assert np.array_equal(getattr(rows, k), case[k]), k
    B, th, ph = dayfile.read_sky(tmp_path / "sky.vsky")
    assert np.array_equal(B, case["B"]) and np.array_equal(th, case["theta"])
    assert np.array_equal(ph, case["phi"])


def test_executable_checks_headers(tmp_path):
    rows = dayfile.observation_rows(
        synth.make_observation(synth.scaled(synth.CONFIGS["c2"], nside=4, n_snap=3, n_sat=3)), 1e7)
    dayfile.write_day(tmp_path / "day2.vday", rows, day=2, frequency=1e7)
    out = _exe("--info", str(tmp_path / "day2.vday")).stdout
    assert '"kind": "VISSDAY"' in out and f'"count": {rows.uvw.shape[0]}' in out and '"day": 2' in out
    raw = open(tmp_path / "day2.vday", "rb").read()
    open(tmp_path / "short.vday", "wb").write(raw[:-4])
    r = _exe("--info", str(tmp_path / "short.vday"), ok=False)
    assert r.returncode != 0 and "header says" in r.stderr
    open(tmp_path / "bad.vday", "wb").write(b"NOTVISS\0" + raw[8:])
    r = _exe("--info", str(tmp_path / "bad.vday"), ok=False)
    assert r.returncode != 0 and "unknown file kind" in r.stderr
