"""The drop-in executables (same command lines, CWD-relative text inputs and
output directories as the reference's vissgen3d_* and pix2ang programs) on a
small synthetic case, against the FP64 oracle's restatement of vissGen
(vissgen3d_blockage.cu:195-563).  Outputs are 6-significant-digit text, as the
reference writes them (:549), so values are compared at 2e-5 of the largest."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "viss_optimize_3d_b200", "bin")
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import refcase  # noqa: E402


def run(exe, cwd, *args):
    r = subprocess.run([os.path.join(BIN, exe), *args], cwd=cwd, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return r.stdout


def viss_lines(stdout):
    out = []
    for m in re.finditer(r"Viss\[(\d)\]: \(([^,]+),([^)]+)\)", stdout):
        out.append(complex(float(m.group(2)), float(m.group(3))))
    return np.array(out)


@pytest.mark.parametrize("exe,blockage", [("vissgen3d_noblockage_10m", False),
                                          ("vissgen3d_blockage_10m", True)])
def test_vissgen_10m(tmp_path, oracle, exe, blockage):
    case = refcase.make_case()
    refcase.write_inputs(case, str(tmp_path), variant_10m=True)
    outdir = "3dblockage10M" if blockage else "3dnoblockage10M"
    os.makedirs(tmp_path / outdir)
    stdout = run(exe, tmp_path)                        # no arguments, like the reference
    C = np.loadtxt(tmp_path / outdir / "C1day1M.txt")
    V0, Co = refcase.oracle_vissgen(case, blockage)
    assert C.shape == Co.shape
    assert np.abs(C - Co).max() <= 2e-5 * np.abs(Co).max(), np.abs(C - Co).max()
    V = viss_lines(stdout)
    assert V.size == 3
    np.testing.assert_allclose(V, V0[:3], rtol=2e-5, atol=2e-5 * np.abs(V0).max())
    assert "npix: 192" in stdout and "total time:" in stdout


def test_ref_dcf_shift(tmp_path, oracle):
    """--ref-dcf-shift: the blockage program's own (shifted) DCF table.  A
    compact formation (baselines of 1-3 wavelengths) over 40 snapshots fills
    the inner shells, so the weights sit below the 1/8 clamp and the shift
    shows in the image."""
    case = refcase.make_case(n_snap=40, spacing=(5.0, 20.0), cross_sigma=5.0)
    refcase.write_inputs(case, str(tmp_path), variant_10m=True)
    os.makedirs(tmp_path / "3dblockage10M")
    run("vissgen3d_blockage_10m", tmp_path, "--ref-dcf-shift")
    C = np.loadtxt(tmp_path / "3dblockage10M" / "C1day1M.txt")
    _, Co = refcase.oracle_vissgen(case, True, dcf_shift=True)
    _, Cu = refcase.oracle_vissgen(case, True)
    assert np.abs(C - Co).max() <= 2e-5 * np.abs(Co).max(), np.abs(C - Co).max()
    assert np.abs(Co - Cu).max() > 1e-3 * np.abs(Cu).max()    # the shift is visible in the image


def test_vissgen_1m_two_days(tmp_path, oracle):
    case = refcase.make_case()
    refcase.write_inputs(case, str(tmp_path), variant_10m=False)
    os.makedirs(tmp_path / "3dblockage")
    stdout = run("vissgen3d_blockage", tmp_path, "--days", "2")
    C1 = np.loadtxt(tmp_path / "3dblockage" / "C1day1M.txt")
    _, Co = refcase.oracle_vissgen(case, True, frequency=1e6)
    assert np.abs(C1 - Co).max() <= 2e-5 * np.abs(Co).max()
    # day 2 has no input files: zero rows, a zero image (as the reference)
    C2 = np.loadtxt(tmp_path / "3dblockage" / "C2day1M.txt")
    assert C2.shape == Co.shape and not C2.any()
    assert "for loop: 2" in stdout


def test_pix2ang_executable(tmp_path, oracle):
    nside = 8
    npix = 12 * nside * nside
    with open(tmp_path / "B.txt", "w") as f:
        f.write(f"{npix}\n" + "1.0\n" * npix)
    run("pix2ang", tmp_path)
    th = np.loadtxt(tmp_path / "theta_heal.txt")
    ph = np.loadtxt(tmp_path / "phi_heal.txt")
    oth, oph, _ = oracle.pix2ang(nside, nest=True)
    # 6 significant digits of text: relative error up to 5e-6
    np.testing.assert_allclose(th, oth.astype(np.float32), rtol=6e-6, atol=1e-6)
    np.testing.assert_allclose(ph, oph.astype(np.float32), rtol=6e-6, atol=1e-6)


def test_noblockage_10m_reproduces_reference_output(tmp_path):
    """Our drop-in on the inputs the reference program was run on
    (tests/golden/ref_noblockage_10m) against the reference's own output."""
    import shutil
    fix = os.path.join(ROOT, "tests", "golden", "ref_noblockage_10m")
    shutil.copytree(os.path.join(fix, "earth_10Mhz"), tmp_path / "earth_10Mhz")
    os.makedirs(tmp_path / "3dnoblockage10M")
    stdout = run("vissgen3d_noblockage_10m", tmp_path)
    C = np.loadtxt(tmp_path / "3dnoblockage10M" / "C1day1M.txt")
    Cref = np.loadtxt(os.path.join(fix, "3dnoblockage10M", "C1day1M.txt"))
    assert np.abs(C - Cref).max() <= 2e-5 * np.abs(Cref).max()
    ref_out = open(os.path.join(fix, "reference_stdout.txt")).read()
    np.testing.assert_allclose(viss_lines(stdout), viss_lines(ref_out), rtol=2e-5,
                               atol=2e-5 * np.abs(viss_lines(ref_out)).max())


def test_malformed_inputs_end_with_a_message(tmp_path):
    """Short or missing text inputs: a non-zero exit with a message naming the
    problem (the reference reads missing files as zero rows and short ones as
    garbage, vissgen3d_blockage.cu:216-237,317-326)."""
    def call(*args):
        return subprocess.run([os.path.join(BIN, "vissgen3d_blockage_10m"), *args], cwd=tmp_path,
                              capture_output=True, text=True, timeout=300)
    r = call()                                           # no earth_10Mhz/ at all
    assert r.returncode != 0 and "cannot read npix" in r.stderr
    case = refcase.make_case()
    d = refcase.write_inputs(case, str(tmp_path), variant_10m=True)
    lines = open(os.path.join(d, "theta_heal_10Mhz.txt")).read().splitlines()
    open(os.path.join(d, "theta_heal_10Mhz.txt"), "w").write("\n".join(lines[:-5]) + "\n")
    r = call()
    assert r.returncode != 0 and "fewer than npix" in r.stderr
    refcase.write_inputs(case, str(tmp_path), variant_10m=True)          # restore
    rows = open(os.path.join(d, "bll1day1M.txt")).read().splitlines()
    open(os.path.join(d, "bll1day1M.txt"), "w").write("\n".join(rows[:-7]) + "\n")
    os.makedirs(tmp_path / "3dblockage10M", exist_ok=True)
    r = call()
    assert r.returncode != 0 and "fewer rows than uvw" in r.stderr


LIMB = os.path.join(ROOT, "tests", "golden", "ref_noblockage_10m_limb")


def test_noblockage_10m_at_the_limb_differs_from_the_reference_only_by_its_fp32_bits(tmp_path, oracle):
    """The limb fixture: ten bright probe pixels 3e-8 to 2e-6 (in the cosine)
    from one satellite's occultation cone each, run through the reference's
    own vissgen3d_noblockage_10m.  Its mask bits there are recovered from its
    image (refcase.infer_limb_bits).  The drop-in applies the FP64 predicate:
    its image equals the oracle's with the FP64 bits, and differs from the
    reference's image by exactly the effect of the probes whose bits the two
    predicates set differently (2e-5 of the largest value, the text's
    precision)."""
    case = refcase.read_inputs(LIMB)
    refcase.write_inputs(case, str(tmp_path), variant_10m=True)
    os.makedirs(tmp_path / "3dnoblockage10M")
    run("vissgen3d_noblockage_10m", tmp_path)
    C = np.loadtxt(tmp_path / "3dnoblockage10M" / "C1day1M.txt")
    Cref = np.loadtxt(os.path.join(LIMB, "3dnoblockage10M", "C1day1M.txt"))
    pairs, margins, ref_bits, our_bits, r_best, _r_next, dC = refcase.infer_limb_bits(case, Cref)
    _, Co = refcase.oracle_vissgen(case, blockage=False)
    scale = np.abs(Co).max()
    assert np.abs(C - Co).max() <= 2e-5 * scale, np.abs(C - Co).max()
    flip = (our_bits.astype(float) - ref_bits.astype(float)) @ dC
    assert np.abs(C - (Cref + flip)).max() <= 4e-5 * scale, np.abs(C - (Cref + flip)).max()


FIX1M = os.path.join(ROOT, "tests", "golden", "ref_noblockage_1m")


def test_noblockage_1m_reproduces_reference_days(tmp_path, oracle):
    """The 1 MHz drop-in (vissgen3d_noblockage) against the reference's own
    1 MHz program on three days: its images C1..C3 to 2e-5 of the largest
    value (the text's precision)."""
    for d in (1, 2, 3):
        refcase.write_inputs(refcase.read_inputs(FIX1M, variant_10m=False, day=d), str(tmp_path),
                             variant_10m=False, day=d)
    os.makedirs(tmp_path / "3dnoblockage")
    run("vissgen3d_noblockage", tmp_path, "--days", "3")
    for d in (1, 2, 3):
        C = np.loadtxt(tmp_path / "3dnoblockage" / f"C{d}day1M.txt")
        Cref = np.loadtxt(os.path.join(FIX1M, "3dnoblockage", f"C{d}day1M.txt"))
        assert np.abs(C - Cref).max() <= 2e-5 * np.abs(Cref).max(), (d, np.abs(C - Cref).max())
