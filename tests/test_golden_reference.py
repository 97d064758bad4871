"""Oracle pinned to the reference program itself (CPU).

tests/golden/ref_noblockage_10m/ holds a small synthetic case in the reference's
text formats and what the reference's own vissgen3d_noblockage_10m (built
unmodified from its sources, oracle/build_ref.sh, run on a GPU host by
tests/golden/make_reference_fixtures.py) wrote for it: 3dnoblockage10M/C1day1M.txt
and its stdout (Viss[0..2], the forward visibilities before the w-rotation).
The FP64 oracle's restatement of vissGen must reproduce both to the precision
the reference works in (FP32 arithmetic, 6-significant-digit text): 2e-5 of
the largest value.
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "ref_noblockage_10m")
sys.path.insert(0, os.path.join(HERE, "golden"))

import refcase  # noqa: E402


def reference_viss():
    text = open(os.path.join(FIX, "reference_stdout.txt")).read()
    vals = re.findall(r"Viss\[(\d)\]: \(([^,]+),([^)]+)\)", text)
    return np.array([complex(float(a), float(b)) for _, a, b in vals])


def test_fixture_inputs_are_the_generator_case():
    case = refcase.read_inputs(FIX)
    gen = refcase.make_case()
    for k in gen:
        np.testing.assert_array_equal(case[k], gen[k])


def test_oracle_reproduces_reference_image(oracle):
    case = refcase.read_inputs(FIX)
    _, C = refcase.oracle_vissgen(case, blockage=False)
    Cref = np.loadtxt(os.path.join(FIX, "3dnoblockage10M", "C1day1M.txt"))
    assert Cref.shape == C.shape == (192,)
    assert np.abs(C - Cref).max() <= 2e-5 * np.abs(Cref).max(), np.abs(C - Cref).max()


def test_oracle_reproduces_reference_forward(oracle):
    case = refcase.read_inputs(FIX)
    V0, _ = refcase.oracle_vissgen(case, blockage=False)
    Vref = reference_viss()
    assert Vref.size == 3
    np.testing.assert_allclose(V0[:3], Vref, rtol=2e-5, atol=2e-5 * np.abs(Vref).max())


# ------------------------------------------------------------------ the limb
LIMB = os.path.join(HERE, "golden", "ref_noblockage_10m_limb")
LIMB_BAND = 5e-6      # |s.q - cos(phi)| within which the FP32 and FP64 predicates may differ


def limb_reference_bits():
    """The reference's own visibility bits at the limb probes, recovered from
    its image (refcase.infer_limb_bits), with our FP64 predicate's bits."""
    case = refcase.read_inputs(LIMB)
    Cref = np.loadtxt(os.path.join(LIMB, "3dnoblockage10M", "C1day1M.txt"))
    return case, Cref, refcase.infer_limb_bits(case, Cref, band=LIMB_BAND)


def test_limb_fixture_inputs_are_the_generator_case():
    case = refcase.read_inputs(LIMB)
    gen = refcase.make_limb_case()
    for k in ("theta", "phi", "B", "uvw", "xyza", "xyzb", "bll"):
        np.testing.assert_array_equal(case[k], gen[k])


def test_limb_reference_bits_are_determined(oracle):
    """The reference program's image fixes its mask bit at every probe: one
    combination reproduces it to the text's precision, the next best is at
    least a hundred times worse.  Every (pixel, satellite) pair outside the band
    takes the FP64 predicate's bit (any other bit would leave a residual of
    ~1e-4 or more, far above the one accepted here)."""
    case, Cref, (pairs, margins, ref_bits, our_bits, r_best, r_next, dC) = limb_reference_bits()
    assert len(pairs) == len(refcase.LIMB_TARGETS)
    assert np.abs(margins).max() <= LIMB_BAND
    assert r_best <= 2e-5, r_best
    assert r_next >= 100 * r_best, (r_best, r_next)
    # every single flip moves the image far more than the accepted residual
    assert (np.linalg.norm(dC, axis=1) / np.linalg.norm(Cref)).min() > 100 * r_best


def test_limb_bits_agree_outside_the_fp32_error_band(oracle):
    """Where the two predicates may disagree: the reference tests acosf(s.P/|P|)
    <= phi in FP32 (vissgen3d_blockage.cu:88-94) with (l, m, n) from FP32
    sinf/cosf of its FP32 angle edits (:53-74); this repository tests
    s.P/|P| >= cos(phi) in FP64.  Their FP32 rounding moves the reference's
    boundary by a few 1e-7 in the cosine, so a bit may differ only within that
    distance of the cone: the probes at |margin| >= 5e-7 must agree."""
    case, Cref, (pairs, margins, ref_bits, our_bits, r_best, r_next, dC) = limb_reference_bits()
    far = np.abs(margins) >= 5e-7
    assert far.sum() >= 4
    np.testing.assert_array_equal(ref_bits[far], our_bits[far])


# ----------------------------------------------------- the 1 MHz program
FIX1M = os.path.join(HERE, "golden", "ref_noblockage_1m")


def test_1m_fixture_inputs_are_the_generator_days():
    for d, gen in enumerate(refcase.make_days_1m(), start=1):
        case = refcase.read_inputs(FIX1M, variant_10m=False, day=d)
        for k in ("theta", "phi", "B", "uvw", "xyza", "xyzb", "bll"):
            np.testing.assert_array_equal(case[k], gen[k])


def test_oracle_reproduces_the_1m_reference_days(oracle):
    """The reference's 1 MHz vissgen3d_noblockage (lamda = 300 m, 667 shells),
    run over its 450 days: the oracle's restatement of vissGen reproduces its
    images of days 1-3 and its printed forward visibilities of day 1."""
    for d in (1, 2, 3):
        case = refcase.read_inputs(FIX1M, variant_10m=False, day=d)
        V0, C = refcase.oracle_vissgen(case, blockage=False, frequency=1e6)
        Cref = np.loadtxt(os.path.join(FIX1M, "3dnoblockage", f"C{d}day1M.txt"))
        assert Cref.shape == C.shape == (192,)
        assert np.abs(C - Cref).max() <= 2e-5 * np.abs(Cref).max(), (d, np.abs(C - Cref).max())
        if d == 1:
            text = open(os.path.join(FIX1M, "reference_stdout_days1-3.txt")).read()
            vals = re.findall(r"Viss\[(\d)\]: \(([^,]+),([^)]+)\)", text)[:3]
            Vref = np.array([complex(float(a), float(b)) for _, a, b in vals])
            np.testing.assert_allclose(V0[:3], Vref, rtol=2e-5, atol=2e-5 * np.abs(Vref).max())
