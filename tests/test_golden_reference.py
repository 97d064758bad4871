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
