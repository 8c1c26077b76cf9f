"""The FP64 oracle against the reference's own golden dumps (subsampled in tests/golden).

Inputs are regenerated exactly as the reference's script tests do
(tests/test-exchange/cmp-ref*.py, tests/test-demag/cmp-ref*.py); see
tests/golden/make_golden.py for the recipe and the full-dump errors.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import demag, fields, native
from tests.golden.make_golden import CELL_PROGRAM, MU0_PY, N, demag_inputs, exchange_inputs

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "golden_subsample.npz"))
SAMPLE = GOLD["sample_flat_index"]


def _rel(new, ref):
    new = new.reshape(3, -1)[:, SAMPLE]
    return float(np.abs(new - ref).max() / np.abs(ref).max()), float(np.abs(new - ref).sum(0).mean())


@pytest.fixture(scope="module")
def exch_inputs():
    return exchange_inputs()


@pytest.fixture(scope="module")
def demag_in():
    return demag_inputs()


@pytest.mark.parametrize("tag,pbc", [("", (0, 0, 0)), ("_pbc", (1, 1, 1))])
def test_exchange_matches_golden(exch_inputs, tag, pbc):
    msk, lex, m = exch_inputs
    lex0 = math.sqrt(2 * 1.3e-11 / (MU0_PY * 800e3 * 800e3))
    # the golden was produced by the kernel version with harmonic means of lex (not lex^2)
    H = fields.exchange6(m, lex, 800e3, lex0, CELL_PROGRAM, pbc, weight_power=1)
    rel, mean_abs = _rel(H, GOLD["hex_ref%s" % tag])
    assert rel < 5e-7
    # and the current (squared) weights differ from it by orders of magnitude
    H2 = fields.exchange6(m, lex, 800e3, lex0, CELL_PROGRAM, pbc, weight_power=2)
    assert _rel(H2, GOLD["hex_ref%s" % tag])[0] > 1.0


@pytest.mark.parametrize("tag,pbc,tol", [("", (0, 0, 0), 4e-7), ("_pbc", (2, 4, 8), 1.5e-6)])
def test_demag_matches_golden(demag_in, tag, pbc, tol):
    msk, m = demag_in
    logic = demag.pad_size([N, N, N], pbc)
    K = native.kernel_arne(logic, CELL_PROGRAM, pbc, 6)
    B = demag.demag_field(m, msk, 800e3, demag.kernel_spectrum(K), logic)
    rel, mean_abs = _rel(B, GOLD["B_ref%s" % tag])
    assert rel < tol
    assert mean_abs < 1e-6          # the reference test's own pass criterion


def test_kernel_arne_c_equals_numpy():
    for size, pbc in (([8, 16, 32], [0, 0, 0]), ([4, 8, 8], [2, 1, 3]), ([1, 16, 16], [0, 0, 0])):
        cs = [1e-9, 2.5e-9, 5e-9]
        a = native.kernel_arne(size, cs, pbc)
        b = demag.kernel_arne(size, cs, pbc)
        assert np.abs(a - b).max() <= 1e-11 * np.abs(b).max()


def test_golden_report_recorded():
    rep = json.load(open(os.path.join(HERE, "golden", "golden_report.json")))
    assert rep["demag"]["rel_to_max"] < 4e-7
    assert rep["exchange_weightpow1"]["rel_to_max"] < 5e-7
