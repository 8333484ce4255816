"""Gauss-law test (core/plasma_gaussTest.c): the oracle's charge density
(walls folded) and residual rows against the reference built with
MC_GAUSS_TEST (core_gauss.out), frozen in tests/golden/gauss_<case>.npz."""
import os

import numpy as np
import pytest

import oracle_port
import parity

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ("periodic_thermal", "mur_mixed")


def golden_rows(name):
    return np.load(os.path.join(HERE, "golden", "gauss_%s.npz" % name))["rows"]


def oracle_rows(name):
    g = parity.load_golden(name)
    case, m0, E0, H0 = parity.initial_state(name, g["h"])
    o = oracle_port.OracleRun(case["n"], g["h"], g["tau"], case["bc_min"], case["bc_max"])
    o.set_fields(E0, H0)
    o.set_markers(m0)
    o.init()
    return o.step_gauss(case["steps"])


def check_rows(got, ref):
    """The reference prints 7 significant digits; continuity residuals at
    round-off level (periodic runs) only have to stay at round-off."""
    assert got.shape == ref.shape
    np.testing.assert_allclose(got[:, 0], ref[:, 0], rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(got[:, 2], ref[:, 2], rtol=1e-6)
    scale = np.max(ref[:, 2])
    for a, b in zip(got[:, 1], ref[:, 1]):
        if b > 1e-9 * scale:
            assert abs(a - b) <= 1e-6 * b
        else:
            assert a <= 1e-9 * scale


@pytest.mark.parametrize("name", CASES)
def test_oracle_gauss_rows_match_the_reference(name):
    check_rows(oracle_rows(name), golden_rows(name))
