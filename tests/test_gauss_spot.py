"""Hard gauss-spot source (core/em_gaussSpot.c): the oracle's fields against
the reference core.out run with the same .gaussSpot.cfg, frozen in
tests/golden/gauss_spot.npz by tests/golden/make_golden.py."""
import os
import sys

import numpy as np

import oracle_port
import parity

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402


def golden():
    return np.load(os.path.join(HERE, "golden", "gauss_spot.npz"))


def test_oracle_matches_the_reference():
    g = golden()
    h, tau = tuple(g["h"]), float(g["tau"])
    o = oracle_port.OracleRun(make_golden.SPOT_N, h, tau, (2, 2, 2), (2, 2, 2))
    z = np.zeros(o.shape())
    o.set_fields(z, z)
    o.set_markers(np.zeros(0, oracle_port.MARKER_DTYPE))
    o.set_gauss_spot(**make_golden.spot_params(h))
    o.init()
    o.step(make_golden.SPOT_STEPS)
    E, H = o.fields()
    assert np.max(np.abs(g["E"])) > 0.1
    assert parity.rel_err(E, g["E"]) < 1e-12
    assert parity.rel_err(H, g["H"]) < 1e-12
