"""The reference's focused-laser soft source (scpic/em_mirror.c): the oracle
against core.out playing a mirror file made by setup.out
(tests/golden/mirror.npz, tests/golden/make_golden.py make_mirror)."""
import os
import sys

import numpy as np
import pytest

import oracle_port
import parity
import refrun

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "mirror.npz"))
BC = (2, 2, 2)


def mirror(direction):
    return refrun.read_mirror(GOLD["file%d" % direction], make_golden.MIRROR_N)


def oracle_fields(direction):
    n, h, tau = make_golden.MIRROR_N, tuple(GOLD["h"]), float(GOLD["tau"])
    o = oracle_port.OracleRun(n, h, tau, BC, BC)
    o.set_fields(np.zeros(o.shape()), np.zeros(o.shape()))
    o.set_markers(np.zeros(0, oracle_port.MARKER_DTYPE))
    vals, d, E, H = mirror(direction)
    u = GOLD["units%d" % direction]
    o.add_mirror(vals, d, u[0], u[2], E, H)
    o.init()
    o.step(make_golden.MIRROR_STEPS)
    return o.fields()


def test_mirror_file_reads():
    vals, d, E, H = mirror(1)
    assert d == 1 and vals[0] == -1.5 and vals[1] == 0.9
    assert E.shape == H.shape == ((make_golden.MIRROR_N[1] - 9) * (make_golden.MIRROR_N[2] - 9), 4)
    assert np.abs(E).max() > 0 and np.abs(H).max() > 0
    assert mirror(-1)[1] == -1


@pytest.mark.parametrize("direction", [1, -1])
def test_oracle_plays_the_reference_mirror(direction):
    E, H = oracle_fields(direction)
    wE, wH = GOLD["E%d" % direction], GOLD["H%d" % direction]
    if direction == 1:
        assert np.abs(wE).max() > 1.0
        assert parity.rel_err(E, wE) < 1e-12 and parity.rel_err(H, wH) < 1e-12
    else:
        # The reference's backward delay subtracts the focus from the cell
        # count (scpic/em_mirror.c:330): for this box the pulse peak is
        # pushed 23 periods away and nothing reaches the grid in 40 steps.
        assert np.abs(wE).max() == 0.0 and np.abs(E).max() == 0.0 and np.abs(H).max() == 0.0
