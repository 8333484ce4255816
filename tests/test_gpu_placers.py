"""Device placers of the reference tags against their fixtures: [DF:foil]
bit-identical to setup.out's markers, [plasma] + [DF:Maxwell] bit-identical
to the lattice and the reference sampler's pattern (tests/test_placers.py)."""
import math
import os
import sys

import numpy as np
import pytest

import refrun
from test_placers import HERE, lattice_expected, make_golden

pytestmark = pytest.mark.gpu

mg = pytest.importorskip("mandor3_b200")

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "rho", "qDivM", "id")


def foil_fixture():
    g = np.load(os.path.join(HERE, "golden", "place_foil.npz"))
    return tuple(g["h"]), float(g["tau"]), np.frombuffer(g["markers"].tobytes(), refrun.MARKER_DTYPE)


def test_foil_is_bit_identical_to_setup():
    h, tau, want = foil_fixture()
    cfg = make_golden.FOIL
    r = mg.Run(cfg["n"], h, tau, cfg["bc"], cfg["bc"])
    r.place_foil(**cfg["spec"], lambda_cm=1e-4)
    got = r.markers()
    assert len(got) == len(want)
    for f in FIELDS:
        assert np.array_equal(got[f], want[f]), f


def test_foil_in_the_precision_form():
    h, tau, want = foil_fixture()
    cfg = make_golden.FOIL
    r = mg.Run(cfg["n"], h, tau, cfg["bc"], cfg["bc"], precision=mg.FP32_OFFSET)
    r.place_foil(**cfg["spec"], lambda_cm=1e-4)
    got = r.markers()
    got = got[np.argsort(got["id"])]
    assert np.array_equal(got["id"], want["id"])
    for a, ax in enumerate("xyz"):
        assert np.array_equal(np.floor(got[ax] / h[a]), np.floor(want[ax] / h[a]))
        assert np.max(np.abs(got[ax] - want[ax])) < 1e-7 * h[a]
    for f in ("rho", "qDivM"):
        assert np.array_equal(got[f], want[f])


@pytest.mark.parametrize("q", [0, 1])
def test_maxwell_lattice_is_bit_identical(q):
    s = dict(make_golden.MAXWELL_SPECS[q])
    pattern = np.load(os.path.join(HERE, "golden", "place_maxwell.npz"))["pattern%d" % q]
    n = (8, 8, 8)
    h = (0.05, 0.05, 0.05)
    tau = 0.5 / math.sqrt(3 / 0.05 ** 2)
    r = mg.Run(n, h, tau, (0, 0, 0), (0, 0, 0))
    r.place_maxwell(**s, id0=7)
    got = r.markers()
    want = lattice_expected(n, h, s, pattern, id0=7)
    assert len(got) == len(want)
    for f in FIELDS:
        assert np.array_equal(got[f], want[f]), f
