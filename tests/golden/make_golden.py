"""Freezes the reference's output for every case of tests/cases.py.

Runs the reference setup.out / core.out (built from the reference sources by
oracle/Makefile into oracle/_ref) on each case's initial state and stores the
final markers, E, H and the diag.dat energy rows in tests/golden/<case>.npz;
for two cases also the Gauss-law rows of core_gauss.out in
tests/golden/gauss_<case>.npz, and the fields of an empty Mur box driven by
the hard gauss-spot source in tests/golden/gauss_spot.npz.

    make -C oracle ref REF=/path/to/reference
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import cases  # noqa: E402
import oracle_port  # noqa: E402
from refrun import RefRun, have_reference  # noqa: E402


def make(name):
    case = cases.CASES[name]
    n, L_um = cases.geometry(case)
    rr = RefRun()
    try:
        dom = rr.setup(n, L_um, -0.5, case["bc_min"], case["bc_max"])
        h, tau = dom["h"], dom["tau"]
        m0 = oracle_port.place(**cases.placer_args(case, h))
        E0, H0 = cases.initial_fields(case, h)
        rr.set_state(m0, E0, H0)
        rr.run(case["steps"])
        m, E, H = rr.final()
        diag = rr.diag()
        np.savez_compressed(os.path.join(HERE, name + ".npz"), h=h, tau=tau,
                            n_markers0=len(m0), markers=m.tobytes(), E=E, H=H, diag=diag)
        print("%-18s markers %d -> %d, diag rows %d" % (name, len(m0), len(m), len(diag)))
    finally:
        rr.cleanup()


def make_gauss(name):
    """The reference built with MC_GAUSS_TEST (core_gauss.out) on the case:
    its output/gauss_test.dat rows {t, deltaRho_J, deltaRho_E}."""
    case = cases.CASES[name]
    n, L_um = cases.geometry(case)
    rr = RefRun()
    try:
        dom = rr.setup(n, L_um, -0.5, case["bc_min"], case["bc_max"])
        h = dom["h"]
        m0 = oracle_port.place(**cases.placer_args(case, h))
        E0, H0 = cases.initial_fields(case, h)
        rr.set_state(m0, E0, H0)
        rr.run(case["steps"], exe="core_gauss.out")
        rows = np.loadtxt(rr.path("output", "gauss_test.dat"), skiprows=1, ndmin=2)
        np.savez_compressed(os.path.join(HERE, "gauss_" + name + ".npz"), rows=rows)
        print("%-18s gauss rows %d" % (name, len(rows)))
    finally:
        rr.cleanup()


GAUSS_CASES = ("periodic_thermal", "mur_mixed")

# Hard gauss-spot source in an empty Mur box (core/em_gaussSpot.c).
SPOT_N = (20, 16, 16)
SPOT_L_UM = (1.0, 0.8, 0.8)
SPOT_STEPS = 40


def spot_params(h):
    return dict(ampl=2.0, frequency=1.0, x=6 * h[0], y=0.4, z=0.4, width=0.2, duration=0.3,
                front_offset=0.4, t_plateau=0.1, ey=1, ez=-1)


def make_gauss_spot():
    rr = RefRun()
    try:
        dom = rr.setup(SPOT_N, SPOT_L_UM, -0.5, (2, 2, 2), (2, 2, 2))
        h, tau = dom["h"], dom["tau"]
        rr.set_state(np.zeros(0, dtype=oracle_port.MARKER_DTYPE))
        rr.set_gauss_spot(**spot_params(h))
        rr.run(SPOT_STEPS)
        m, E, H = rr.final()
        np.savez_compressed(os.path.join(HERE, "gauss_spot.npz"), h=h, tau=tau, E=E, H=H, diag=rr.diag())
        print("gauss_spot: E max %.3e" % np.max(np.abs(E)))
    finally:
        rr.cleanup()


if __name__ == "__main__":
    if not have_reference():
        sys.exit("reference binaries missing: make -C oracle ref REF=<reference tree>")
    for name in (sys.argv[1:] or list(cases.CASES) + ["gauss_spot"]):
        if name == "gauss_spot":
            make_gauss_spot()
            continue
        make(name)
        if name in GAUSS_CASES:
            make_gauss(name)
