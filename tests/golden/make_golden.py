"""Freezes the reference's output for every case of tests/cases.py.

Runs the reference setup.out / core.out (built from the reference sources by
oracle/Makefile into oracle/_ref) on each case's initial state and stores the
final markers, E, H and the diag.dat energy rows in tests/golden/<case>.npz;
for two cases also the Gauss-law rows of core_gauss.out in
tests/golden/gauss_<case>.npz.

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


if __name__ == "__main__":
    if not have_reference():
        sys.exit("reference binaries missing: make -C oracle ref REF=<reference tree>")
    for name in (sys.argv[1:] or list(cases.CASES)):
        make(name)
        if name in GAUSS_CASES:
            make_gauss(name)
