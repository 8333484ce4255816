"""The CPU restatement (oracle/pic_oracle.c) against the reference on the
runs at the benchmark configurations' sizes and the field-only runs:
the cavity resonator set up by the reference's [EMResonator] tag, a free
pulse absorbed by Mur walls on all six faces, BASELINE configuration 1 (the
32^3 thermal plasma, 200 steps) and the grid and foil of configuration 2
(256 x 128 x 128, 4.46e6 markers, 10 steps).  The reference's outputs are
frozen in tests/golden/{resonator,mur_pulse,thermal_c1,foil_c2}.npz by
tests/golden/make_golden.py; these tests pin the restatement the GPU tests
of the same runs are also checked against."""
import os

import numpy as np
import pytest

import cases
import oracle_port
from refrun import MARKER_DTYPE

HERE = os.path.dirname(os.path.abspath(__file__))


def golden(name):
    return np.load(os.path.join(HERE, "golden", name + ".npz"))


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def diag_close(rows, diag, cols=5, tol=2e-6):
    """Energy rows against diag.dat, which prints 7 significant digits
    (core/diag_WDensity.c:103-104): within 2e-6 of each quantity's largest
    magnitude.  diag.dat row s is the step after row s of the run."""
    for q in range(cols):
        scale = max(float(np.max(np.abs(diag[:, 1 + q]))), 1e-300)
        err = float(np.max(np.abs(rows[1:len(diag) + 1, q] - diag[:, 1 + q]))) / scale
        assert err < tol, (q, err)


def test_resonator_restatement():
    g = golden("resonator")
    c = cases.RESONATOR
    o = oracle_port.OracleRun(c["n"], g["h"], float(g["tau"]), c["bc"], c["bc"])
    o.set_fields(g["E0"], g["H0"])
    o.init()
    rows = o.step(c["steps"])
    E, H = o.fields()
    assert rel(E, g["E"]) < 1e-12 and rel(H, g["H"]) < 1e-12
    diag_close(rows, g["diag"], cols=2)


def test_mur_pulse_restatement():
    g = golden("mur_pulse")
    c = cases.MUR_PULSE
    E0, H0 = cases.mur_pulse_fields()
    o = oracle_port.OracleRun(c["n"], g["h"], float(g["tau"]), c["bc"], c["bc"])
    o.set_fields(E0, H0)
    o.init()
    rows = []
    for q in range(1, c["records"] + 1):
        rows.append(o.step(c["period"]))
        E, H = o.fields()
        assert rel(E, g["E%d" % q]) < 1e-12 and rel(H, g["H%d" % q]) < 1e-12, q
    diag_close(np.concatenate(rows), g["diag"], cols=2)


def test_thermal_c1_restatement():
    g = golden("thermal_c1")
    c = cases.THERMAL_C1
    n, h = c["n"], g["h"]
    o = oracle_port.OracleRun(n, h, float(g["tau"]), c["bc"], c["bc"])
    z = np.zeros((n[0] + 1, n[1] + 1, n[2] + 1, 3))
    o.set_fields(z, z)
    o.set_markers(cases.thermal_c1_markers(h))
    o.init()
    rows = o.step(c["steps"])
    diag_close(rows, g["diag"])
    E, H = o.fields()
    sel = tuple(g["nodes"].T)
    assert rel(E[sel], g["E"]) < 1e-12 and rel(H[sel], g["H"]) < 1e-12
    for F, key in ((E, "spec_E"), (H, "spec_H")):
        s = cases.shell_spectrum(F, n)
        assert np.max(np.abs(s - g[key]) / g[key].max(axis=1, keepdims=True)) < 1e-12
    m = np.sort(o.markers(), order="id")
    want = np.frombuffer(g["markers"].tobytes(), MARKER_DTYPE)
    got = m[(m["id"] - 1) % c["sample_every"] == 0]
    assert np.array_equal(got["id"], want["id"])
    for f in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.max(np.abs(got[f] - want[f])) < 1e-15, f


@pytest.mark.timeout(300)
def test_foil_c2_restatement():
    g = golden("foil_c2")
    c = cases.FOIL_C2
    n, h = c["n"], g["h"]
    o = oracle_port.OracleRun(n, h, float(g["tau"]), c["bc"], c["bc"])
    z = np.zeros((n[0] + 1, n[1] + 1, n[2] + 1, 3))
    o.set_fields(z, z)
    o.set_markers(cases.foil_c2_markers(h))
    o.init()
    rows = o.step(c["steps"])
    diag_close(rows, g["diag"])
    E, H = o.fields()
    sel = tuple(g["nodes"].T)
    for q in range(3):
        assert np.max(np.abs(E[sel][:, q] - g["E"][:, q])) < 1e-12 * g["E_max"][q]
        assert np.max(np.abs(H[sel][:, q] - g["H"][:, q])) < 1e-12 * g["H_max"][q]
    m = np.sort(o.markers(), order="id")
    want = np.frombuffer(g["markers"].tobytes(), MARKER_DTYPE)
    got = m[(m["id"] - 1) % c["sample_every"] == 0]
    assert np.array_equal(got["id"], want["id"])
    for a, f in enumerate("xyz"):
        assert np.array_equal(np.floor(got[f] / h[a]), np.floor(want[f] / h[a]))
    for f in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.max(np.abs(got[f] - want[f])) < 1e-12 * max(np.max(np.abs(want[f])), 1.0), f
