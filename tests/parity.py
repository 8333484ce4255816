"""Comparison helpers for parity tests (test infrastructure)."""
import numpy as np

import cases
from refrun import MARKER_DTYPE


def load_golden(name):
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", name + ".npz")
    z = np.load(path)
    m = np.frombuffer(z["markers"].tobytes(), MARKER_DTYPE).copy()
    return {"h": z["h"], "tau": float(z["tau"]), "markers": m, "E": z["E"], "H": z["H"],
            "diag": z["diag"], "n_markers0": int(z["n_markers0"])}


def rel_err(a, b):
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) / scale


def by_id(m):
    return np.sort(np.asarray(m, MARKER_DTYPE), order="id")


def compare_markers(got, want, h, pos_tol=1e-12, mom_tol=1e-12):
    """Markers matched by id: same set of ids, same cell indices (bit-exact),
    positions and momenta within the given tolerances."""
    g, w = by_id(got), by_id(want)
    assert len(g) == len(w), "marker count %d != %d" % (len(g), len(w))
    assert np.array_equal(g["id"], w["id"]), "marker id sets differ"
    for a, ax in enumerate("xyz"):
        cg = np.floor(g[ax] / h[a]).astype(np.int64)
        cw = np.floor(w[ax] / h[a]).astype(np.int64)
        assert np.array_equal(cg, cw), "cell index along %s differs for %d markers" % (
            ax, int(np.sum(cg != cw)))
        err = float(np.max(np.abs(g[ax] - w[ax]))) if len(g) else 0.0
        assert err <= pos_tol * max(h[a], 1e-300) * 1e3, "position %s off by %g" % (ax, err)
    umax = max(float(np.max(np.abs(np.stack([w["vx"], w["vy"], w["vz"]])))) if len(w) else 1.0, 1e-300)
    for ax in ("vx", "vy", "vz"):
        err = float(np.max(np.abs(g[ax] - w[ax]))) if len(g) else 0.0
        assert err <= mom_tol * umax, "momentum %s off by %g (scale %g)" % (ax, err, umax)
    assert np.array_equal(g["rho"], w["rho"]) and np.array_equal(g["qDivM"], w["qDivM"])


def initial_state(name, h):
    import oracle_port
    case = cases.CASES[name]
    m0 = oracle_port.place(**cases.placer_args(case, h))
    E0, H0 = cases.initial_fields(case, h)
    return case, m0, E0, H0
