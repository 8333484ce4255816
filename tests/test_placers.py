"""The reference placers (row a-24): fixtures of [DF:foil] (setup.out) and
of the Maxwell quiet-start pattern (the reference's sampler and mapper,
oracle/_ref/maxwell_pattern.out), and the host logic that recomputes the
expected markers for the device tests."""
import os
import subprocess
import sys

import numpy as np
import pytest

import refrun

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402


def lattice_expected(n, h, spec, pattern, id0=1):
    """[plasma] + [DF:Maxwell] markers in setup.out's order: cells I-major,
    in-cell p = ((i ny + j) nz + k) layers + l, x = (i + 1/2) h/nx + I h
    (tag_plasma.c:99-122), momenta and weight of pattern entry p."""
    nx, ny, nz, L = spec["nx"], spec["ny"], spec["nz"], spec["layers"]
    ppc = nx * ny * nz * L
    q = np.arange(ppc * n[0] * n[1] * n[2])
    cell, p = q // ppc, q % ppc
    K, J, I = cell % n[2], (cell // n[2]) % n[1], cell // (n[2] * n[1])
    s = p // L
    k, j, i = s % nz, (s // nz) % ny, s // (nz * ny)
    out = np.zeros(len(q), refrun.MARKER_DTYPE)
    for ax, (c, a, m) in enumerate(((I, i, nx), (J, j, ny), (K, k, nz))):
        d = h[ax] * 1 / float(m)
        out["xyz"[ax]] = (a + 0.5) * d + c * h[ax]
    out["vx"], out["vy"], out["vz"] = pattern[p, 0], pattern[p, 1], pattern[p, 2]
    out["rho"] = pattern[p, 3].astype(np.float32)
    out["qDivM"] = np.float32(spec["qDivM"])
    out["id"] = id0 + q
    return out


@pytest.mark.skipif(not os.path.exists(os.path.join(refrun.REF_DIR, "maxwell_pattern.out")),
                    reason="reference harness not built")
def test_maxwell_pattern_fixture_is_the_reference_sampler_output():
    g = np.load(os.path.join(HERE, "golden", "place_maxwell.npz"))
    for q, s in enumerate(make_golden.MAXWELL_SPECS):
        args = [str(s[k]) for k in ("nx", "ny", "nz", "layers", "omega_pe2", "qDivM", "ux", "uy", "uz",
                                    "tune_energy", "uniform_weight")]
        out = subprocess.run([os.path.join(refrun.REF_DIR, "maxwell_pattern.out")] + args,
                             stdout=subprocess.PIPE, check=True).stdout.decode()
        pat = np.array([[float(v) for v in line.split()] for line in out.splitlines()])
        assert np.array_equal(pat, g["pattern%d" % q])


def test_maxwell_pattern_is_mirrored_and_normalised():
    g = np.load(os.path.join(HERE, "golden", "place_maxwell.npz"))
    for q, s in enumerate(make_golden.MAXWELL_SPECS):
        pat = g["pattern%d" % q]
        ppc = s["nx"] * s["ny"] * s["nz"] * s["layers"]
        assert pat.shape == (ppc, 4)
        np.testing.assert_array_equal(pat[0::2, :3], -pat[1::2, :3])
        rho = s["omega_pe2"] * 4 * np.pi ** 2 / s["qDivM"] / ppc
        assert abs(pat[:, 3].sum() - ppc * rho) <= 1e-12 * abs(ppc * rho)


def test_foil_fixture_is_inside_its_slab():
    g = np.load(os.path.join(HERE, "golden", "place_foil.npz"))
    m = np.frombuffer(g["markers"].tobytes(), refrun.MARKER_DTYPE)
    s = make_golden.FOIL["spec"]
    assert len(m) > 500 and np.array_equal(m["id"], np.arange(1, len(m) + 1))
    l = np.array([s["lx"], s["ly"], s["lz"]]) / np.linalg.norm([s["lx"], s["ly"], s["lz"]])
    d = (m["x"] - s["x0"]) * l[0] + (m["y"] - s["y0"]) * l[1] + (m["z"] - s["z0"]) * l[2]
    assert np.all(np.abs(d - s["shift"]) <= 0.5 * s["width"] + 1e-12)
