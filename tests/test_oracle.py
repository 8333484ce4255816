"""The CPU restatement (oracle/pic_oracle.c) pinned against the reference:
the reference's own ranmar known-answer test and golden outputs of the
reference core.out frozen in tests/golden (see tests/golden/make_golden.py)."""
import numpy as np
import pytest

import cases
import oracle_port
import parity
from refrun import MARKER_DTYPE, have_reference


def test_ranmar_known_answer():
    # misc_ranmar.c:37-56: seeds (1802, 9373), 20000 draws, then six values
    # times 4096^2.
    v = oracle_port.ranmar(1802, 9373, 20006)
    got = np.round(v[20000:] * 4096.0 * 4096.0, 1)
    assert got.tolist() == [6533892.0, 14220222.0, 7275067.0, 6172232.0, 8354498.0, 10633180.0]


def test_ranmar_values_are_multiples_of_2_pow_minus_24():
    v = oracle_port.ranmar(31328, 30081, 5000)
    assert np.all(v >= 0) and np.all(v < 1)
    assert np.all(v * 16777216.0 == np.floor(v * 16777216.0))


def test_placer_layout():
    h = (0.1, 0.2, 0.3)
    m = oracle_port.place((1, 2, 3), (3, 4, 5), 3, -1.5, -1.0, h, uth=(0.01, 0.02, 0.03), id0=7)
    assert len(m) == 2 * 2 * 2 * 3
    assert m["id"].tolist() == list(range(7, 7 + 24))
    # i-major, k-minor cell order; markers of one cell are consecutive.
    cells = np.stack([np.floor(m[a] / h[q]).astype(int) for q, a in enumerate("xyz")], 1)
    want = [(i, j, k) for i in (1, 2) for j in (2, 3) for k in (3, 4) for _ in range(3)]
    assert [tuple(c) for c in cells] == want
    # Positions are (cell + u) * h with the first three draws of each marker.
    u = oracle_port.ranmar(1802, 9373, 7 * 24).reshape(24, 7)
    assert np.array_equal(m["x"], (cells[:, 0] + u[:, 0]) * h[0])
    assert np.array_equal(m["z"], (cells[:, 2] + u[:, 2]) * h[2])
    # skip: the second half equals a placement started 7*12 draws later.
    m2 = oracle_port.place((2, 2, 3), (3, 4, 5), 3, -1.5, -1.0, h, uth=(0.01, 0.02, 0.03),
                           skip=7 * 12, id0=19)
    assert np.array_equal(m2.tobytes(), m[12:].tobytes())


def test_placer_box_muller_is_the_normal_transform():
    """The placer's own logarithm and sine/cosine (series in IEEE
    arithmetic, identical on the device) give the Box-Muller normals of the
    C library's functions to 2e-15 of their size, over 20 000 markers."""
    n = 20000
    m = oracle_port.place((0, 0, 0), (n, 1, 1), 1, -1.0, -1.0, (1.0, 1.0, 1.0), uth=(1.0, 1.0, 1.0))
    u = oracle_port.ranmar(1802, 9373, 7 * n).reshape(n, 7)
    r1, r2 = np.sqrt(-2 * np.log(1 - u[:, 3])), np.sqrt(-2 * np.log(1 - u[:, 5]))
    want = np.stack([r1 * np.cos(2 * np.pi * u[:, 4]), r1 * np.sin(2 * np.pi * u[:, 4]),
                     r2 * np.cos(2 * np.pi * u[:, 6])])
    got = np.stack([m["vx"], m["vy"], m["vz"]])
    assert np.max(np.abs(got - want)) < 2e-15 * max(1.0, np.max(np.abs(want)))
    assert abs(np.mean(got)) < 0.03 and abs(np.std(got) - 1) < 0.03


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_oracle_matches_reference_golden(name):
    g = parity.load_golden(name)
    case, m0, E0, H0 = parity.initial_state(name, g["h"])
    assert len(m0) == g["n_markers0"]
    o = oracle_port.OracleRun(case["n"], g["h"], g["tau"], case["bc_min"], case["bc_max"])
    o.set_fields(E0, H0)
    o.set_markers(m0)
    o.init()
    rows = o.step(case["steps"])
    E, H = o.fields()
    assert parity.rel_err(E, g["E"]) < 1e-13
    assert parity.rel_err(H, g["H"]) < 1e-13
    parity.compare_markers(o.markers(), g["markers"], g["h"], pos_tol=1e-15, mom_tol=1e-14)
    # diag.dat rows (t >= tau/2, printed with %e): W_E, W_M, W_Tx, W_Ty, W_Tz.
    d = g["diag"]
    ours = rows[1:]
    assert d.shape[0] == ours.shape[0]
    for c in range(5):
        np.testing.assert_allclose(ours[:, c], d[:, 1 + c], rtol=5e-6, atol=1e-300)


@pytest.mark.skipif(not have_reference(), reason="reference binaries not built")
def test_oracle_matches_live_reference_with_wall_hits():
    """A fresh case run through the reference binaries here: hot markers at
    all walls, 12 steps."""
    from refrun import RefRun
    case = dict(n=(10, 10, 12), bc_min=(2, 1, 0), bc_max=(2, 1, 0), steps=12, ppc=1,
                uth=(2.0, 2.0, 2.0), drift=(0, 0, 0), field_amp=1.5, box="full")
    n, L_um = cases.geometry(case)
    rr = RefRun()
    try:
        dom = rr.setup(n, L_um, -0.5, case["bc_min"], case["bc_max"])
        h, tau = dom["h"], dom["tau"]
        m0 = oracle_port.place(**cases.placer_args(case, h))
        E0, H0 = cases.initial_fields(case, h)
        rr.set_state(m0, E0, H0)
        rr.run(case["steps"])
        mr, Er, Hr = rr.final()
    finally:
        rr.cleanup()
    o = oracle_port.OracleRun(n, h, tau, case["bc_min"], case["bc_max"])
    o.set_fields(E0, H0)
    o.set_markers(m0)
    o.init()
    o.step(case["steps"])
    E, H = o.fields()
    assert parity.rel_err(E, Er) < 1e-13 and parity.rel_err(H, Hr) < 1e-13
    assert len(mr) < len(m0)          # the open x walls removed markers
    parity.compare_markers(o.markers(), mr, h, pos_tol=1e-15, mom_tol=1e-14)
