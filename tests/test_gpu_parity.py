"""CUDA path against the reference (golden outputs of its core.out) and the
CPU restatement, through the C ABI.  FP64 form: fields within 1e-12
relative, marker cell indices bit-exact, positions and momenta within
1e-12, energy rows within 1e-12 of the restatement."""
import numpy as np
import pytest

import cases
import oracle_port
import parity

pytestmark = pytest.mark.gpu

mg = pytest.importorskip("mandor3_b200")


def gpu_run(name, g, use_graph=True):
    case, m0, E0, H0 = parity.initial_state(name, g["h"])
    r = mg.Run(case["n"], g["h"], g["tau"], case["bc_min"], case["bc_max"])
    r.set_fields(E0, H0)
    r.set_markers(m0)
    r.init()
    if use_graph:
        rows = r.step(case["steps"])
    else:
        rows = []
        for _ in range(case["steps"]):
            r.em_HHalfStep()
            we, wm = r.em_energy()
            r.plasma_move()
            wt = r.plasma_temperature()
            r.em_HStep()
            r.em_EStep_start()
            r.jbc_finish()
            r.em_EStep_finish()
            rows.append((0.0, we, wm) + tuple(wt))
        rows = np.array(rows)
    return case, r, rows


@pytest.mark.parametrize("name", sorted(cases.CASES))
@pytest.mark.parametrize("use_graph", [True, False])
def test_fp64_matches_reference(name, use_graph):
    g = parity.load_golden(name)
    case, r, rows = gpu_run(name, g, use_graph)
    E, H = r.fields()
    assert parity.rel_err(E, g["E"]) < 1e-12
    assert parity.rel_err(H, g["H"]) < 1e-12
    parity.compare_markers(r.markers(), g["markers"], g["h"], pos_tol=1e-15, mom_tol=1e-12)
    d = g["diag"]
    for c in range(5):
        np.testing.assert_allclose(rows[1:, 1 + c], d[:, 1 + c], rtol=5e-6, atol=1e-300)


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_fp64_energy_rows_match_restatement(name):
    g = parity.load_golden(name)
    case, r, rows = gpu_run(name, g, True)
    _, m0, E0, H0 = parity.initial_state(name, g["h"])
    o = oracle_port.OracleRun(case["n"], g["h"], g["tau"], case["bc_min"], case["bc_max"])
    o.set_fields(E0, H0)
    o.set_markers(m0)
    o.init()
    orows = o.step(case["steps"])
    t = g["tau"] * np.arange(case["steps"])
    np.testing.assert_allclose(rows[:, 0], t, rtol=1e-12, atol=1e-15)
    for c in range(5):
        np.testing.assert_allclose(rows[:, 1 + c], orows[:, c], rtol=1e-12, atol=1e-18)


def test_current_matches_restatement_after_one_step():
    name = "mirror_hot"
    g = parity.load_golden(name)
    case, m0, E0, H0 = parity.initial_state(name, g["h"])
    r = mg.Run(case["n"], g["h"], g["tau"], case["bc_min"], case["bc_max"])
    r.set_fields(E0, H0)
    r.set_markers(m0)
    r.init()
    r.em_HHalfStep()
    r.em_energy()
    r.plasma_move()
    r.em_HStep()
    r.em_EStep_start()
    r.jbc_finish()
    J = r.current()
    o = oracle_port.OracleRun(case["n"], g["h"], g["tau"], case["bc_min"], case["bc_max"])
    o.set_fields(E0, H0)
    o.set_markers(m0)
    o.init()
    lib = oracle_port.lib()
    import ctypes as C
    for f in ("po_em_h_half",):
        getattr(lib, f).argtypes = [C.c_void_p]
    lib.po_em_h_half(o.ptr)
    wt = np.zeros(3)
    lib.po_plasma_move.argtypes = [C.c_void_p, C.c_void_p]
    lib.po_plasma_move(o.ptr, wt.ctypes.data)
    lib.po_jbc.argtypes = [C.c_void_p]
    lib.po_jbc(o.ptr)
    Jo = o.current()
    assert parity.rel_err(J, Jo) < 1e-12


def test_laser_source_matches_restatement():
    n, h, tau = (40, 24, 24), (0.05, 0.05, 0.05), 0.5 * 0.05 / np.sqrt(3)
    bc = (2, 2, 2)
    kw = dict(a0=3.0, waist=0.4, x_focus=1.0, duration=2.0, t_start=0.0, phase=0.3,
              plane=5, margin=5)
    r = mg.Run(n, h, tau, bc, bc)
    z = np.zeros(r.field_shape())
    r.set_fields(z, z)
    r.set_laser(**kw)
    r.init()
    rows = r.step(60)
    E, H = r.fields()
    o = oracle_port.OracleRun(n, h, tau, bc, bc)
    o.set_fields(z, z)
    o.set_laser(**kw)
    o.init()
    orows = o.step(60)
    Eo, Ho = o.fields()
    assert np.max(np.abs(Eo)) > 1.0          # the pulse entered the box
    assert parity.rel_err(E, Eo) < 1e-12
    assert parity.rel_err(H, Ho) < 1e-12
    np.testing.assert_allclose(rows[:, 1], orows[:, 0], rtol=1e-12, atol=1e-20)


def test_device_placer_is_bit_exact():
    n, h = (12, 10, 16), (0.03, 0.04, 0.05)
    tau = 0.4 * min(h) / np.sqrt(3)
    r = mg.Run(n, h, tau, (0, 0, 0), (0, 0, 0))
    spec = dict(lo=(1, 2, 3), hi=(11, 9, 16), ppc=5, rho=-3.0, qDivM=-1.0,
                drift=(0.1, 0.0, -0.2), uth=(0.05, 0.02, 0.01), seed=(4321, 777), skip=12345,
                id0=100)
    r.place_uniform(**spec)
    got = parity.by_id(r.markers())
    want = parity.by_id(oracle_port.place(h=h, **spec))
    assert len(got) == len(want)
    assert np.array_equal(got["id"], want["id"])
    for ax in ("x", "y", "z", "vx", "vy", "vz", "rho", "qDivM"):
        assert np.array_equal(got[ax], want[ax]), ax          # bit-exact positions and momenta


def test_stage_order_is_enforced():
    r = mg.Run((8, 8, 8), (0.1, 0.1, 0.1), 0.02, (0, 0, 0), (0, 0, 0))
    z = np.zeros(r.field_shape())
    r.set_fields(z, z)
    with pytest.raises(mg.MandorError) as e:
        r.em_HHalfStep()            # init not called
    assert e.value.code == -4
    r.init()
    with pytest.raises(mg.MandorError) as e:
        r.em_HStep()                # out of order
    assert e.value.code == -4


def test_marker_far_outside_is_reported_not_faulted():
    n, h = (8, 8, 8), (0.1, 0.1, 0.1)
    r = mg.Run(n, h, 0.02, (0, 0, 0), (0, 0, 0))
    z = np.zeros(r.field_shape())
    r.set_fields(z, z)
    m = np.zeros(2, mg.MARKER_DTYPE)
    m["x"] = [0.35, -5 * 0.8]       # the second is four periods below the box
    m["y"] = m["z"] = 0.4
    m["rho"] = -1.0
    m["qDivM"] = -1.0
    m["id"] = [1, 2]
    r.set_markers(m)
    r.init()
    with pytest.raises(mg.MandorError) as e:
        r.step(1)
    assert e.value.code == -6


def test_graph_and_stage_paths_agree():
    name = "periodic_thermal"
    g = parity.load_golden(name)
    _, r1, rows1 = gpu_run(name, g, True)
    _, r2, rows2 = gpu_run(name, g, False)
    E1, H1 = r1.fields()
    E2, H2 = r2.fields()
    assert parity.rel_err(E1, E2) < 1e-13 and parity.rel_err(H1, H2) < 1e-13
    np.testing.assert_allclose(rows1[:, 1:], rows2[:, 1:], rtol=1e-13)
