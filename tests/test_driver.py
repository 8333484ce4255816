"""core_b200.out, the drop-in for the reference's core.out: it reads a
Mandor run directory (run_mandor.cfg, binData/ record 0) and writes the
reference's checkpoint records and diag.dat.

CPU part: the record-0 file set written by tests/refrun.py is accepted by the
reference core.out (skipped without oracle/_ref).  GPU part: core_b200.out on
the same directory matches the CPU restatement (and, where present, the
reference core.out) record for record."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

import cases
import oracle_port
import parity
import refrun

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "mandor3_b200", "core_b200.out")

CASE = dict(n=(12, 10, 14), bc_min=(2, 0, 1), bc_max=(2, 0, 1), steps=12, ppc=2,
            uth=(0.8, 0.8, 0.8), drift=(0.3, 0, 0), field_amp=1.0, box="full")


def prepare(root):
    n, L_um = cases.geometry(CASE)
    h = [L_um[a] / n[a] for a in range(3)]
    tau = 0.5 / np.sqrt(sum(1 / v ** 2 for v in h))
    m0 = oracle_port.place(**cases.placer_args(CASE, h))
    E0, H0 = cases.initial_fields(CASE, h)
    refrun.write_checkpoint0(root, n, h, tau, CASE["bc_min"], CASE["bc_max"], E0, H0, m0)
    refrun.write_run_cfg(root, CASE["steps"], 5)
    return n, h, tau, m0, E0, H0


def oracle(n, h, tau, m0, E0, H0, steps):
    o = oracle_port.OracleRun(n, h, tau, CASE["bc_min"], CASE["bc_max"])
    o.set_fields(E0, H0)
    o.set_markers(m0)
    o.init()
    rows = o.step(steps)
    E, H = o.fields()
    return rows, E, H, o.markers()


def read_record(root, k):
    b = os.path.join(root, "binData")
    m = refrun.read_markers(os.path.join(b, "plasma_%06d_000.bin" % k))
    _, _, E = refrun.read_mesh(os.path.join(b, "sys_E_%06d(000).bin" % k))
    _, _, H = refrun.read_mesh(os.path.join(b, "sys_H_%06d(000).bin" % k))
    return m, E, H


@pytest.mark.skipif(not refrun.have_reference(), reason="reference binaries not built")
def test_reference_core_reads_our_record_zero():
    root = tempfile.mkdtemp(prefix="mg_drv_")
    try:
        rr = refrun.RefRun(root)
        n, h, tau, m0, E0, H0 = prepare(root)
        rr._run("core.out")
        m, E, H = read_record(root, 3)          # records at steps 5, 10, final 12
        rows, Eo, Ho, mo = oracle(n, h, tau, m0, E0, H0, CASE["steps"])
        assert parity.rel_err(E, Eo) < 1e-12 and parity.rel_err(H, Ho) < 1e-12
        parity.compare_markers(m, mo, h, pos_tol=1e-15, mom_tol=1e-12)
    finally:
        shutil.rmtree(root, ignore_errors=True)


@pytest.mark.gpu
def test_driver_writes_the_reference_records():
    root = tempfile.mkdtemp(prefix="mg_drv_")
    try:
        n, h, tau, m0, E0, H0 = prepare(root)
        out = subprocess.run([DRIVER], cwd=root, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                             timeout=600)
        assert out.returncode == 0, out.stdout.decode()
        assert "main loop have taken" in out.stdout.decode()
        b = os.path.join(root, "binData")
        assert open(os.path.join(b, "sys.N")).read().startswith("@ 4")
        assert not os.path.exists(os.path.join(root, "tmp", "stop.flag"))
        rows, Eo, Ho, mo = oracle(n, h, tau, m0, E0, H0, CASE["steps"])
        m, E, H = read_record(root, 3)
        assert parity.rel_err(E, Eo) < 1e-12 and parity.rel_err(H, Ho) < 1e-12
        parity.compare_markers(m, mo, h, pos_tol=1e-15, mom_tol=1e-12)
        # record 1 is the state after 5 steps
        o5 = oracle(n, h, tau, m0, E0, H0, 5)
        m1, E1, H1 = read_record(root, 1)
        assert parity.rel_err(E1, o5[1]) < 1e-12
        parity.compare_markers(m1, o5[3], h, pos_tol=1e-15, mom_tol=1e-12)
        d = refrun.read_diag(os.path.join(b, "diag.dat"))
        assert d.shape == (CASE["steps"] - 1, 10)           # the t = 0 row is skipped
        np.testing.assert_allclose(d[:, 1:6], rows[1:, :5], rtol=5e-6, atol=1e-300)
        np.testing.assert_allclose(d[:, 9], d[:, 1:6].sum(1), rtol=1e-5)
        if refrun.have_reference():
            ref = tempfile.mkdtemp(prefix="mg_ref_")
            try:
                rr = refrun.RefRun(ref)
                prepare(ref)
                rr._run("core.out")
                mr, Er, Hr = read_record(ref, 3)
                assert parity.rel_err(E, Er) < 1e-12 and parity.rel_err(H, Hr) < 1e-12
                parity.compare_markers(m, mr, h, pos_tol=1e-15, mom_tol=1e-12)
                dr = refrun.read_diag(os.path.join(ref, "binData", "diag.dat"))
                np.testing.assert_allclose(d, dr, rtol=2e-6, atol=1e-300)
            finally:
                shutil.rmtree(ref, ignore_errors=True)
    finally:
        shutil.rmtree(root, ignore_errors=True)


@pytest.mark.gpu
def test_driver_continues_from_the_last_record():
    root = tempfile.mkdtemp(prefix="mg_drv_")
    try:
        n, h, tau, m0, E0, H0 = prepare(root)
        refrun.write_run_cfg(root, 6, 6)
        assert subprocess.run([DRIVER], cwd=root, stdout=subprocess.DEVNULL).returncode == 0
        with open(os.path.join(root, "run_mandor.cfg"), "w") as fp:
            fp.write("@ 6\n@ 6\n@ -1\n@ 1\n@ 100000000\n@ -100\n")
        assert subprocess.run([DRIVER], cwd=root, stdout=subprocess.DEVNULL).returncode == 0
        m, E, H = read_record(root, 2)
        # A restart re-initialises the walls from the loaded record (cap_init,
        # core/em_caps.c:343-392: Mur history from the stored E), so the
        # comparison restarts the restatement the same way.
        _, E6, H6, m6 = oracle(n, h, tau, m0, E0, H0, 6)
        o = oracle_port.OracleRun(n, h, tau, CASE["bc_min"], CASE["bc_max"], time=6 * tau)
        o.set_fields(E6, H6)
        o.set_markers(m6)
        o.init()
        o.step(6)
        Eo, Ho = o.fields()
        assert parity.rel_err(E, Eo) < 1e-12 and parity.rel_err(H, Ho) < 1e-12
        parity.compare_markers(m, o.markers(), h, pos_tol=1e-15, mom_tol=1e-12)
        d = refrun.read_diag(os.path.join(root, "binData", "diag.dat"))
        assert d.shape[0] == 11
    finally:
        shutil.rmtree(root, ignore_errors=True)


@pytest.mark.gpu
def test_driver_stops_on_request():
    root = tempfile.mkdtemp(prefix="mg_drv_")
    try:
        prepare(root)
        refrun.write_run_cfg(root, 40, 100, stop=4)
        with open(os.path.join(root, "tmp", "stop.flag"), "w") as fp:
            fp.write("1\n100000\n")
        out = subprocess.run([DRIVER], cwd=root, stdout=subprocess.PIPE)
        assert out.returncode == 0
        # stopped at step 4: one final record written after the check
        assert open(os.path.join(root, "binData", "sys.N")).read().startswith("@ 2")
        txt = open(os.path.join(root, "binData", "sys_000001.txt")).read()
        t = float(txt.split()[1])
        assert abs(t / (0.5 / np.sqrt(sum(1 / v ** 2 for v in
                   [cases.H_LAMBDA] * 3))) - 4) < 1e-6
    finally:
        shutil.rmtree(root, ignore_errors=True)


@pytest.mark.gpu
def test_driver_applies_the_gauss_spot_config():
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_golden
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "gauss_spot.npz"))
    h, tau = tuple(g["h"]), float(g["tau"])
    root = tempfile.mkdtemp(prefix="mg_drv_")
    try:
        n = make_golden.SPOT_N
        z = np.zeros((n[0] + 1, n[1] + 1, n[2] + 1, 3))
        refrun.write_checkpoint0(root, n, h, tau, (2, 2, 2), (2, 2, 2), z, z,
                                 np.zeros(0, refrun.MARKER_DTYPE))
        refrun.write_run_cfg(root, make_golden.SPOT_STEPS, 10 ** 6)
        refrun.RefRun(root).set_gauss_spot(**make_golden.spot_params(h))
        out = subprocess.run([DRIVER], cwd=root, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                             timeout=600)
        assert out.returncode == 0, out.stdout.decode()
        m, E, H = read_record(root, 1)
        assert parity.rel_err(E, g["E"]) < 1e-12 and parity.rel_err(H, g["H"]) < 1e-12
    finally:
        shutil.rmtree(root, ignore_errors=True)


@pytest.mark.gpu
def test_driver_writes_the_reference_tecplot_records():
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_golden
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tecplot.npz"))
    root = tempfile.mkdtemp(prefix="mg_drv_")
    try:
        prepare(root)
        with open(os.path.join(root, "run_mandor.cfg"), "w") as fp:
            fp.write("@ %d\ttotal\n@ %d\tfull\n@ %d\ttecplot\n@ 0\tcontinue\n@ %d\tstop\n@ -100\tspectr\n"
                     % (CASE["steps"], 10 ** 6, make_golden.TEC_PERIOD, 10 ** 6))
        out = subprocess.run([DRIVER], cwd=root, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                             timeout=600)
        assert out.returncode == 0, out.stdout.decode()
        assert open(os.path.join(root, "binData", "tecplot.N")).read().startswith("@ 4")
        for num in (1, 2, 3):
            t = make_golden.read_tecplot(root, num)
            for f in ("E", "H", "J", "rho"):
                assert parity.rel_err(t[f], g["%s%d" % (f, num)]) < 1e-12, (f, num)
            assert abs(t["time"] - g["time%d" % num]) <= 1e-15
            assert np.array_equal(t["ids"], g["ids%d" % num])
    finally:
        shutil.rmtree(root, ignore_errors=True)


@pytest.mark.gpu
def test_snapshot_is_the_state_at_its_step():
    """mg_run_snapshot: the copy equals mg_run_get_fields / get_markers at the
    step it was taken, however many steps run before it is read."""
    import mandor3_b200 as mg
    root = tempfile.mkdtemp(prefix="mg_drv_")
    try:
        n, h, tau, m0, E0, H0 = prepare(root)
    finally:
        shutil.rmtree(root, ignore_errors=True)
    for prec in (mg.FP64, mg.FP32_OFFSET):
        r = mg.Run(n, h, tau, CASE["bc_min"], CASE["bc_max"], precision=prec)
        r.set_fields(E0, H0)
        r.set_markers(m0)
        r.init()
        r.step(3)
        E, H = r.fields()
        m = r.markers()
        wait = r.snapshot()
        r.step(5)
        Es, Hs, ms = wait()
        assert np.array_equal(Es, E) and np.array_equal(Hs, H)
        assert np.array_equal(np.sort(ms, order="id"), np.sort(m, order="id"))
        assert not np.array_equal(r.fields()[0], E)
        r.close()
