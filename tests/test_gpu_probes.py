"""Device probes (mg_run_set_probes / mg_run_probe_samples) and the drop-in
driver's probe and spectral-dump files, against the oracle and the reference
core.out's files (tests/golden/probes.npz)."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

import oracle_port
import parity
import refrun
import test_driver
from test_probes import GOLD, case_state, first_step_rows, golden_probes, make_golden, oracle_run

pytestmark = pytest.mark.gpu

mg = pytest.importorskip("mandor3_b200")


def device_run(precision, state):
    n, h, tau, m0, E0, H0 = state
    r = mg.Run(n, h, tau, test_driver.CASE["bc_min"], test_driver.CASE["bc_max"], precision=precision)
    r.set_fields(E0, H0)
    r.set_markers(m0)
    return r


@pytest.mark.parametrize("precision", [mg.FP64, mg.FP32_OFFSET])
def test_probe_samples_match_the_oracle(precision):
    state = case_state()
    ijk = sorted(golden_probes())
    r = device_run(precision, state)
    r.set_probes(ijk)
    r.init()
    steps = test_driver.CASE["steps"]
    r.step(steps)
    got = r.probe_samples(steps)
    want = oracle_run(*state).step_probes(ijk, steps)
    assert np.array_equal(got[:, :, 0], want[:, :, 0])
    # FP32 fields: single-precision interpolation of single-precision values.
    tol = 1e-12 if precision == mg.FP64 else 1e-4
    assert parity.rel_err(got[:, :, 1:], want[:, :, 1:]) < tol
    r.close()


def test_staged_step_samples_its_fields():
    """mg_em_HHalfStep records the row of a stage-by-stage step."""
    state = case_state()
    ijk = sorted(golden_probes())[:5]
    r = device_run(mg.FP64, state)
    r.set_probes(ijk)
    r.init()
    r.step(3)
    r.em_HHalfStep()
    r.em_energy()
    staged = r.probe_samples(1)
    r.plasma_move()
    r.plasma_temperature()
    r.em_HStep()
    r.em_EStep_start()
    r.jbc_finish()
    r.em_EStep_finish()
    want = oracle_run(*state).step_probes(ijk, 4)[3:]
    assert parity.rel_err(staged, want) < 1e-12
    r.step(2)
    want = oracle_run(*state).step_probes(ijk, 6)[4:]
    assert parity.rel_err(r.probe_samples(2), want) < 1e-12
    r.close()


def test_probe_arguments_are_checked():
    r = device_run(mg.FP64, case_state())
    with pytest.raises(mg.MandorError):
        r.set_probes([(0, 0, test_driver.CASE["n"][2])])
    r.set_probes([])
    r.close()


def run_driver(root):
    out = subprocess.run([test_driver.DRIVER], cwd=root, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                         timeout=600)
    assert out.returncode == 0, out.stdout.decode()


def compare_dump(got, want):
    a, b = refrun.read_chunks(got), refrun.read_chunks(want)
    assert [c[:2] for c in a] == [c[:2] for c in b]
    assert a[0][2] == b[0][2] and a[1][2] == b[1][2]            # parameters text, region
    for x, y in zip(a[2:], b[2:]):
        assert parity.rel_err(np.frombuffer(x[2], "<f8"), np.frombuffer(y[2], "<f8")) < 1e-12, x[0]


def test_driver_writes_the_reference_probe_and_spectral_files():
    root = tempfile.mkdtemp(prefix="mg_drv_")
    try:
        test_driver.prepare(root)
        n, L_um = test_driver.cases.geometry(test_driver.CASE)
        with open(os.path.join(root, "run_mandor.cfg"), "w") as fp:
            fp.write(make_golden.probe_run_cfg(test_driver.CASE["steps"]))
        with open(os.path.join(root, "run_probes.cfg"), "w") as fp:
            fp.write(make_golden.probe_deck([L_um[a] / n[a] for a in range(3)]))
        # a stale probe file of an earlier run is removed on a fresh start
        open(os.path.join(root, "binData", "probe_99_0_0.bin"), "wb").write(b"stale")
        run_driver(root)
        files = make_golden.probe_files(root)
        assert sorted(files) == sorted(GOLD.files)
        for k in GOLD.files:
            want = bytes(GOLD[k])
            if k.startswith("binData/probe_") and k != "binData/probe_globals.bin":
                ijk, a = refrun.read_probe(files[k])
                _, b = refrun.read_probe(want)
                assert files[k][:20] == want[:20] and a.shape == b.shape
                rows = first_step_rows(ijk)
                assert np.array_equal(a[:, 0], b[:, 0])
                assert parity.rel_err(a[rows, 1:], b[rows, 1:]) < 1e-12, k
            elif k.startswith("tmp/spectrDump_"):
                compare_dump(files[k], want)
            else:
                assert files[k] == want, k
        # the tecplot dump of step 10 is written beside the spectral dump
        assert open(os.path.join(root, "binData", "tecplot.N")).read().startswith("@ 2")
    finally:
        shutil.rmtree(root, ignore_errors=True)


def test_driver_continues_probe_and_spectral_files():
    """A continued run appends to the probe files and numbers its spectral
    dumps after binData/spectr.N; the first step after the driver's own
    record samples H^n like the oracle restarted from that record."""
    root = tempfile.mkdtemp(prefix="mg_drv_")
    try:
        n, h, tau, m0, E0, H0 = test_driver.prepare(root)
        nodes = [(0, 0, 0), (5, 4, 7), (11, 9, 13)]
        with open(os.path.join(root, "run_probes.cfg"), "w") as fp:
            for node in nodes:
                fp.write("@ point\n" + "".join("> %.9f\n" % ((c + 0.5) * h[a]) for a, c in enumerate(node)))
            fp.write("@ end\n")
        with open(os.path.join(root, "run_mandor.cfg"), "w") as fp:
            fp.write("@ 5\n@ 5\n@ -1\n@ 0\n@ 100000000\n@ 4\n")
        run_driver(root)
        with open(os.path.join(root, "run_mandor.cfg"), "w") as fp:
            fp.write("@ 4\n@ 100\n@ -1\n@ 1\n@ 100000000\n@ 4\n")
        run_driver(root)
        # dumps at the 4th step of each run: numbered 0, then 1
        assert open(os.path.join(root, "binData", "spectr.N")).read() == "@ 2  spectr dumps written.\n"
        b = os.path.join(root, "binData")
        m5, E5, H5 = test_driver.read_record(root, 1)
        o = oracle_port.OracleRun(n, h, tau, test_driver.CASE["bc_min"], test_driver.CASE["bc_max"],
                                  time=5 * tau)
        o.set_fields(E5, H5)
        o.set_markers(m5)
        o.init()
        want2 = o.step_probes(nodes, 4)
        want1 = oracle_run(n, h, tau, m0, E0, H0).step_probes(nodes, 5)
        for q, node in enumerate(nodes):
            ijk, rows = refrun.read_probe(open(os.path.join(b, "probe_%d_%d_%d.bin" % node), "rb").read())
            assert ijk == node and rows.shape == (9, 7)
            first = first_step_rows(node)
            assert parity.rel_err(rows[:5][first, 1:], want1[first, q, 1:]) < 1e-12
            assert parity.rel_err(rows[5:], want2[:, q]) < 1e-12
    finally:
        shutil.rmtree(root, ignore_errors=True)
