"""Failure paths of the host side, without a GPU: core_b200.out given a
truncated or inconsistent checkpoint (the reference's loaders,
core/plasma_IO.c:227-266 and IO_sys.c:130-142, end the run through DIE) or a
malformed run_mandor.cfg (core/main.c:205-213) stops before it touches the
device, with a message naming the file and exit status 7 (MG_ERR_IO); the
serving loop refuses a solve larger than its whole memory budget with
MG_ERR_ADMISSION before building anything."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

import test_driver

DRIVER = test_driver.DRIVER
mg = pytest.importorskip("mandor3_b200")

pytestmark = pytest.mark.skipif(not os.path.exists(DRIVER), reason="core_b200.out not built")


@pytest.fixture
def rundir():
    root = tempfile.mkdtemp(prefix="mg_fail_")
    test_driver.prepare(root)
    yield root
    shutil.rmtree(root, ignore_errors=True)


def run_driver(root):
    res = subprocess.run([DRIVER], cwd=root, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                         timeout=120, env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    return res.returncode, res.stdout.decode(errors="replace")


def truncate(path, keep):
    with open(path, "rb") as fp:
        raw = fp.read()
    with open(path, "wb") as fp:
        fp.write(raw[:keep(len(raw))])


@pytest.mark.parametrize("name,keep", [
    ("plasma_000000_000.bin", lambda n: n - 64),         # one marker short
    ("plasma_000000_000.bin", lambda n: 4),              # count itself cut
    ("sys_E_000000(000).bin", lambda n: n - 8),          # one double short
    ("sys_H_000000(000).bin", lambda n: 100),            # header cut
])
def test_truncated_checkpoint_is_refused(rundir, name, keep):
    truncate(os.path.join(rundir, "binData", name), keep)
    rc, out = run_driver(rundir)
    assert rc == 7, out
    assert "truncated" in out and name in out


def test_negative_marker_count_is_refused(rundir):
    path = os.path.join(rundir, "binData", "plasma_000000_000.bin")
    with open(path, "r+b") as fp:
        fp.write(np.array([-3], "<i8").tobytes())
    rc, out = run_driver(rundir)
    assert rc == 7 and "negative marker count" in out, out


def test_mesh_region_mismatch_is_refused(rundir):
    path = os.path.join(rundir, "binData", "sys_E_000000(000).bin")
    with open(path, "r+b") as fp:
        fp.seek(12)
        fp.write(np.array([5], "<i4").tobytes())          # max i of the valid region
    rc, out = run_driver(rundir)
    assert rc == 7 and "region does not match" in out, out


@pytest.mark.parametrize("text,msg", [
    ("@ 12\ttotal\n@ x\tfull\n", "bad integer line"),
    ("@ 12\ttotal\n@ 5\tfull\n@ -1\ttecplot\n", "bad integer line"),           # lines missing
    ("@ 12\ttotal\n@ 0\tfull\n@ -1\ttecplot\n@ 0\tcont\n@ 100\tstop\n@ -100\tspectr\n",
     "contains zero step(s)"),
])
def test_bad_run_config_is_refused(rundir, text, msg):
    with open(os.path.join(rundir, "run_mandor.cfg"), "w") as fp:
        fp.write(text)
    rc, out = run_driver(rundir)
    assert rc == 7 and msg in out, out


def test_missing_checkpoint_is_refused(rundir):
    os.remove(os.path.join(rundir, "binData", "sys.N"))
    rc, out = run_driver(rundir)
    assert rc == 7 and "initial checkpoint is not prepared" in out, out


def test_server_refuses_a_solve_beyond_its_budget():
    from mandor3_b200 import scan
    small = scan.FoilSolve((64, 32, 32), 4, 2.0, 0.5, 30.0, 100)
    big = scan.FoilSolve((256, 128, 128), 16, 2.0, 0.5, 30.0, 100)
    budget = scan.footprint(small) * 3
    assert scan.footprint(big) > budget
    srv = scan.Server(budget=budget)
    with pytest.raises(mg.MandorError) as e:
        srv.serve([(0.0, big)])
    assert e.value.code == scan.ERR_ADMISSION and "budget" in str(e.value)
