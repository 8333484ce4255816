"""Device focused-laser soft source (mg_run_add_mirror) against the
reference's core.out playing a setup.out mirror file (tests/golden/mirror.npz)
and against the oracle; the drop-in driver reading the mirror file itself."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle_port
import parity
import refrun
from test_mirror import BC, GOLD, make_golden, mirror

pytestmark = pytest.mark.gpu

mg = pytest.importorskip("mandor3_b200")


def device(precision, mirrors):
    n, h, tau = make_golden.MIRROR_N, tuple(GOLD["h"]), float(GOLD["tau"])
    r = mg.Run(n, h, tau, BC, BC, precision=precision, capacity=1)
    shape = tuple(v + 1 for v in n) + (3,)
    r.set_fields(np.zeros(shape), np.zeros(shape))
    r.set_markers(np.zeros(0, mg.MARKER_DTYPE))
    for args in mirrors:
        r.add_mirror(*args)
    return r


def mirror_args(direction, focus_x=None):
    vals, d, E, H = mirror(direction)
    u = GOLD["units%d" % direction]
    vals = list(vals)
    if focus_x is not None:
        vals[2] = focus_x
    return (vals, d, u[0], u[2], E, H)


def oracle(mirrors, steps):
    n, h, tau = make_golden.MIRROR_N, tuple(GOLD["h"]), float(GOLD["tau"])
    o = oracle_port.OracleRun(n, h, tau, BC, BC)
    o.set_fields(np.zeros(o.shape()), np.zeros(o.shape()))
    o.set_markers(np.zeros(0, oracle_port.MARKER_DTYPE))
    for args in mirrors:
        o.add_mirror(*args)
    o.init()
    o.step(steps)
    return o.fields()


@pytest.mark.parametrize("precision", [mg.FP64, mg.FP32_OFFSET])
@pytest.mark.parametrize("direction", [1, -1])
def test_device_plays_the_reference_mirror(direction, precision):
    r = device(precision, [mirror_args(direction)])
    r.init()
    r.step(make_golden.MIRROR_STEPS)
    E, H = r.fields()
    wE, wH = GOLD["E%d" % direction], GOLD["H%d" % direction]
    if direction == 1:
        tol = 1e-12 if precision == mg.FP64 else 1e-4
        assert parity.rel_err(E, wE) < tol and parity.rel_err(H, wH) < tol
    else:
        # the reference's backward delay keeps the pulse off this grid
        assert np.abs(E).max() == 0.0 and np.abs(H).max() == 0.0 and np.abs(wE).max() == 0.0
    r.close()


def backward_on_grid():
    """The backward mirror with its focus moved so that the reference's
    backward delay (cell count minus focus) equals the forward one: the
    pulse then enters through the x = n0 - 4 planes within the run."""
    u = GOLD["units1"]
    n0, h1 = make_golden.MIRROR_N[0], float(GOLD["h"][0])
    xf_fwd = 0.6e-4 / u[0]
    xf = n0 - xf_fwd             # n0 - 5 h1 - xf == xf_fwd - 5 h1
    return mirror_args(-1, focus_x=xf * u[0] * 1e4)


@pytest.mark.parametrize("precision", [mg.FP64, mg.FP32_OFFSET])
def test_backward_and_two_mirrors_match_the_oracle(precision):
    """Both play planes and two sources at once, staged and graph steps
    mixed, against the oracle."""
    ms = [mirror_args(1), backward_on_grid()]
    steps = make_golden.MIRROR_STEPS
    wE, wH = oracle(ms, steps)
    assert np.abs(wE[-6, :, :]).max() > 0.1          # the backward plane radiates
    r = device(precision, ms)
    r.init()
    r.step(7)
    for _ in range(5):
        r.em_HHalfStep()
        r.em_energy()
        r.plasma_move()
        r.plasma_temperature()
        r.em_HStep()
        r.em_EStep_start()
        r.jbc_finish()
        r.em_EStep_finish()
    r.step(steps - 12)
    E, H = r.fields()
    tol = 1e-12 if precision == mg.FP64 else 1e-4
    assert parity.rel_err(E, wE) < tol and parity.rel_err(H, wH) < tol
    r.clear_mirrors()
    r.close()


def test_mirror_arguments_are_checked():
    vals, d, E, H = mirror(1)
    u = GOLD["units1"]
    r = device(mg.FP64, [])
    with pytest.raises(mg.MandorError):
        r.add_mirror(vals, d, 0.0, u[2], E, H)          # no units
    bad = list(vals)
    bad[5] = 0.0
    with pytest.raises(mg.MandorError):
        r.add_mirror(bad, d, u[0], u[2], E, H)          # no duration
    r.close()
    small = mg.Run((24, 9, 20), tuple(GOLD["h"]), float(GOLD["tau"]), BC, BC, precision=mg.FP64, capacity=1)
    with pytest.raises(mg.MandorError):
        small.add_mirror(vals, d, u[0], u[2], E[:0], H[:0])
    small.close()


def test_driver_plays_the_mirror_file():
    """core_b200.out finds .EM_sources/laser/mirror_00 and plays it as
    core.out does."""
    from test_driver import DRIVER
    root = tempfile.mkdtemp(prefix="mg_mirror_")
    rr = refrun.RefRun(root)
    try:
        n, h, tau = make_golden.MIRROR_N, tuple(GOLD["h"]), float(GOLD["tau"])
        shape = tuple(v + 1 for v in n) + (3,)
        refrun.write_checkpoint0(root, n, h, tau, BC, BC, np.zeros(shape), np.zeros(shape),
                                 np.zeros(0, mg.MARKER_DTYPE))
        with open(os.path.join(root, "binData", "units.bin"), "wb") as fp:
            fp.write(np.asarray(GOLD["units1"], "<f8").tobytes())
        os.makedirs(os.path.join(root, ".EM_sources", "laser"), exist_ok=True)
        with open(os.path.join(root, ".EM_sources", "laser", "mirror_00"), "wb") as fp:
            fp.write(bytes(GOLD["file1"]))
        refrun.write_run_cfg(root, make_golden.MIRROR_STEPS, 10 ** 6)
        out = subprocess.run([DRIVER], cwd=root, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, timeout=600)
        assert out.returncode == 0, out.stdout.decode()
        assert b"1 focused-laser source" in out.stdout
        _, E, H = rr.final()
        assert parity.rel_err(E, GOLD["E1"]) < 1e-12 and parity.rel_err(H, GOLD["H1"]) < 1e-12
    finally:
        rr.cleanup()
