"""Device TF/SF interface (mg_run_set_tfsf and friends) against the
reference's record and play runs (tests/golden/tfsf.npz) and the oracle."""
import numpy as np
import pytest

import parity
import refrun
import test_tfsf
from test_tfsf import BC, GOLD, box_cfg, make_golden, merged_frames, raw, streams

pytestmark = pytest.mark.gpu

mg = pytest.importorskip("mandor3_b200")


def device(precision=mg.FP64, markers=None):
    h, tau = tuple(GOLD["h"]), float(GOLD["tau"])
    n = make_golden.TFSF_N
    m = markers if markers is not None else np.zeros(0, mg.MARKER_DTYPE)
    r = mg.Run(n, h, tau, BC, BC, precision=precision, capacity=max(len(m), 1))
    shape = tuple(v + 1 for v in n) + (3,)
    r.set_fields(np.zeros(shape), np.zeros(shape))
    r.set_markers(m)
    return r, h


def tfsf_args(mode, frames=0, ring=2):
    c = box_cfg(mode, frames=frames)
    return dict(lo=c["lo"], hi=c["hi"], mode=mode, open=c["open"], frames=frames, ring=ring)


@pytest.mark.parametrize("precision", [mg.FP64, mg.FP32_OFFSET])
def test_record_matches_the_reference(precision):
    r, h = device(precision)
    r.set_gauss_spot(**make_golden.tfsf_spot(h))
    r.set_tfsf(**tfsf_args(mg.TFSF_RECORD))
    r.init()
    steps = make_golden.TFSF_STEPS
    r.step(steps)
    heads, want = streams("rec/")
    regions, size = r.tfsf_faces()
    assert np.array_equal(regions, heads[:, :6]) and size == want.shape[1]
    got = r.tfsf_recorded(steps)
    assert parity.rel_err(got, want) < (1e-13 if precision == mg.FP64 else 1e-5)
    r.close()


@pytest.mark.parametrize("mode", [0, 2])
@pytest.mark.parametrize("precision", [mg.FP64, mg.FP32_OFFSET])
def test_play_matches_the_reference(mode, precision):
    markers = make_golden.tfsf_plasma(tuple(GOLD["h"])) if mode == 0 else None
    r, h = device(precision, markers)
    frames = merged_frames()
    r.set_tfsf(**tfsf_args(mode, frames=len(frames), ring=len(frames)))
    r.tfsf_put_frames(0, frames)
    r.init()
    rows = r.step(make_golden.TFSF_STEPS)
    E, H = r.fields()
    tol = 1e-12 if precision == mg.FP64 else 1e-4
    assert parity.rel_err(E, np.frombuffer(raw("play%d/E" % mode), "<f8").reshape(E.shape)) < tol
    if mode == 0:
        assert parity.rel_err(H, np.frombuffer(raw("play0/H"), "<f8").reshape(H.shape)) < tol
        d = np.frombuffer(raw("play0/diag"), "<f8").reshape(-1, 10)
        np.testing.assert_allclose(d[:, 1:6], rows[1:, 1:6], rtol=5e-6 if precision == mg.FP64 else 1e-3,
                                   atol=1e-12)
    r.close()


def test_play_through_a_small_ring_and_staged_steps():
    """Frames streamed a few at a time into a 4-slot ring, graph and staged
    steps mixed: the same fields as the oracle."""
    frames = merged_frames()
    mode = 0
    markers = make_golden.tfsf_plasma(tuple(GOLD["h"]))
    r, h = device(mg.FP64, markers)
    r.set_tfsf(**tfsf_args(mode, frames=len(frames), ring=4))
    r.init()
    n = 0
    while n < make_golden.TFSF_STEPS:
        k = min(2, make_golden.TFSF_STEPS - n)
        need = range(n, min(n + k + 1, len(frames)))
        r.tfsf_put_frames(need[0], frames[need[0]:need[-1] + 1])
        if n % 4 == 2:
            for _ in range(k):
                r.em_HHalfStep()
                r.em_energy()
                r.plasma_move()
                r.plasma_temperature()
                r.em_HStep()
                r.em_EStep_start()
                r.jbc_finish()
                r.em_EStep_finish()
        else:
            r.step(k)
        n += k
    o, _ = test_tfsf.oracle(markers)
    o.set_tfsf(**box_cfg(mode, frames=len(frames)), frames_data=frames)
    o.init()
    o.step(make_golden.TFSF_STEPS)
    E, H = r.fields()
    Eo, Ho = o.fields()
    assert parity.rel_err(E, Eo) < 1e-12 and parity.rel_err(H, Ho) < 1e-12
    r.close()


def test_a_missing_frame_fails_the_step():
    frames = merged_frames()
    r, _ = device()
    r.set_tfsf(**tfsf_args(0, frames=len(frames), ring=4))
    r.tfsf_put_frames(0, frames[:2])
    r.init()
    r.step(1)                        # frames 0 and 1
    with pytest.raises(mg.MandorError):
        r.step(1)                    # needs frame 2
    r.close()


def test_played_faces_must_stay_inside():
    r, _ = device()
    args = tfsf_args(0, frames=4, ring=4)
    args["hi"] = (13, 8, 8)
    with pytest.raises(mg.MandorError):
        r.set_tfsf(**args)
    r.close()


# ---- the drop-in driver ------------------------------------------------------

def driver_dir(markers, mode, tecplot=-1):
    import os
    import tempfile
    root = tempfile.mkdtemp(prefix="mg_tfsf_")
    rr = refrun.RefRun(root)
    n, h, tau = make_golden.TFSF_N, tuple(GOLD["h"]), float(GOLD["tau"])
    shape = tuple(v + 1 for v in n) + (3,)
    refrun.write_checkpoint0(root, n, h, tau, BC, BC, np.zeros(shape), np.zeros(shape), markers)
    with open(os.path.join(root, "run_mandor.cfg"), "w") as fp:
        fp.write("@ %d\ttotal\n@ %d\tfull\n@ %d\ttecplot\n@ 0\tcontinue\n@ %d\tstop\n@ -100\tspectr\n"
                 % (make_golden.TFSF_STEPS, 10 ** 6, tecplot, 10 ** 6))
    rr.set_tfsf(make_golden.TFSF_BOX, mode)
    return rr


def run_driver(rr):
    import subprocess
    from test_driver import DRIVER
    out = subprocess.run([DRIVER], cwd=rr.dir, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, timeout=600)
    assert out.returncode == 0, out.stdout.decode()
    return out.stdout.decode()


@pytest.mark.parametrize("tecplot", [-1, 5])
def test_driver_records_the_reference_streams(tecplot):
    import os
    rr = driver_dir(np.zeros(0, mg.MARKER_DTYPE), mg.TFSF_RECORD, tecplot)
    try:
        rr.set_gauss_spot(**make_golden.tfsf_spot(tuple(GOLD["h"])))
        run_driver(rr)
        d = rr.path(".EM_sources", "TFSF")
        for k in refrun.TFSF_FACES:
            got = open(os.path.join(d, k + "_000.bin"), "rb").read()
            want = raw("rec/" + k)
            assert got[:44] == want[:44] and len(got) == len(want), k
            _, a = refrun.read_tfsf_stream(got)
            _, b = refrun.read_tfsf_stream(want)
            assert parity.rel_err(a, b) < 1e-13, k
        for f in ("consistencyCheck.dat", "TFSF_defrag.map", "lastFrameTime.bin"):
            assert open(os.path.join(d, f), "rb").read() == raw("rec/" + f), f
        # a second run refuses streams that were not merged
        import subprocess
        from test_driver import DRIVER
        out = subprocess.run([DRIVER], cwd=rr.dir, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
        assert out.returncode != 0 and b"TFSFdefrag" in out.stdout
    finally:
        rr.cleanup()


@pytest.mark.parametrize("mode,tecplot", [(0, -1), (0, 5), (2, -1)])
def test_driver_plays_the_reference_streams(mode, tecplot):
    import os
    h = tuple(GOLD["h"])
    markers = make_golden.tfsf_plasma(h) if mode == 0 else np.zeros(0, mg.MARKER_DTYPE)
    rr = driver_dir(markers, mode, tecplot)
    try:
        d = rr.path(".EM_sources", "TFSF")
        for k in refrun.TFSF_FACES:
            open(os.path.join(d, k + "_99999.bin"), "wb").write(raw("merged/" + k))
        open(os.path.join(d, "lastFrameTime.bin"), "wb").write(raw("merged/lastFrameTime.bin"))
        open(os.path.join(d, "consistencyCheck.dat"), "wb").write(raw("rec/consistencyCheck.dat"))
        run_driver(rr)
        _, E, H = rr.final()
        assert parity.rel_err(E, np.frombuffer(raw("play%d/E" % mode), "<f8").reshape(E.shape)) < 1e-12
        if mode == 0:
            assert parity.rel_err(H, np.frombuffer(raw("play0/H"), "<f8").reshape(H.shape)) < 1e-12
    finally:
        rr.cleanup()
