"""Continuous-batching server: a solve's result is the same alone and in a
mix of solves that arrive while it runs (within FP32 round-off for the
precision form, 1e-10 for the FP64 form), and admission keeps the admitted
footprints within the memory budget."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

mg = pytest.importorskip("mandor3_b200")
from mandor3_b200 import scan  # noqa: E402


def specs():
    return [scan.FoilSolve((48, 24, 24), 2, 2.0, 0.25, 20.0, 60),
            scan.FoilSolve((40, 24, 16), 3, 5.0, 0.2, 40.0, 45, seed=(11, 12)),
            scan.FoilSolve((32, 16, 16), 2, 1.0, 0.3, 10.0, 70, precision=mg.FP64, seed=(13, 14)),
            scan.PeriodicSolve((16, 16, 16), 4, 0.05, 50, seed=(15, 16))]


def close(got, want, precision):
    tol = 1e-10 if precision == mg.FP64 else 1e-5
    scale = float(np.max(np.abs(want[:, 1:6].sum(1))))
    np.testing.assert_allclose(got, want, rtol=tol, atol=tol * scale)


def test_result_is_the_same_alone_and_in_the_mix():
    ss = specs()
    alone = [scan.run_alone(s) for s in ss]
    stream = [(0.0, ss[0]), (0.0, ss[1]), (0.02, ss[2]), (0.05, ss[3])]
    res = scan.Server(chunk=20).serve(stream)
    for s, (rows, count, _), r in zip(ss, alone, res):
        assert r.rows.shape == rows.shape
        close(r.rows, rows, s.precision)
        assert r.markers == count
        assert r.latency >= 0 and r.finished >= r.admitted >= r.arrival - 1e-9


def test_admission_keeps_footprints_within_the_budget():
    ss = specs()
    need = sorted(scan.footprint(s) for s in ss)
    budget = need[-1] + need[-2]
    srv = scan.Server(chunk=25, budget=budget)
    res = srv.serve([(0.0, s) for s in ss])
    assert len(res) == len(ss)
    assert 0 < srv.peak_used <= budget
    # Two solves at most fit at once, so some waited in the queue.
    assert max(r.admitted - r.arrival for r in res) > 0


def test_tuned_solve_matches_the_default_one():
    s = scan.FoilSolve((48, 24, 24), 2, 2.0, 0.25, 20.0, 40)
    t = scan.Tuner(steps=4, sorts=(4, 8))
    tile, every, warps = t.choose(s)
    assert tile in scan.Tuner.TILES and every in (4, 8) and warps in scan.Tuner.WARPS
    rows, count, _ = scan.run_alone(s, tile=tile, sort_every=every, warps=warps)
    ref, count0, _ = scan.run_alone(s)
    close(rows, ref, s.precision)
    assert count == count0


def test_served_precision_is_within_the_conditioning_floor():
    """Accuracy of the precision form on served laser-foil solves.  These
    strongly driven solves amplify any relative perturbation of their state
    by 1e3-1e5 over a few thousand steps, so no single-precision form can
    stay within 1e-4 of FP64 over a whole solve: the FP64 form itself, with
    the laser amplitude moved by 2^-24 (single-precision rounding of one
    input), leaves its own history by 2e-4 .. 1.6e-2 on the served stream.
    The rule: over the whole history, the precision form's largest
    total-energy difference from FP64 stays within 10 times that floor
    (measured on the 24-solve stream: 0.67 .. 5.4 times).  Two full solves
    of the stream's smallest grid (requests 3 and 8 of the benchmark's
    stream) are checked here."""
    import dataclasses
    tot = lambda a: a[:, 1] + a[:, 2] + a[:, 3:6].sum(1)
    for s in (scan.FoilSolve((64, 32, 32), 4, 2.214395523957853, 1.0130362634300774, 99.70541371379576,
                             2581, seed=(1802, 9376)),
              scan.FoilSolve((64, 32, 32), 5, 4.680910375735458, 1.0720577463625738, 91.33073865907738,
                             1982, seed=(1802, 9381))):
        r32, _, _ = scan.run_alone(s)
        p = dataclasses.replace(s, precision=mg.FP64)
        r64, _, _ = scan.run_alone(p)
        rs, _, _ = scan.run_alone(dataclasses.replace(p, a0=p.a0 * (1 + 2.0 ** -24)))
        scale = np.max(np.abs(tot(r64)))
        e32 = np.max(np.abs(tot(r32) - tot(r64))) / scale
        floor = np.max(np.abs(tot(rs) - tot(r64))) / scale
        assert floor > 0
        assert e32 <= 10 * floor, (e32, floor)
