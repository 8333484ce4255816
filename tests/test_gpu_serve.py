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
    tile, every = t.choose(s)
    assert tile in scan.Tuner.TILES and every in (4, 8)
    rows, count, _ = scan.run_alone(s, tile=tile, sort_every=every)
    ref, count0, _ = scan.run_alone(s)
    close(rows, ref, s.precision)
    assert count == count0
