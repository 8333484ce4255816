"""Host logic of the scan layer (no GPU): footprints, stream generation,
tuner classes and the tuner's search order."""
import pytest

mg = pytest.importorskip("mandor3_b200")
from mandor3_b200 import scan  # noqa: E402


def test_footprint_grows_with_grid_and_markers():
    a = scan.FoilSolve((64, 32, 32), 4, 1.0, 0.5, 10.0, 100)
    b = scan.FoilSolve((128, 64, 64), 4, 1.0, 0.5, 10.0, 100)
    c = scan.FoilSolve((64, 32, 32), 16, 1.0, 0.5, 10.0, 100)
    fa, fb, fc = scan.footprint(a), scan.footprint(b), scan.footprint(c)
    assert fa < fb and fa < fc
    assert fa > a.markers() * 80


def test_foil_geometry_stays_inside_the_walls():
    for n in [(16, 16, 16), (64, 32, 32), (256, 128, 128)]:
        for th in (0.1, 0.5, 2.0):
            s = scan.FoilSolve(n, 4, 1.0, th, 10.0, 10)
            n_, lo, hi = s.geometry()
            assert all(0 <= lo[a] < hi[a] <= n_[a] for a in range(3))


def test_poisson_stream_is_seeded_and_ordered():
    ss = list(range(50))
    a = scan.poisson_stream(ss, 200.0, seed=3)
    b = scan.poisson_stream(ss, 200.0, seed=3)
    assert a == b
    t = [x[0] for x in a]
    assert t[0] == 0.0 and all(u <= v for u, v in zip(t, t[1:]))
    assert 0.1 < t[-1] < 0.5          # 49 gaps of mean 5 ms


def test_tuner_classes_group_similar_solves():
    k = scan.Tuner.key
    assert k(scan.FoilSolve((64, 32, 32), 4, 1, 0.5, 10, 10)) == k(scan.FoilSolve((64, 32, 32), 4, 5, 1.0, 50, 99))
    assert k(scan.FoilSolve((64, 32, 32), 4, 1, 0.5, 10, 10)) != k(scan.FoilSolve((256, 128, 128), 4, 1, 0.5, 10, 10))


def test_tuner_picks_each_knob_by_its_own_timing(monkeypatch):
    # Timings are faked: the tile by push time at the first warps count and
    # the shortest sort interval, then the warps count at that tile, then the
    # sort interval by whole-step time (over at least two sort intervals).
    calls = []

    def fake_time(self, spec, steps, which, tile, sort_every, warps):
        calls.append((which, tile, sort_every, warps, steps))
        t = {(8, 8, 4): 3.0, (4, 4, 4): 1.0, (8, 8, 8): 2.0}[tile] + {8: 0.5, 4: 0.2, 16: 0.9}[warps]
        if which == "step":
            t += {4: 0.4, 8: 0.1, 16: 0.3}[sort_every]
        return t

    monkeypatch.setattr(scan.Tuner, "_time", fake_time)
    tuner = scan.Tuner(steps=12)
    spec = scan.FoilSolve((64, 32, 32), 4, 1.0, 0.5, 10.0, 100)
    assert tuner.choose(spec) == ((4, 4, 4), 8, 4)
    assert [c[1] for c in calls[:3]] == list(scan.Tuner.TILES)
    assert all(c[3] == scan.Tuner.WARPS[0] and c[2] == min(scan.Tuner.SORTS) for c in calls[:3])
    assert [c[3] for c in calls[3:6]] == list(scan.Tuner.WARPS) and all(c[1] == (4, 4, 4) for c in calls[3:6])
    assert [(c[0], c[2], c[4]) for c in calls[6:]] == [("step", e, max(12, 2 * e)) for e in scan.Tuner.SORTS]
    n = len(calls)
    same_class = scan.FoilSolve((64, 32, 32), 4, 5.0, 1.0, 50.0, 300)
    assert tuner.choose(same_class) == ((4, 4, 4), 8, 4) and len(calls) == n
    plain = scan.FoilSolve((64, 32, 32), 4, 1.0, 0.5, 10.0, 100, precision=mg.FP64)
    assert tuner.choose(plain) == ((0, 0, 0), 0, 0) and len(calls) == n
