"""Host logic of the scan layer (no GPU): footprints, stream generation,
tuner classes."""
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
