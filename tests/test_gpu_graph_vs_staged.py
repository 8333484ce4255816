"""The graph-captured step (fused H half steps, fused E step with -tau J,
wall launches) against the staged step (mg_em_HHalfStep ... mg_em_EStep_finish,
one reference call each, separate kernels), node for node: in the FP64 form
E and H bit-identical and energies equal to round-off after 30 steps of a
field-only run, for periodic, mirror, Mur and mixed walls on a grid of
uneven sides; the precision form within 1e-5 of its field scale; graph and
staged steps interleaving on one run; and a run with markers and the
analytic laser (whose current sums differ between launches at round-off).
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

mg = pytest.importorskip("mandor3_b200")

N = (20, 19, 37)
H_ = (0.05, 0.045, 0.04)
TAU = 0.5 / math.sqrt(sum(1 / v ** 2 for v in H_))

WALLS = [((0, 0, 0), (0, 0, 0)), ((1, 1, 1), (1, 1, 1)), ((2, 2, 2), (2, 2, 2)),
         ((2, 0, 1), (2, 0, 1)), ((1, 2, 0), (2, 1, 0)), ((2, 1, 2), (1, 2, 1))]


def fields(n=N):
    i, j, k = np.meshgrid(*[np.arange(v + 1) / v for v in n], indexing="ij")
    E = np.zeros((n[0] + 1, n[1] + 1, n[2] + 1, 3))
    H = np.zeros_like(E)
    E[..., 0] = np.sin(2 * np.pi * (j + 2 * k)) * np.cos(2 * np.pi * i) + 0.3 * np.exp(-30 * ((i - .4) ** 2 + (k - .6) ** 2))
    E[..., 1] = 0.7 * np.cos(2 * np.pi * (i - k)) + 0.2 * np.sin(6 * np.pi * j)
    E[..., 2] = 0.4 * np.sin(2 * np.pi * (2 * i + j))
    H[..., 0] = 0.3 * np.cos(2 * np.pi * (j - k))
    H[..., 1] = 0.6 * np.sin(2 * np.pi * (i + k)) * np.cos(2 * np.pi * j)
    H[..., 2] = 0.5 * np.cos(2 * np.pi * (i + 2 * j))
    return E, H


def staged(r, steps):
    rows = []
    for _ in range(steps):
        r.em_HHalfStep()
        we, wm = r.em_energy()
        r.plasma_move()
        r.plasma_temperature()
        r.em_HStep()
        r.em_EStep_start()
        r.jbc_finish()
        r.em_EStep_finish()
        rows.append((we, wm))
    return np.array(rows)


def make(walls, precision, n=N):
    r = mg.Run(n, H_, TAU, walls[0], walls[1], precision=precision)
    E, H = fields(n)
    r.set_fields(E, H)
    r.init()
    return r


@pytest.mark.parametrize("walls", WALLS)
def test_graph_step_matches_staged_kernels(walls):
    a = make(walls, mg.FP64)
    rows = a.step(30)
    b = make(walls, mg.FP64)
    ref = staged(b, 30)
    Ea, Ha = a.fields()
    Eb, Hb = b.fields()
    assert np.array_equal(Ea, Eb) and np.array_equal(Ha, Hb)
    np.testing.assert_allclose(rows[:, 1:3], ref, rtol=1e-13, atol=1e-300)


# The smallest grids a run accepts (8 cells per axis, core/plasma.c:392-396)
# leave the merged wall launch three face lines per axis and three edge
# slices; odd sides give the slot passes a partial last slot.
@pytest.mark.parametrize("n", [(8, 9, 11), (9, 8, 8)])
@pytest.mark.parametrize("walls", [WALLS[0], WALLS[1], WALLS[4], WALLS[5]])
def test_graph_step_matches_staged_kernels_on_small_grids(walls, n):
    a = make(walls, mg.FP64, n)
    rows = a.step(20)
    b = make(walls, mg.FP64, n)
    ref = staged(b, 20)
    Ea, Ha = a.fields()
    Eb, Hb = b.fields()
    assert np.array_equal(Ea, Eb) and np.array_equal(Ha, Hb)
    np.testing.assert_allclose(rows[:, 1:3], ref, rtol=1e-13, atol=1e-300)


# A field-only run steps its fields as (y, z) tiles of 8 x 32 nodes over
# chunks of 16 x-planes: these grids give several tiles per axis, partial
# last tiles and chunks, sides that are whole multiples of the tile (the
# last tile then owns node n through its halo) and a last chunk of one plane.
@pytest.mark.parametrize("n", [(40, 37, 70), (20, 45, 33), (33, 32, 64)])
@pytest.mark.parametrize("walls", [WALLS[2], WALLS[3], WALLS[5]])
def test_graph_step_matches_staged_kernels_on_tiled_grids(walls, n):
    a = make(walls, mg.FP64, n)
    rows = a.step(15)
    b = make(walls, mg.FP64, n)
    ref = staged(b, 15)
    Ea, Ha = a.fields()
    Eb, Hb = b.fields()
    assert np.array_equal(Ea, Eb) and np.array_equal(Ha, Hb)
    np.testing.assert_allclose(rows[:, 1:3], ref, rtol=1e-13, atol=1e-300)


def test_batch_branch_matches_the_run_alone_bit_for_bit():
    # A run stepped as a batch branch keeps the per-axis wall kernels, alone
    # it takes the merged launch: a field-only FP64 run gives the same bits.
    alone = make(WALLS[4], mg.FP64)
    alone.step(25)
    a = make(WALLS[4], mg.FP64)
    other = make(WALLS[0], mg.FP64)
    b = mg.Batch([a, other])
    b.step(25)
    b.close()
    Ea, Ha = a.fields()
    Eb, Hb = alone.fields()
    assert np.array_equal(Ea, Eb) and np.array_equal(Ha, Hb)
    a.step(5)                   # alone again after the batch: merged walls
    alone.step(5)
    Ea, Ha = a.fields()
    Eb, Hb = alone.fields()
    assert np.array_equal(Ea, Eb) and np.array_equal(Ha, Hb)


@pytest.mark.parametrize("walls", [WALLS[3], WALLS[5]])
def test_graph_and_staged_steps_interleave(walls):
    a = make(walls, mg.FP64)
    a.step(7)
    staged(a, 3)
    a.step(5)
    b = make(walls, mg.FP64)
    staged(b, 15)
    Ea, Ha = a.fields()
    Eb, Hb = b.fields()
    assert np.array_equal(Ea, Eb) and np.array_equal(Ha, Hb)


@pytest.mark.parametrize("precision", ["FP64", "FP32_OFFSET"])
def test_one_pass_pair_and_profiled_parts_interleave(precision):
    # A field-only run alternates between two sets of E and H arrays; the
    # profiled step (three part graphs, no swap) taken after an odd number
    # of steps must continue from the current set.
    p = getattr(mg, precision)
    a = make(WALLS[5], p)
    a.step(3)
    a.profile(True)
    a.step(2)
    a.profile(False)
    a.step(3)
    b = make(WALLS[5], p)
    b.step(8)
    Ea, Ha = a.fields()
    Eb, Hb = b.fields()
    if precision == "FP64":
        assert np.array_equal(Ea, Eb) and np.array_equal(Ha, Hb)
    else:
        scale = max(np.max(np.abs(Eb)), np.max(np.abs(Hb)))
        assert np.max(np.abs(Ea - Eb)) < 1e-5 * scale and np.max(np.abs(Ha - Hb)) < 1e-5 * scale


@pytest.mark.parametrize("walls", [WALLS[0], WALLS[4]])
def test_graph_step_precision_form(walls):
    a = make(walls, mg.FP32_OFFSET)
    a.step(30)
    b = make(walls, mg.FP32_OFFSET)
    staged(b, 30)
    Ea, Ha = a.fields()
    Eb, Hb = b.fields()
    scale = max(np.max(np.abs(Eb)), np.max(np.abs(Hb)))
    assert np.max(np.abs(Ea - Eb)) < 1e-5 * scale and np.max(np.abs(Ha - Hb)) < 1e-5 * scale


def laser_foil_run(precision):
    """A small laser-foil run: Mur walls, the analytic laser from x-plane 5,
    a warm foil of electrons and protons."""
    n, h = (48, 24, 24), (0.05, 0.05, 0.05)
    tau = 0.5 / math.sqrt(sum(1 / v ** 2 for v in h))
    r = mg.Run(n, h, tau, (2, 2, 2), (2, 2, 2), precision=precision, capacity=20000)
    z = np.zeros(r.field_shape())
    r.set_fields(z, z)
    r.set_laser(a0=3.0, waist=0.4, x_focus=1.4, duration=2.0, t_start=0.0, phase=0.0, plane=5, margin=3)
    r.place_uniform((28, 6, 6), (34, 18, 18), 4, -30 * 4 * math.pi ** 2 / 4, -1.0, uth=(0.05,) * 3)
    r.place_uniform((28, 6, 6), (34, 18, 18), 4, 30 * 4 * math.pi ** 2 / 4, 1.0 / 1836, uth=(0.001,) * 3,
                    skip=7 * 6 * 12 * 12 * 4, id0=1 + 6 * 12 * 12 * 4)
    r.init()
    return r


@pytest.mark.parametrize("precision,tol", [("FP64", 1e-12), ("FP32_OFFSET", 1e-4)])
def test_graph_step_with_markers_and_laser(precision, tol):
    """With markers and the analytic laser: the current sums' atomics make
    the two paths differ at round-off only in FP64; in FP32 the graph's
    fused E pass and the staged passes also round differently (contraction
    into fused multiply-adds), and the driven foil amplifies that to about
    4e-5 of the field scale over 80 steps (bound 1e-4, the precision form's
    tolerance against the reference)."""
    p = getattr(mg, precision)
    a = laser_foil_run(p)
    rows = a.step(80)
    b = laser_foil_run(p)
    rows_b = []
    for _ in range(80):
        b.em_HHalfStep()
        we, wm = b.em_energy()
        b.plasma_move()
        wt = b.plasma_temperature()
        b.em_HStep()
        b.em_EStep_start()
        b.jbc_finish()
        b.em_EStep_finish()
        rows_b.append((we, wm) + tuple(wt))
    rows_b = np.array(rows_b)
    Ea, Ha = a.fields()
    Eb, Hb = b.fields()
    assert np.max(np.abs(Eb)) > 1.0                     # the laser entered
    scale = max(np.max(np.abs(Eb)), np.max(np.abs(Hb)))
    assert np.max(np.abs(Ea - Eb)) < tol * scale and np.max(np.abs(Ha - Hb)) < tol * scale
    tot = np.max(np.abs(rows_b.sum(1)))
    assert np.max(np.abs(rows[:, 1:6] - rows_b)) < tol * tot
    ma = np.sort(a.markers(), order="id")
    mb = np.sort(b.markers(), order="id")
    assert np.array_equal(ma["id"], mb["id"])
    for f in ("x", "y", "z"):
        assert np.max(np.abs(ma[f] - mb[f])) < tol * 10
