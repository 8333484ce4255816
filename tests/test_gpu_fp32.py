"""Precision form (integer cell + FP32 offset markers, FP32 fields, FP64
reductions) against the FP64 form and the reference golden outputs.

Tolerances: fields and marker state within 1e-4 relative of the reference
after a few steps (FP32 rounding is ~6e-8 per operation); energy histories of
a 32^3 thermal plasma within 1e-4 relative of the FP64 form over 200 steps.
"""
import math

import numpy as np
import pytest

import cases
import parity

pytestmark = pytest.mark.gpu

mg = pytest.importorskip("mandor3_b200")


def fp32_run(name, g):
    case, m0, E0, H0 = parity.initial_state(name, g["h"])
    r = mg.Run(case["n"], g["h"], g["tau"], case["bc_min"], case["bc_max"],
               precision=mg.FP32_OFFSET)
    r.set_fields(E0, H0)
    r.set_markers(m0)
    r.init()
    rows = r.step(case["steps"])
    return case, r, rows


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_fp32_matches_reference_within_single_precision(name):
    g = parity.load_golden(name)
    case, r, rows = fp32_run(name, g)
    E, H = r.fields()
    assert parity.rel_err(E, g["E"]) < 1e-4
    assert parity.rel_err(H, g["H"]) < 1e-4
    got, want = parity.by_id(r.markers()), parity.by_id(g["markers"])
    assert len(got) == len(want) and np.array_equal(got["id"], want["id"])
    for a, ax in enumerate("xyz"):
        assert np.max(np.abs(got[ax] - want[ax])) < 1e-4 * g["h"][a]
    u = np.stack([want["vx"], want["vy"], want["vz"]])
    for ax in ("vx", "vy", "vz"):
        assert np.max(np.abs(got[ax] - want[ax])) < 1e-4 * max(np.max(np.abs(u)), 1e-30)
    # Energy rows: each quantity within 1e-4 of the run's total energy scale
    # (small quantities such as a cold slab's thermal energy carry FP32
    # rounding relative to the whole system, not to themselves).
    d = g["diag"]
    scale = float(np.max(np.abs(d[:, 1:6].sum(1))))
    for c in range(5):
        np.testing.assert_allclose(rows[1:, 1 + c], d[:, 1 + c], rtol=1e-4, atol=1e-4 * scale)


def thermal_plasma(precision, steps, sort_every=0):
    """32^3 periodic plasma at the critical density, h = 0.05 c/omega_p,
    Courant 0.5, 8 electrons per cell from ranmar (1802, 9373), u_th = 0.01."""
    n = (32, 32, 32)
    hh = 0.05 / (2 * math.pi)
    h = (hh, hh, hh)
    tau = 0.5 / math.sqrt(3 / hh ** 2)
    r = mg.Run(n, h, tau, (0, 0, 0), (0, 0, 0), precision=precision, sort_every=sort_every)
    z = np.zeros(r.field_shape())
    r.set_fields(z, z)
    r.place_uniform((0, 0, 0), n, 8, -4 * math.pi ** 2 / 8, -1.0, uth=(0.01, 0.01, 0.01))
    r.init()
    return r, r.step(steps)


def test_fp32_energy_history_tracks_fp64():
    _, r64 = thermal_plasma(mg.FP64, 200)
    _, r32 = thermal_plasma(mg.FP32_OFFSET, 200)
    wt64 = r64[:, 3:6].sum(1)
    wt32 = r32[:, 3:6].sum(1)
    tot64 = r64[:, 1] + r64[:, 2] + wt64
    tot32 = r32[:, 1] + r32[:, 2] + wt32
    assert np.max(np.abs(tot32 - tot64) / np.abs(tot64)) < 1e-4
    assert np.max(np.abs(wt32 - wt64) / np.abs(wt64)) < 1e-4


def test_fp32_sorting_does_not_change_the_physics():
    _, a = thermal_plasma(mg.FP32_OFFSET, 60, sort_every=1)
    _, b = thermal_plasma(mg.FP32_OFFSET, 60, sort_every=10000)
    tot_a = a[:, 1] + a[:, 2] + a[:, 3:6].sum(1)
    tot_b = b[:, 1] + b[:, 2] + b[:, 3:6].sum(1)
    assert np.max(np.abs(tot_a - tot_b) / np.abs(tot_b)) < 1e-5


def test_fp32_markers_round_trip():
    n, h = (10, 12, 14), (0.03, 0.04, 0.05)
    tau = 0.4 * min(h) / math.sqrt(3)
    import oracle_port
    m = oracle_port.place((0, 0, 0), n, 3, -1.0, -1.0, h, uth=(0.1, 0.2, 0.3))
    r = mg.Run(n, h, tau, (0, 0, 0), (0, 0, 0), precision=mg.FP32_OFFSET)
    r.set_markers(m)
    got = parity.by_id(r.markers())
    want = parity.by_id(m)
    for a, ax in enumerate("xyz"):
        assert np.array_equal(np.floor(got[ax] / h[a]), np.floor(want[ax] / h[a]))
        assert np.max(np.abs(got[ax] - want[ax])) < 1e-7 * h[a]
    for ax in ("vx", "vy", "vz"):
        np.testing.assert_allclose(got[ax], want[ax], rtol=1e-7)


def test_fp32_device_placer_matches_fp64_placement():
    n, h = (12, 10, 16), (0.03, 0.04, 0.05)
    tau = 0.4 * min(h) / math.sqrt(3)
    spec = dict(lo=(1, 2, 3), hi=(11, 9, 16), ppc=5, rho=-3.0, qDivM=-1.0,
                drift=(0.1, 0.0, -0.2), uth=(0.05, 0.02, 0.01), seed=(4321, 777), skip=12345,
                id0=100)
    r32 = mg.Run(n, h, tau, (0, 0, 0), (0, 0, 0), precision=mg.FP32_OFFSET)
    r32.place_uniform(**spec)
    r64 = mg.Run(n, h, tau, (0, 0, 0), (0, 0, 0))
    r64.place_uniform(**spec)
    a, b = parity.by_id(r32.markers()), parity.by_id(r64.markers())
    assert np.array_equal(a["id"], b["id"])
    for q, ax in enumerate("xyz"):
        assert np.array_equal(np.floor(a[ax] / h[q]), np.floor(b[ax] / h[q]))
        assert np.max(np.abs(a[ax] - b[ax])) < 1e-7 * h[q]


def beams(sort_every, n=(20, 12, 28), bc=(0, 1, 0), drift=0.3, steps=20, tile=(0, 0, 0), warps=0):
    """Two counter-drifting electron beams on a grid whose sides are not
    multiples of the tile, mirror walls on y, 6 markers per cell each."""
    hh = 0.05 / (2 * math.pi)
    h = (hh, 1.1 * hh, 0.9 * hh)
    tau = 0.5 / math.sqrt(sum(1 / x ** 2 for x in h))
    r = mg.Run(n, h, tau, bc, bc, precision=mg.FP32_OFFSET, sort_every=sort_every, tile=tile,
               tile_warps=warps)
    z = np.zeros(r.field_shape())
    r.set_fields(z, z)
    rho = -4 * math.pi ** 2 / 12
    r.place_uniform((0, 0, 0), n, 6, rho, -1.0, drift=(drift, 0.0, 0.5 * drift),
                    uth=(0.02, 0.02, 0.02), seed=(11, 22))
    r.place_uniform((0, 0, 0), n, 6, rho, -1.0, drift=(-drift, 0.0, -0.5 * drift),
                    uth=(0.02, 0.02, 0.02), seed=(33, 44), id0=10 ** 6)
    r.init()
    rows = r.step(steps)
    return r, rows


@pytest.mark.parametrize("tile,warps", [((0, 0, 0), 0), ((4, 4, 4), 0), ((8, 8, 8), 0),
                                        ((0, 0, 0), 4), ((0, 0, 0), 16), ((4, 4, 4), 16)])
def test_tiled_push_matches_untiled_push(tile, warps):
    # The tiled push sums currents in fixed point per tile, the untiled one
    # in FP32 atomics: the two agree to single-precision round-off, for every
    # tile shape and block size the push is built for.
    rt, a = beams(0, tile=tile, warps=warps)
    ru, b = beams(-1)
    scale = float(np.max(np.abs(b[:, 1:6].sum(1))))
    np.testing.assert_allclose(a[:, 1:], b[:, 1:], rtol=1e-5, atol=1e-6 * scale)
    Jt, Ju = rt.current(), ru.current()
    assert np.max(np.abs(Jt - Ju)) <= 1e-4 * np.max(np.abs(Ju))
    got, want = parity.by_id(rt.markers()), parity.by_id(ru.markers())
    assert np.array_equal(got["id"], want["id"])
    for ax in "xyz":
        assert np.max(np.abs(got[ax] - want[ax])) < 1e-4 * 0.05


def slabs(sort_every, steps=20):
    """A dense slab (24 markers per cell) and a sparse one (2 per cell, two
    cells thick): the tiles over the sparse slab hold fewer markers than the
    shared-memory staging threshold, those over the dense one more."""
    n = (32, 16, 16)
    hh = 0.05 / (2 * math.pi)
    h = (hh, hh, hh)
    tau = 0.5 / math.sqrt(sum(1 / x ** 2 for x in h))
    r = mg.Run(n, h, tau, (0, 0, 0), (0, 0, 0), precision=mg.FP32_OFFSET, sort_every=sort_every)
    z = np.zeros(r.field_shape())
    r.set_fields(z, z)
    rho = -4 * math.pi ** 2 / 24
    r.place_uniform((2, 0, 0), (10, 16, 16), 24, rho, -1.0, drift=(0.3, 0.1, 0.0),
                    uth=(0.05, 0.05, 0.05), seed=(11, 22))
    r.place_uniform((21, 0, 0), (23, 16, 16), 2, 12 * rho, -1.0, drift=(-0.3, 0.0, 0.1),
                    uth=(0.05, 0.05, 0.05), seed=(33, 44), id0=10 ** 6)
    r.init()
    rows = r.step(steps)
    return r, rows


def test_sparse_and_dense_tiles_match_the_untiled_push():
    rt, a = slabs(0)
    ru, b = slabs(-1)
    scale = float(np.max(np.abs(b[:, 1:6].sum(1))))
    np.testing.assert_allclose(a[:, 1:], b[:, 1:], rtol=1e-5, atol=1e-6 * scale)
    Jt, Ju = rt.current(), ru.current()
    assert np.max(np.abs(Jt - Ju)) <= 1e-4 * np.max(np.abs(Ju))
    got, want = parity.by_id(rt.markers()), parity.by_id(ru.markers())
    assert np.array_equal(got["id"], want["id"])
    for ax in "xyz":
        assert np.max(np.abs(got[ax] - want[ax])) < 1e-4 * 0.05


def test_tiled_push_handles_markers_far_from_their_tile():
    # Sorted once at init: after 120 steps at 0.6c most markers sit several
    # cells away from the tile they were sorted into.
    rt, a = beams(10 ** 6, drift=0.6, steps=120)
    ru, b = beams(-1, drift=0.6, steps=120)
    tot_a = a[:, 1] + a[:, 2] + a[:, 3:6].sum(1)
    tot_b = b[:, 1] + b[:, 2] + b[:, 3:6].sum(1)
    assert np.max(np.abs(tot_a - tot_b) / np.abs(tot_b)) < 1e-4
    assert rt.marker_count() == ru.marker_count()


def test_tile_shape_outside_the_built_set_is_rejected():
    with pytest.raises(mg.MandorError) as e:
        mg.Run((8, 8, 8), (0.1,) * 3, 0.02, (0, 0, 0), (0, 0, 0), precision=mg.FP32_OFFSET, tile=(2, 4, 4))
    assert e.value.code == -2
    with pytest.raises(mg.MandorError) as e:
        mg.Run((8, 8, 8), (0.1,) * 3, 0.02, (0, 0, 0), (0, 0, 0), precision=mg.FP32_OFFSET, tile_warps=6)
    assert e.value.code == -2 and "warps" in str(e.value)
