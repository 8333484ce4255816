"""Batches of independent runs (one graph launch per step for all runs):
every run of a batch follows the same history as the same run stepped
alone."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

mg = pytest.importorskip("mandor3_b200")

N_CR = 4 * math.pi ** 2


def thermal(n, ppc, precision, seed):
    hh = 0.05 / (2 * math.pi)
    tau = 0.5 / math.sqrt(3 / hh ** 2)
    r = mg.Run(n, (hh,) * 3, tau, (0, 0, 0), (0, 0, 0), precision=precision)
    z = np.zeros(r.field_shape())
    r.set_fields(z, z)
    r.place_uniform((0, 0, 0), n, ppc, -N_CR / ppc, -1.0, uth=(0.05, 0.05, 0.05), seed=seed)
    r.init()
    return r


def foil(n, precision):
    h = (0.05,) * 3
    tau = 0.5 / math.sqrt(3 / 0.05 ** 2)
    r = mg.Run(n, h, tau, (2, 2, 2), (2, 2, 2), precision=precision)
    z = np.zeros(r.field_shape())
    r.set_fields(z, z)
    r.set_laser(a0=2.0, waist=0.3, x_focus=0.5 * n[0] * h[0], duration=2.0, t_start=0.0, phase=0.0,
                plane=3, margin=2)
    lo, hi = (n[0] // 2, 2, 2), (n[0] // 2 + 4, n[1] - 2, n[2] - 2)
    r.place_uniform(lo, hi, 4, -10 * N_CR / 4, -1.0, seed=(7, 8))
    r.init()
    return r


SPECS = [lambda: thermal((12, 10, 8), 6, mg.FP64, (1, 2)),
         lambda: thermal((20, 12, 28), 8, mg.FP32_OFFSET, (3, 4)),
         lambda: foil((32, 16, 16), mg.FP32_OFFSET),
         lambda: foil((24, 12, 12), mg.FP64)]


def test_batch_matches_runs_stepped_alone():
    alone = [spec() for spec in SPECS]
    rows_alone = [r.step(40) for r in alone]
    runs = [spec() for spec in SPECS]
    b = mg.Batch(runs)
    rows = b.step(25)
    more = b.step(15)
    for q, (a, r) in enumerate(zip(rows_alone, runs)):
        got = np.concatenate([rows[q], more[q]])
        tol = 1e-10 if r.precision == mg.FP64 else 1e-5
        scale = float(np.max(np.abs(a[:, 1:6].sum(1))))
        np.testing.assert_allclose(got, a, rtol=tol, atol=tol * scale)
        assert abs(r.time() - alone[q].time()) < 1e-12
        assert r.marker_count() == alone[q].marker_count()
    b.close()
    # The runs keep working on their own afterwards.
    r = runs[1]
    r.step(3)


def test_batch_refuses_a_run_that_is_not_initialised():
    r = thermal((8, 8, 8), 2, mg.FP64, (5, 6))
    r2 = mg.Run((8, 8, 8), (0.1,) * 3, 0.02, (0, 0, 0), (0, 0, 0))
    with pytest.raises(mg.MandorError) as e:
        mg.Batch([r, r2])
    assert e.value.code == -4
