"""Device setup tags (mg_run_place_two_stream, mg_run_shift_velocity,
mg_run_df_uniform) against the reference's outputs (tests/golden/
setup_tags.npz) and the C library's rand ()."""
import numpy as np
import pytest

from test_setup_tags import GOLD, df_uniform, libc_rand, make_golden, markers

pytestmark = pytest.mark.gpu

mg = pytest.importorskip("mandor3_b200")


def run(precision, capacity):
    h, L = tuple(GOLD["domain"][:3]), tuple(GOLD["domain"][3:])
    tau = 0.5 / np.sqrt(sum(1 / v ** 2 for v in h))
    return mg.Run(make_golden.TS["n"], h, tau, (0, 0, 0), (0, 0, 0), precision=precision,
                  capacity=capacity), L


def by_id(m):
    return m[np.argsort(m["id"], kind="stable")]


@pytest.mark.parametrize("precision", [mg.FP64, mg.FP32_OFFSET])
@pytest.mark.parametrize("shift", [0, 1])
def test_two_stream_matches_setup(precision, shift):
    want = markers("two_stream%d" % shift)
    r, L = run(precision, len(want))
    ts = make_golden.TS
    r.place_two_stream(ts["gamma"], ts["qDivM"], ts["N"], ts["m"], L, id0=1)
    if shift:
        r.shift_velocity(0, len(want), ts["dv"])
    got = by_id(r.markers())
    assert len(got) == len(want)
    exact = precision == mg.FP64
    for f in ("x", "y", "z", "vx", "vy", "vz"):
        if exact:
            assert np.array_equal(got[f], want[f]), f
        else:
            np.testing.assert_allclose(got[f], want[f], rtol=2e-7, atol=1e-7, err_msg=f)
    for f in ("rho", "qDivM", "id"):
        assert np.array_equal(got[f], want[f]), f
    r.close()


@pytest.mark.parametrize("precision", [mg.FP64, mg.FP32_OFFSET])
def test_df_uniform_matches_the_reference_tag(precision):
    for q, c in enumerate(make_golden.DF_CASES):
        want = GOLD["df%d" % q]
        n = len(want)
        r, _ = run(precision, n)
        r.place_uniform((0, 0, 0), make_golden.TS["n"], 3, 1.0, 1.0)     # positions only
        count = r.marker_count()
        assert count >= n
        r.df_uniform(0, n, c["rho"], c["qDivM"], c["u"], c["du"], make_golden.DF_PPC, c["lam"] * 1e-4,
                     draws_before=c["skip"])
        got = r.markers()[:n]
        for a, f in enumerate(("vx", "vy", "vz")):
            if precision == mg.FP64:
                assert np.array_equal(got[f], want[:, a]), f
            else:
                assert np.array_equal(got[f], want[:, a].astype(np.float32).astype(np.float64)), f
        assert np.array_equal(got["rho"], want[:, 3].astype(np.float32))
        assert np.array_equal(got["qDivM"], want[:, 4].astype(np.float32))
        r.close()


def test_df_uniform_at_scale_follows_the_c_library():
    """About 300 000 markers after 12 345 earlier draws, threads starting
    from jumped-ahead windows: every draw equals the C library's."""
    c = dict(rho=-1.0, qDivM=-1.0, u=(0.0, 0.1, 0.2), du=(1.0, 2.0, 3.0))
    skip = 12345
    r, _ = run(mg.FP64, 470 * 640)
    r.place_uniform((0, 0, 0), make_golden.TS["n"], 470, 1.0, 1.0)
    n = r.marker_count()
    assert n == 470 * 640
    r.df_uniform(0, n, c["rho"], c["qDivM"], c["u"], c["du"], make_golden.DF_PPC, 1e-4, draws_before=skip)
    got = r.markers()
    u, rho = df_uniform(c, n, libc_rand(3 * n, skip))
    assert np.array_equal(got["vx"], u[:, 0]) and np.array_equal(got["vy"], u[:, 1])
    assert np.array_equal(got["vz"], u[:, 2])
    r.close()


def test_tags_need_unordered_markers():
    r, L = run(mg.FP64, 200)
    ts = make_golden.TS
    r.place_two_stream(ts["gamma"], ts["qDivM"], ts["N"], ts["m"], L)
    with pytest.raises(mg.MandorError):
        r.shift_velocity(0, 1000, (0, 0, 0))
    r.init()
    with pytest.raises(mg.MandorError):
        r.shift_velocity(0, 10, (0.1, 0, 0))
    r.close()
