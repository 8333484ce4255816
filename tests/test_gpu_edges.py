"""Edge cases of the C ABI on the device: runs without markers, capacity
limits and short output buffers are reported as errors, not faults."""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

mg = pytest.importorskip("mandor3_b200")

N = (16, 12, 20)
HH = 0.05 / (2 * math.pi)
TAU = 0.5 / math.sqrt(3 / HH ** 2)


def pulse(r):
    """A transverse E pulse in the middle of the box."""
    E = np.zeros(r.field_shape())
    x = np.arange(N[0] + 1)[:, None, None]
    E[..., 1] = np.exp(-((x - N[0] / 2) / 2.0) ** 2) * np.ones((1, N[1] + 1, N[2] + 1))
    r.set_fields(E, np.zeros(r.field_shape()))


@pytest.mark.parametrize("precision", [mg.FP64, mg.FP32_OFFSET])
def test_a_run_without_markers_steps_its_fields(precision):
    bc = (0, 0, 0)
    r = mg.Run(N, (HH,) * 3, TAU, bc, bc, precision=precision)
    pulse(r)
    r.set_markers(np.zeros(0, mg.MARKER_DTYPE))
    r.init()
    rows = r.step(12)
    assert r.marker_count() == 0
    assert np.all(rows[:, 3:6] == 0.0)                 # no thermal energy
    w = rows[:, 1] + rows[:, 2]
    assert w[0] > 0 and np.max(np.abs(w - w[0])) < 1e-2 * w[0]   # periodic box keeps its field energy
    assert len(r.markers()) == 0
    r.close()


def test_precision_form_capacity_beyond_its_index_range_is_refused():
    with pytest.raises(mg.MandorError) as e:
        mg.Run(N, (HH,) * 3, TAU, (0, 0, 0), (0, 0, 0), precision=mg.FP32_OFFSET, capacity=2 ** 31)
    assert e.value.code == -5


@pytest.mark.parametrize("precision", [mg.FP64, mg.FP32_OFFSET])
def test_short_marker_buffer_is_refused(precision):
    bc = (0, 0, 0)
    r = mg.Run(N, (HH,) * 3, TAU, bc, bc, precision=precision, capacity=N[0] * N[1] * N[2] * 2)
    z = np.zeros(r.field_shape())
    r.set_fields(z, z)
    r.place_uniform((0, 0, 0), N, 2, -0.1, -1.0, uth=(0.01,) * 3)
    r.init()
    n = r.marker_count()
    out = np.zeros(n - 1, mg.MARKER_DTYPE)
    got = C.c_longlong()
    rc = mg.load().mg_run_get_markers(r.ptr, out.ctypes.data, n - 1, C.byref(got))
    assert rc == -5 and got.value == n
    # the run is still usable
    r.step(2)
    assert len(r.markers()) == n
    r.close()
