"""Placement into caller-owned device memory without any allocation
(mg_place_uniform_static), checked against the allocating entry point
mg_run_place_uniform on two calls in a row, and against the CPU oracle's
placer (oracle/pic_oracle.c po_place).

The entry point exists for callers that cannot call cudaMalloc: a host
application whose own caching allocator already holds the GPU's memory and
hands this library slices of it, and code that must not take the implicit
device-wide synchronisation of cudaMalloc/cudaFree.  Here the test itself
provides the output arrays (torch tensors), the library provides only a
fixed static scratch array.  This file is collected last so that a run
stopping at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
mg = pytest.importorskip("mandor3_b200")

import oracle_port  # noqa: E402


class DeviceMarkers(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in ("x", "y", "z", "vx", "vy", "vz", "rho", "qDivM", "id")]


def _lib():
    lib = mg.load()
    lib.mg_place_uniform_static.argtypes = [C.POINTER(mg.Place), C.POINTER(C.c_double),
                                            C.POINTER(DeviceMarkers), C.c_longlong, C.c_int,
                                            C.c_void_p]
    lib.mg_place_uniform_static.restype = C.c_int
    return lib


def _spec(lo, hi, ppc, rho, qDivM, drift, uth, seed, skip, id0):
    return mg.Place((C.c_int * 3)(*lo), (C.c_int * 3)(*hi), ppc, rho, qDivM,
                    (C.c_double * 3)(*drift), (C.c_double * 3)(*uth), seed[0], seed[1],
                    skip, id0)


def place_static(kw, h, capacity, threads=0):
    dev = torch.device("cuda", 0)
    f64 = {f: torch.zeros(capacity, dtype=torch.float64, device=dev)
           for f in ("x", "y", "z", "vx", "vy", "vz")}
    f32 = {f: torch.zeros(capacity, dtype=torch.float32, device=dev) for f in ("rho", "qDivM")}
    ids = torch.zeros(capacity, dtype=torch.int32, device=dev)
    dm = DeviceMarkers(*[t.data_ptr() for t in (f64["x"], f64["y"], f64["z"], f64["vx"],
                                                f64["vy"], f64["vz"], f32["rho"],
                                                f32["qDivM"], ids)])
    spec = _spec(**kw)
    rc = _lib().mg_place_uniform_static(C.byref(spec), (C.c_double * 3)(*h), C.byref(dm),
                                        capacity, threads, None)
    torch.cuda.synchronize()
    if rc:
        raise mg.MandorError(rc, mg.load().mg_last_error().decode())
    n = int(np.prod([b - a for a, b in zip(kw["lo"], kw["hi"])])) * kw["ppc"]
    out = np.zeros(n, mg.MARKER_DTYPE)
    for f in f64:
        out[f] = f64[f][:n].cpu().numpy()
    out["rho"] = f32["rho"][:n].cpu().numpy()
    out["qDivM"] = f32["qDivM"][:n].cpu().numpy()
    out["id"] = ids[:n].cpu().numpy()
    return out


def place_with_run(kw, n_cells, h):
    tau = 0.4 * min(h) / np.sqrt(3)
    with mg.Run(n_cells, h, tau, (0, 0, 0), (0, 0, 0)) as r:
        r.place_uniform(**kw)
        return np.sort(r.markers(), order="id")


CALLS = [
    dict(lo=(1, 2, 3), hi=(11, 9, 16), ppc=5, rho=-3.0, qDivM=-1.0, drift=(0.1, 0.0, -0.2),
         uth=(0.05, 0.02, 0.01), seed=(4321, 777), skip=12345, id0=100),
    dict(lo=(0, 0, 0), hi=(12, 10, 16), ppc=3, rho=2.5, qDivM=1.0 / 1836, drift=(0.0, 0.3, 0.0),
         uth=(0.2, 0.2, 0.2), seed=(1802, 9373), skip=0, id0=1),
]


def test_static_placement_matches_allocating_entry_point_twice():
    n_cells, h = (12, 10, 16), (0.03, 0.04, 0.05)
    for kw in CALLS:                      # two calls in a row share the scratch
        got = np.sort(place_static(kw, h, capacity=6000), order="id")
        want = place_with_run(kw, n_cells, h)
        assert len(got) == len(want)
        assert np.array_equal(got["id"], want["id"])
        for f in ("x", "y", "z", "vx", "vy", "vz", "rho", "qDivM"):
            assert np.array_equal(got[f], want[f]), f        # the same kernel and draws
        # The CPU oracle's placer: positions and momenta bit-exact.
        ref = np.sort(oracle_port.place(h=h, **kw), order="id")
        assert np.array_equal(got["id"], ref["id"])
        for f in ("x", "y", "z", "vx", "vy", "vz", "rho", "qDivM"):
            assert np.array_equal(got[f], ref[f]), f


def test_static_placement_rejects_what_does_not_fit():
    h = (0.03, 0.04, 0.05)
    with pytest.raises(mg.MandorError) as e:
        place_static(CALLS[0], h, capacity=6000, threads=5000)     # more states than the scratch
    assert e.value.code == -2 and "4096" in str(e.value)
    with pytest.raises(mg.MandorError) as e:
        place_static(CALLS[0], h, capacity=100)                    # output arrays too small
    assert e.value.code == -5
