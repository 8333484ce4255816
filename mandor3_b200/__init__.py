"""B200-native particle-in-cell core with the capabilities of Mandor's
``core.out`` hot path.

The compute lives in ``libmandor_b200.so`` (hand-written sm_100a CUDA kernels
behind the C ABI declared in ``include/mandor_b200.h``).  This module is a
thin ctypes mirror of that ABI for Python callers; there is no CPU fallback:
importing the package without the built library, or creating a run without
a CUDA device, raises.
"""
import ctypes as C
import os

import numpy as np

__all__ = ["Run", "Params", "Laser", "Place", "MARKER_DTYPE", "MandorError",
           "BC_PERIODIC", "BC_MIRROR", "BC_OPEN", "FP64", "FP32_OFFSET",
           "library_path", "load"]

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmandor_b200.so")

BC_PERIODIC, BC_MIRROR, BC_OPEN = 0, 1, 2
FP64, FP32_OFFSET = 0, 1

# marker_t with the tracer id (reference type_marker.h:12-25), 64 bytes.
MARKER_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"),
                         ("vx", "<f8"), ("vy", "<f8"), ("vz", "<f8"),
                         ("rho", "<f4"), ("qDivM", "<f4"), ("id", "<i4"),
                         ("pad", "<i4")])

ERRORS = {-1: "cuda", -2: "argument", -3: "out of memory", -4: "stage order",
          -5: "capacity", -6: "bounds", -7: "io", -8: "admission", -9: "timeout"}


class MandorError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s error (%d): %s" % (ERRORS.get(code, "unknown"), code, msg))
        self.code = code


class Params(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("h", C.c_double * 3), ("tau", C.c_double),
                ("bc_min", C.c_int * 3), ("bc_max", C.c_int * 3), ("time", C.c_double),
                ("precision", C.c_int), ("device", C.c_int), ("capacity", C.c_longlong),
                ("sort_every", C.c_int), ("tile", C.c_int * 3), ("tile_warps", C.c_int)]


class Laser(C.Structure):
    _fields_ = [("a0", C.c_double), ("waist", C.c_double), ("x_focus", C.c_double),
                ("duration", C.c_double), ("t_start", C.c_double), ("phase", C.c_double),
                ("plane", C.c_int), ("margin", C.c_int)]


class GaussSpot(C.Structure):
    _fields_ = [("ampl", C.c_double), ("frequency", C.c_double), ("x", C.c_double),
                ("y", C.c_double), ("z", C.c_double), ("width", C.c_double),
                ("duration", C.c_double), ("front_offset", C.c_double), ("t_plateau", C.c_double),
                ("ey", C.c_int), ("ez", C.c_int)]


TFSF_PLAY_FORWARD, TFSF_RECORD, TFSF_PLAY_BACKWARD = 0, 1, 2


class Tfsf(C.Structure):
    """mg_tfsf_t: TF/SF interface box, mode, open faces, frames, ring slots."""
    _fields_ = [("lo", C.c_int * 3), ("hi", C.c_int * 3), ("mode", C.c_int),
                ("open", (C.c_int * 3) * 2), ("frames", C.c_int), ("ring", C.c_int)]


class Mirror(C.Structure):
    """mg_mirror_t: a focused-laser mirror file's values, direction, units and profiles."""
    _fields_ = [("values", C.c_double * 9), ("direction", C.c_int), ("r0", C.c_double),
                ("t0", C.c_double), ("E", C.c_void_p), ("H", C.c_void_p)]


class TwoStream(C.Structure):
    _fields_ = [("gamma", C.c_double), ("qDivM", C.c_double), ("n", C.c_int * 3), ("m", C.c_int * 3),
                ("L", C.c_double * 3), ("id0", C.c_int)]


class DfUniform(C.Structure):
    _fields_ = [("rho", C.c_double), ("qDivM", C.c_double), ("ux", C.c_double), ("uy", C.c_double),
                ("uz", C.c_double), ("dux", C.c_double), ("duy", C.c_double), ("duz", C.c_double),
                ("ppc", C.c_int), ("lambda_cm", C.c_double), ("draws_before", C.c_longlong)]


class Maxwell(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("layers", C.c_int),
                ("omega_pe2", C.c_double), ("qDivM", C.c_double), ("ux", C.c_double),
                ("uy", C.c_double), ("uz", C.c_double), ("tune_energy", C.c_int),
                ("uniform_weight", C.c_int), ("id0", C.c_int)]


class Foil(C.Structure):
    _fields_ = [("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double), ("lx", C.c_double),
                ("ly", C.c_double), ("lz", C.c_double), ("width", C.c_double), ("shift", C.c_double),
                ("profile", C.c_int), ("n1", C.c_double), ("n2", C.c_double), ("q", C.c_double),
                ("M", C.c_double), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("lambda_cm", C.c_double), ("id0", C.c_int)]


class Place(C.Structure):
    _fields_ = [("lo", C.c_int * 3), ("hi", C.c_int * 3), ("ppc", C.c_int),
                ("rho", C.c_double), ("qDivM", C.c_double),
                ("drift", C.c_double * 3), ("uth", C.c_double * 3),
                ("seed_ij", C.c_int), ("seed_kl", C.c_int), ("skip", C.c_longlong),
                ("id0", C.c_int)]


_lib = None


def library_path():
    return LIB_PATH


def load():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libmandor_b200.so is not built; run `python -m mandor3_b200.build` "
                          "(the B200 core has no CPU path)")
    lib = C.CDLL(LIB_PATH)
    vp, i, ll, d = C.c_void_p, C.c_int, C.c_longlong, C.c_double
    sig = {
        "mg_run_create": [C.POINTER(Params), C.POINTER(vp)],
        "mg_run_destroy": [vp],
        "mg_run_set_fields": [vp, vp, vp],
        "mg_run_get_fields": [vp, vp, vp],
        "mg_run_get_current": [vp, vp],
        "mg_run_set_markers": [vp, vp, ll],
        "mg_run_get_markers": [vp, vp, ll, C.POINTER(ll)],
        "mg_run_marker_count": [vp, C.POINTER(ll)],
        "mg_run_set_laser": [vp, vp],
        "mg_run_set_time": [vp, d],
        "mg_run_get_time": [vp, C.POINTER(d)],
        "mg_run_place_uniform": [vp, C.POINTER(Place)],
        "mg_run_init": [vp],
        "mg_em_HHalfStep": [vp],
        "mg_em_energy": [vp, C.POINTER(d), C.POINTER(d)],
        "mg_plasma_move": [vp],
        "mg_plasma_temperature": [vp, C.POINTER(d), C.POINTER(d), C.POINTER(d)],
        "mg_em_HStep": [vp],
        "mg_em_EStep_start": [vp],
        "mg_jbc_finish": [vp],
        "mg_em_EStep_finish": [vp],
        "mg_plasma_rho": [vp, vp],
        "mg_run_step": [vp, i, vp],
        "mg_run_step_async": [vp, i, vp],
        "mg_run_synchronize": [vp],
        "mg_run_stream": [vp, C.POINTER(vp)],
        "mg_run_kernels_per_step": [vp, C.POINTER(i)],
        "mg_run_device_bytes": [vp, C.POINTER(ll)],
        "mg_run_profile": [vp, i],
        "mg_run_last_timing": [vp, C.POINTER(d), C.POINTER(d)],
        "mg_run_set_gauss_spot": [vp, vp],
        "mg_run_set_tfsf": [vp, vp],
        "mg_run_snapshot": [vp, vp, vp, vp, C.c_longlong, vp],
        "mg_run_snapshot_wait": [vp],
        "mg_run_add_mirror": [vp, vp],
        "mg_run_clear_mirrors": [vp],
        "mg_run_place_two_stream": [vp, vp],
        "mg_run_df_uniform": [vp, C.c_longlong, C.c_longlong, vp],
        "mg_run_shift_velocity": [vp, C.c_longlong, C.c_longlong, vp],
        "mg_run_tfsf_faces": [vp, vp, vp],
        "mg_run_tfsf_put_frames": [vp, i, i, vp],
        "mg_run_tfsf_recorded": [vp, i, vp],
        "mg_run_set_probes": [vp, vp, i],
        "mg_run_probe_samples": [vp, i, vp],
        "mg_tecplot_fields": [vp, vp, vp],
        "mg_tecplot_currents": [vp, vp],
        "mg_run_place_maxwell": [vp, vp],
        "mg_run_place_foil": [vp, vp],
        "mg_gauss_before": [vp],
        "mg_gauss_after": [vp, vp],
        "mg_run_step_gauss": [vp, i, vp],
        "mg_batch_create": [C.POINTER(vp), i, C.POINTER(vp)],
        "mg_batch_step": [vp, i, C.POINTER(C.POINTER(d))],
        "mg_batch_destroy": [vp],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = i
    lib.mg_estimate_bytes.argtypes = [C.POINTER(Params), ll]
    lib.mg_estimate_bytes.restype = ll
    lib.mg_last_error.restype = C.c_char_p
    lib.mg_version.restype = C.c_char_p
    _lib = lib
    return lib


def _check(rc):
    if rc != 0:
        raise MandorError(rc, load().mg_last_error().decode(errors="replace"))


def _f8(a):
    return np.ascontiguousarray(a, dtype="<f8")


class Run:
    """One simulation held on one GPU (the reference's global meshes and
    marker array, core/main.c:90-91, core/plasma.c:40-43)."""

    def __init__(self, n, h, tau, bc_min, bc_max, time=0.0, precision=FP64,
                 device=0, capacity=0, sort_every=0, tile=(0, 0, 0), tile_warps=0):
        lib = load()
        self.n = tuple(int(v) for v in n)
        self.h = tuple(float(v) for v in h)
        self.tau = float(tau)
        self.precision = precision
        p = Params((C.c_int * 3)(*self.n), (C.c_double * 3)(*self.h), self.tau,
                   (C.c_int * 3)(*bc_min), (C.c_int * 3)(*bc_max), float(time),
                   int(precision), int(device), int(capacity), int(sort_every),
                   (C.c_int * 3)(*tile), int(tile_warps))
        self._params = p
        ptr = C.c_void_p()
        _check(lib.mg_run_create(C.byref(p), C.byref(ptr)))
        self.ptr = ptr

    def close(self):
        if getattr(self, "ptr", None):
            load().mg_run_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state ------------------------------------------------------------
    def field_shape(self):
        return (self.n[0] + 1, self.n[1] + 1, self.n[2] + 1, 3)

    def set_fields(self, E=None, H=None):
        Ea = _f8(E) if E is not None else None
        Ha = _f8(H) if H is not None else None
        for a in (Ea, Ha):
            if a is not None and a.size != int(np.prod(self.field_shape())):
                raise ValueError("field arrays must hold %s doubles" % (self.field_shape(),))
        _check(load().mg_run_set_fields(self.ptr, Ea.ctypes.data if Ea is not None else None,
                                        Ha.ctypes.data if Ha is not None else None))

    def fields(self):
        E = np.zeros(self.field_shape())
        H = np.zeros(self.field_shape())
        _check(load().mg_run_get_fields(self.ptr, E.ctypes.data, H.ctypes.data))
        return E, H

    def current(self):
        J = np.zeros((self.n[0] + 5, self.n[1] + 5, self.n[2] + 5, 3))
        _check(load().mg_run_get_current(self.ptr, J.ctypes.data))
        return J

    def rho(self):
        r = np.zeros((self.n[0] + 5, self.n[1] + 5, self.n[2] + 5))
        _check(load().mg_plasma_rho(self.ptr, r.ctypes.data))
        return r

    def set_markers(self, m):
        m = np.ascontiguousarray(m, MARKER_DTYPE)
        _check(load().mg_run_set_markers(self.ptr, m.ctypes.data if len(m) else None, len(m)))

    def marker_count(self):
        n = C.c_longlong()
        _check(load().mg_run_marker_count(self.ptr, C.byref(n)))
        return n.value

    def markers(self):
        n = self.marker_count()
        out = np.zeros(n, MARKER_DTYPE)
        got = C.c_longlong()
        _check(load().mg_run_get_markers(self.ptr, out.ctypes.data if n else None, n, C.byref(got)))
        return out[:got.value]

    def set_laser(self, **kw):
        self._laser = Laser(**kw)
        _check(load().mg_run_set_laser(self.ptr, C.byref(self._laser)))

    def set_probes(self, ijk):
        """Probe nodes (q, 3) ints; every step records E^n and H^n there."""
        a = np.ascontiguousarray(np.asarray(ijk, dtype="<i4").reshape(-1, 3))
        self.nprobes = len(a)
        _check(load().mg_run_set_probes(self.ptr, a.ctypes.data if len(a) else None, len(a)))

    def probe_samples(self, nsteps):
        """(nsteps, nprobes, 7) rows {t, Ex, Ey, Ez, Hx, Hy, Hz} of the last step call."""
        out = np.zeros((nsteps, getattr(self, "nprobes", 0), 7))
        _check(load().mg_run_probe_samples(self.ptr, int(nsteps), out.ctypes.data))
        return out

    def tecplot_fields(self):
        """Node-centred E and H (IO_tecplot.c interpolation) over [0, n]^3."""
        E, H = np.zeros(self.field_shape()), np.zeros(self.field_shape())
        _check(load().mg_tecplot_fields(self.ptr, E.ctypes.data, H.ctypes.data))
        return E, H

    def tecplot_current(self):
        J = np.zeros(self.field_shape())
        _check(load().mg_tecplot_currents(self.ptr, J.ctypes.data))
        return J

    def place_maxwell(self, nx, ny, nz, layers, omega_pe2, qDivM, ux, uy, uz, tune_energy=0,
                      uniform_weight=1, id0=1):
        """[plasma] + [DF:Maxwell] of setup.out on the device (quiet start)."""
        s = Maxwell(nx, ny, nz, layers, omega_pe2, qDivM, ux, uy, uz, tune_energy, uniform_weight, id0)
        _check(load().mg_run_place_maxwell(self.ptr, C.byref(s)))

    def place_foil(self, x0, y0, z0, lx, ly, lz, width, n1, n2, q, M, nx, ny, nz, shift=0.0,
                   profile=0, lambda_cm=1e-4, id0=1):
        """[DF:foil] of setup.out on the device."""
        s = Foil(x0, y0, z0, lx, ly, lz, width, shift, profile, n1, n2, q, M, nx, ny, nz, lambda_cm, id0)
        _check(load().mg_run_place_foil(self.ptr, C.byref(s)))

    def set_gauss_spot(self, **kw):
        """Hard gauss-spot source (the fields of .gaussSpot.cfg); no
        arguments switch it off."""
        self._gspot = GaussSpot(**kw) if kw else None
        _check(load().mg_run_set_gauss_spot(self.ptr, C.byref(self._gspot) if kw else None))

    def snapshot(self):
        """Starts an asynchronous copy of the checkpoint state (mg_run_snapshot);
        returns a function that waits for it and gives (E, H, markers)."""
        E = np.zeros(self.field_shape())
        H = np.zeros(self.field_shape())
        cap = max(self.marker_count(), 1)
        m = np.zeros(cap, MARKER_DTYPE)
        n = C.c_longlong()
        _check(load().mg_run_snapshot(self.ptr, E.ctypes.data, H.ctypes.data, m.ctypes.data, cap,
                                      C.byref(n)))
        def wait():
            _check(load().mg_run_snapshot_wait(self.ptr))
            return E, H, m[:n.value]
        return wait

    def add_mirror(self, values, direction, r0, t0, E, H):
        """Focused-laser mirror (mg_run_add_mirror): the nine values and the
        direction of a mirror file, units r0 and t0, and its E and H profiles
        ((n1-9)(n2-9), 4) doubles."""
        E, H = _f8(E), _f8(H)
        s = Mirror((C.c_double * 9)(*[float(v) for v in values]), int(direction), float(r0), float(t0),
                   E.ctypes.data, H.ctypes.data)
        _check(load().mg_run_add_mirror(self.ptr, C.byref(s)))

    def clear_mirrors(self):
        _check(load().mg_run_clear_mirrors(self.ptr))

    def place_two_stream(self, gamma, qDivM, n, m, L, id0=1):
        """[DF:two-stream] markers (mg_run_place_two_stream)."""
        s = TwoStream(gamma, qDivM, (C.c_int * 3)(*n), (C.c_int * 3)(*m), (C.c_double * 3)(*L), id0)
        _check(load().mg_run_place_two_stream(self.ptr, C.byref(s)))

    def df_uniform(self, first, count, rho, qDivM, u, du, ppc, lambda_cm, draws_before=0):
        """[DF:uniform] on placed markers [first, first + count)."""
        s = DfUniform(rho, qDivM, u[0], u[1], u[2], du[0], du[1], du[2], ppc, lambda_cm, draws_before)
        _check(load().mg_run_df_uniform(self.ptr, int(first), int(count), C.byref(s)))

    def shift_velocity(self, first, count, dv):
        """[velocity shift]: u += dv on placed markers [first, first + count)."""
        _check(load().mg_run_shift_velocity(self.ptr, int(first), int(count), (C.c_double * 3)(*dv)))

    def set_tfsf(self, lo=None, hi=None, mode=TFSF_PLAY_FORWARD, open=((0, 0, 0), (0, 0, 0)), frames=0,
                 ring=2):
        """TF/SF interface (mg_run_set_tfsf); no box removes it."""
        if lo is None:
            _check(load().mg_run_set_tfsf(self.ptr, None))
            return
        t = Tfsf((C.c_int * 3)(*lo), (C.c_int * 3)(*hi), mode,
                 ((C.c_int * 3) * 2)(*[(C.c_int * 3)(*o) for o in open]), frames, ring)
        _check(load().mg_run_set_tfsf(self.ptr, C.byref(t)))

    def tfsf_faces(self):
        """((24, 6) face regions {min, max}, doubles per frame)."""
        regions = np.zeros((24, 6), np.int32)
        size = C.c_longlong(0)
        _check(load().mg_run_tfsf_faces(self.ptr, regions.ctypes.data, C.byref(size)))
        return regions, size.value

    def tfsf_put_frames(self, first, frames):
        """Frames first, first + 1, ... ((k, frame size) doubles) to the device ring."""
        a = np.ascontiguousarray(frames, dtype="<f8")
        _check(load().mg_run_tfsf_put_frames(self.ptr, int(first), len(a), a.ctypes.data))

    def tfsf_recorded(self, nsteps):
        """(nsteps, frame size) recorded frames of the last step call."""
        _, size = self.tfsf_faces()
        out = np.zeros((nsteps, size))
        _check(load().mg_run_tfsf_recorded(self.ptr, int(nsteps), out.ctypes.data))
        return out

    def place_uniform(self, lo, hi, ppc, rho, qDivM, drift=(0, 0, 0), uth=(0, 0, 0),
                      seed=(1802, 9373), skip=0, id0=1):
        s = Place((C.c_int * 3)(*lo), (C.c_int * 3)(*hi), int(ppc), float(rho), float(qDivM),
                  (C.c_double * 3)(*drift), (C.c_double * 3)(*uth), int(seed[0]), int(seed[1]),
                  int(skip), int(id0))
        _check(load().mg_run_place_uniform(self.ptr, C.byref(s)))

    def set_time(self, t):
        _check(load().mg_run_set_time(self.ptr, float(t)))

    def time(self):
        t = C.c_double()
        _check(load().mg_run_get_time(self.ptr, C.byref(t)))
        return t.value

    def init(self):
        _check(load().mg_run_init(self.ptr))

    # -- stage API (core/main.c:353-478) -----------------------------------
    def em_HHalfStep(self):
        _check(load().mg_em_HHalfStep(self.ptr))

    def em_energy(self):
        we, wm = C.c_double(), C.c_double()
        _check(load().mg_em_energy(self.ptr, C.byref(we), C.byref(wm)))
        return we.value, wm.value

    def plasma_move(self):
        _check(load().mg_plasma_move(self.ptr))

    def plasma_temperature(self):
        v = [C.c_double() for _ in range(3)]
        _check(load().mg_plasma_temperature(self.ptr, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def em_HStep(self):
        _check(load().mg_em_HStep(self.ptr))

    def em_EStep_start(self):
        _check(load().mg_em_EStep_start(self.ptr))

    def jbc_finish(self):
        _check(load().mg_jbc_finish(self.ptr))

    def em_EStep_finish(self):
        _check(load().mg_em_EStep_finish(self.ptr))

    # -- whole steps -----------------------------------------------------------
    def step(self, nsteps=1):
        """Runs nsteps steps; returns rows {t, W_E, W_M, W_Tx, W_Ty, W_Tz}."""
        rows = np.zeros((nsteps, 6))
        _check(load().mg_run_step(self.ptr, int(nsteps), rows.ctypes.data if nsteps else None))
        return rows

    def step_gauss(self, nsteps=1):
        """nsteps steps with the Gauss-law test around each: rows {t,
        max |drho/dt + div J|, max |div E - rho|} (output/gauss_test.dat)."""
        rows = np.zeros((nsteps, 3))
        _check(load().mg_run_step_gauss(self.ptr, int(nsteps), rows.ctypes.data))
        return rows

    def gauss_before(self):
        _check(load().mg_gauss_before(self.ptr))

    def gauss_after(self):
        out = np.zeros(2)
        _check(load().mg_gauss_after(self.ptr, out.ctypes.data))
        return out

    def step_async(self, nsteps, energies_dev=None):
        _check(load().mg_run_step_async(self.ptr, int(nsteps), energies_dev))

    def synchronize(self):
        _check(load().mg_run_synchronize(self.ptr))

    def stream(self):
        s = C.c_void_p()
        _check(load().mg_run_stream(self.ptr, C.byref(s)))
        return s.value

    def kernels_per_step(self):
        k = C.c_int()
        _check(load().mg_run_kernels_per_step(self.ptr, C.byref(k)))
        return k.value

    def device_bytes(self):
        b = C.c_longlong()
        _check(load().mg_run_device_bytes(self.ptr, C.byref(b)))
        return b.value

    def profile(self, enable=True):
        _check(load().mg_run_profile(self.ptr, int(enable)))

    def last_timing(self):
        a, b = C.c_double(), C.c_double()
        _check(load().mg_run_last_timing(self.ptr, C.byref(a), C.byref(b)))
        return a.value, b.value


class Batch:
    """Independent runs of one GPU stepped together: one CUDA graph launch
    per step, each run's step graph a branch of it (no counterpart in the
    reference, which runs one simulation per process)."""

    def __init__(self, runs):
        self.runs = list(runs)
        arr = (C.c_void_p * len(self.runs))(*[r.ptr.value for r in self.runs])
        ptr = C.c_void_p()
        _check(load().mg_batch_create(arr, len(self.runs), C.byref(ptr)))
        self.ptr = ptr

    def step(self, nsteps):
        """Steps every run nsteps times; returns one (nsteps, 6) array of
        energy rows per run."""
        rows = [np.zeros((nsteps, 6)) for _ in self.runs]
        ptrs = (C.POINTER(C.c_double) * len(rows))(
            *[r.ctypes.data_as(C.POINTER(C.c_double)) for r in rows])
        _check(load().mg_batch_step(self.ptr, int(nsteps), ptrs))
        return rows

    def close(self):
        if getattr(self, "ptr", None):
            load().mg_batch_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def estimate_bytes(n, h, tau, bc_min, bc_max, markers, precision=FP64):
    p = Params((C.c_int * 3)(*n), (C.c_double * 3)(*h), float(tau), (C.c_int * 3)(*bc_min),
               (C.c_int * 3)(*bc_max), 0.0, int(precision), 0, 0, 0)
    return load().mg_estimate_bytes(C.byref(p), int(markers))
