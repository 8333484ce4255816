"""Test infrastructure: ctypes binding of the CPU restatement in
``oracle/pic_oracle.c`` (built by ``oracle/Makefile`` target ``port``)."""
import ctypes as C
import os
import subprocess

import numpy as np

from refrun import MARKER_DTYPE, ROOT

LIB_PATH = os.path.join(ROOT, "oracle", "_build", "libpic_oracle.so")


def build():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "port"],
                   check=True)


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    I3 = C.c_int * 3
    D3 = C.c_double * 3
    vp = C.c_void_p
    lib.po_create.restype = vp
    lib.po_create.argtypes = [I3, D3, C.c_double, I3, I3, C.c_double]
    lib.po_destroy.argtypes = [vp]
    for f in ("po_set_fields", "po_get_fields"):
        getattr(lib, f).argtypes = [vp, vp, vp]
    lib.po_get_current.argtypes = [vp, vp]
    lib.po_set_markers.argtypes = [vp, vp, C.c_long]
    lib.po_marker_count.restype = C.c_long
    lib.po_marker_count.argtypes = [vp]
    lib.po_get_markers.argtypes = [vp, vp]
    lib.po_set_laser.argtypes = [vp, vp]
    lib.po_init.argtypes = [vp]
    lib.po_step.argtypes = [vp, vp]
    lib.po_step_probes.argtypes = [vp, vp, C.c_int, vp, vp]
    lib.po_fields_n.argtypes = [vp, vp, vp]
    lib.po_add_mirror.argtypes = [vp, vp, C.c_int, C.c_double, C.c_double, vp, vp]
    lib.po_set_tfsf.restype = C.c_int
    lib.po_set_tfsf.argtypes = [vp, vp, vp]
    lib.po_tfsf_faces.restype = C.c_long
    lib.po_tfsf_faces.argtypes = [vp, vp]
    lib.po_tfsf_recorded.restype = C.c_long
    lib.po_tfsf_recorded.argtypes = [vp, vp]
    lib.po_time.restype = C.c_double
    lib.po_time.argtypes = [vp]
    lib.po_em_energy.argtypes = [vp, vp, vp]
    lib.po_rho.argtypes = [vp, vp]
    lib.po_mesh_size.restype = C.c_long
    lib.po_mesh_size.argtypes = [vp]
    lib.po_region.argtypes = [vp, vp, vp]
    lib.po_gauss.argtypes = [vp, vp, vp, vp]
    lib.po_set_gauss_spot.argtypes = [vp, vp]
    lib.po_ranmar_init.argtypes = [vp, C.c_int, C.c_int]
    lib.po_ranmar.argtypes = [vp, vp, C.c_long]
    lib.po_place_count.restype = C.c_long
    lib.po_place_count.argtypes = [vp]
    lib.po_place.restype = C.c_long
    lib.po_place.argtypes = [vp, vp, vp]
    lib.po_laser_ey.restype = C.c_double
    lib.po_laser_ey.argtypes = [vp] + [C.c_double] * 6
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


class Laser(C.Structure):
    _fields_ = [("a0", C.c_double), ("waist", C.c_double), ("x_focus", C.c_double),
                ("duration", C.c_double), ("t_start", C.c_double), ("phase", C.c_double),
                ("plane", C.c_int), ("margin", C.c_int)]


class Place(C.Structure):
    _fields_ = [("lo", C.c_int * 3), ("hi", C.c_int * 3), ("ppc", C.c_int),
                ("rho", C.c_double), ("qDivM", C.c_double),
                ("drift", C.c_double * 3), ("uth", C.c_double * 3),
                ("seed_ij", C.c_int), ("seed_kl", C.c_int), ("skip", C.c_long),
                ("id0", C.c_int)]


TFSF_PLAY, TFSF_REC, TFSF_BACK = 0, 1, 2


class Tfsf(C.Structure):
    """po_tfsf_t (oracle/pic_oracle.h)."""
    _fields_ = [("lo", C.c_int * 3), ("hi", C.c_int * 3), ("mode", C.c_int),
                ("open", (C.c_int * 3) * 2), ("frames", C.c_int)]


def place(lo, hi, ppc, rho, qDivM, h, drift=(0, 0, 0), uth=(0, 0, 0),
          seed=(1802, 9373), skip=0, id0=1):
    s = Place((C.c_int * 3)(*lo), (C.c_int * 3)(*hi), ppc, rho, qDivM,
              (C.c_double * 3)(*drift), (C.c_double * 3)(*uth), seed[0], seed[1],
              skip, id0)
    n = lib().po_place_count(C.byref(s))
    out = np.zeros(n, MARKER_DTYPE)
    lib().po_place(C.byref(s), (C.c_double * 3)(*h), out.ctypes.data)
    return out


def ranmar(ij, kl, n):
    state = C.create_string_buffer(97 * 8 + 3 * 8 + 2 * 4 + 64)
    lib().po_ranmar_init(state, ij, kl)
    out = np.zeros(n, "<f8")
    lib().po_ranmar(state, out.ctypes.data, n)
    return out


class PoGaussSpot(C.Structure):
    _fields_ = [(f, C.c_double) for f in ("ampl", "frequency", "x", "y", "z", "width", "duration",
                                          "front_offset", "t_plateau")] + [("ey", C.c_int), ("ez", C.c_int)]


class OracleRun:
    def __init__(self, n, h, tau, bc_min, bc_max, time=0.0):
        self.n = tuple(int(v) for v in n)
        I3, D3 = C.c_int * 3, C.c_double * 3
        self.ptr = lib().po_create(I3(*self.n), D3(*h), tau, I3(*bc_min), I3(*bc_max), time)

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().po_destroy(self.ptr)
            self.ptr = None

    def shape(self):
        return (self.n[0] + 1, self.n[1] + 1, self.n[2] + 1, 3)

    def set_fields(self, E, H):
        E = np.ascontiguousarray(E, "<f8")
        H = np.ascontiguousarray(H, "<f8")
        lib().po_set_fields(self.ptr, E.ctypes.data, H.ctypes.data)

    def fields(self):
        E = np.zeros(self.shape())
        H = np.zeros(self.shape())
        lib().po_get_fields(self.ptr, E.ctypes.data, H.ctypes.data)
        return E, H

    def current(self):
        J = np.zeros((self.n[0] + 5, self.n[1] + 5, self.n[2] + 5, 3))
        lib().po_get_current(self.ptr, J.ctypes.data)
        return J

    def set_markers(self, m):
        m = np.ascontiguousarray(m, MARKER_DTYPE)
        lib().po_set_markers(self.ptr, m.ctypes.data, len(m))

    def markers(self):
        n = lib().po_marker_count(self.ptr)
        out = np.zeros(n, MARKER_DTYPE)
        lib().po_get_markers(self.ptr, out.ctypes.data)
        return out

    def set_laser(self, **kw):
        self._laser = Laser(**kw)
        lib().po_set_laser(self.ptr, C.byref(self._laser))

    def set_gauss_spot(self, **kw):
        self._gspot = PoGaussSpot(**kw)
        lib().po_set_gauss_spot(self.ptr, C.byref(self._gspot))

    def init(self):
        lib().po_init(self.ptr)

    def step(self, k=1):
        rows = np.zeros((k, 5))
        for s in range(k):
            lib().po_step(self.ptr, rows[s].ctypes.data)
        return rows

    def step_probes(self, ijk, k=1):
        """k steps with the probe samples of each (core/diag_probe.c:409-429):
        (k, nprobes, 7) rows {t, Ex, Ey, Ez, Hx, Hy, Hz} of E^n and H^n."""
        a = np.ascontiguousarray(np.asarray(ijk, dtype=np.int32).reshape(-1, 3))
        out = np.zeros((k, len(a), 7))
        for s in range(k):
            lib().po_step_probes(self.ptr, a.ctypes.data, len(a), out[s].ctypes.data,
                                 np.zeros(5).ctypes.data)
        return out

    def add_mirror(self, values, direction, r0, t0, E, H):
        """Focused-laser mirror from a .EM_sources/laser file's values and profiles."""
        v = np.ascontiguousarray(values, dtype="<f8")
        self._mirrors = getattr(self, "_mirrors", []) + [(np.ascontiguousarray(E, "<f8"), np.ascontiguousarray(H, "<f8"))]
        e, h = self._mirrors[-1]
        lib().po_add_mirror(self.ptr, v.ctypes.data, int(direction), float(r0), float(t0), e.ctypes.data, h.ctypes.data)

    def fields_n(self):
        """E^n and H^n of the coming step over [0, n]^3 (state unchanged)."""
        E = np.zeros(self.shape())
        H = np.zeros(self.shape())
        lib().po_fields_n(self.ptr, E.ctypes.data, H.ctypes.data)
        return E, H

    def set_tfsf(self, lo, hi, mode, open=((0, 0, 0), (0, 0, 0)), frames=0, **kw):
        """TF/SF interface; play modes take the recorded frames (k, size)."""
        t = Tfsf((C.c_int * 3)(*lo), (C.c_int * 3)(*hi), mode,
                 ((C.c_int * 3) * 2)(*[(C.c_int * 3)(*o) for o in open]), frames)
        data = kw.get("frames_data")
        self._tfsf_frames = np.ascontiguousarray(data, dtype="<f8") if data is not None else None
        ptr = self._tfsf_frames.ctypes.data if self._tfsf_frames is not None else None
        if lib().po_set_tfsf(self.ptr, C.byref(t), ptr) != 0:
            raise ValueError("TF/SF face closer than 5 cells to a wall")

    def tfsf_faces(self):
        """(24, 6) face regions {min, max} in the recorded stream order."""
        out = np.zeros((24, 6), np.int32)
        lib().po_tfsf_faces(self.ptr, out.ctypes.data)
        return out

    def tfsf_recorded(self):
        n = lib().po_tfsf_recorded(self.ptr, None)
        size = lib().po_tfsf_faces(self.ptr, None)
        out = np.zeros((n, size))
        lib().po_tfsf_recorded(self.ptr, out.ctypes.data)
        return out

    def time(self):
        return lib().po_time(self.ptr)

    def _rho_mesh(self):
        m = np.zeros(lib().po_mesh_size(self.ptr))
        lib().po_rho(self.ptr, m.ctypes.data)
        return m

    def rho(self):
        """Charge density over nodes [-2, n+2]^3 (walls folded)."""
        m = self._rho_mesh()
        out = np.zeros((self.n[0] + 5, self.n[1] + 5, self.n[2] + 5))
        lib().po_region(self.ptr, m.ctypes.data, out.ctypes.data)
        return out

    def step_gauss(self, k=1):
        """k steps with the Gauss-law test around each (plasma_gaussTest.c):
        rows {t, max |drho/dt + div J|, max |div E - rho|}, t at the start of
        the step as the reference prints it."""
        rows = np.zeros((k, 3))
        rho2 = self._rho_mesh()
        out = np.zeros(2)
        for s in range(k):
            rho1 = rho2
            rows[s, 0] = self.time()
            lib().po_step(self.ptr, np.zeros(5).ctypes.data)
            rho2 = self._rho_mesh()
            lib().po_gauss(self.ptr, rho1.ctypes.data, rho2.ctypes.data, out.ctypes.data)
            rows[s, 1:] = out
        return rows
