"""Test infrastructure: run the reference Mandor binaries and read/write their
binary formats with numpy.

The reference ``setup.out`` / ``core.out`` are built from the reference
sources by ``oracle/Makefile`` into ``oracle/_ref``.  A run directory gets the
layout ``core.out`` expects (``binData/``, ``output/logs``, ``tmp``,
``.EM_sources``) and a stub ``source/import.pl`` that hands the reference's
command-line parser (source/commandLine.c:89) an empty option list.

Formats (reference file:line):
  * marker file: ``long N`` + N x ``marker_t`` (64 B with the tracer id),
    core/plasma_IO.c:273-287, type_marker.h:12-25;
  * mesh file: 6 x int32 valid region + the 88-byte ``mesh_t`` struct + the
    region's nodes, k fastest, 24 B per vector node, type_mesh.c:285-313;
  * ``diag.dat``: text, 10 columns, core/diag_WDensity.c:89-104.
"""
import os
import shutil
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")

MARKER_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"),
                         ("vx", "<f8"), ("vy", "<f8"), ("vz", "<f8"),
                         ("rho", "<f4"), ("qDivM", "<f4"), ("id", "<i4"),
                         ("pad", "<i4")])
assert MARKER_DTYPE.itemsize == 64

MESH_HEADER_BYTES = 6 * 4 + 88

BC = {"periodic": 0, "mirror": 1, "open": 2, "mur": 2}


def have_reference():
    return all(os.path.exists(os.path.join(REF_DIR, f))
               for f in ("setup.out", "core.out"))


def read_markers(path):
    with open(path, "rb") as fp:
        n = int(np.frombuffer(fp.read(8), "<i8")[0])
        return np.frombuffer(fp.read(n * 64), MARKER_DTYPE).copy()


def write_markers(path, m):
    m = np.ascontiguousarray(m, MARKER_DTYPE)
    with open(path, "wb") as fp:
        fp.write(np.array([len(m)], "<i8").tobytes())
        fp.write(m.tobytes())


def read_mesh(path):
    """Returns (region(6 ints), raw header bytes, array[ni, nj, nk, 3])."""
    with open(path, "rb") as fp:
        raw = fp.read()
    reg = np.frombuffer(raw[:24], "<i4")
    ni, nj, nk = (reg[3] - reg[0] + 1, reg[4] - reg[1] + 1, reg[5] - reg[2] + 1)
    data = np.frombuffer(raw[MESH_HEADER_BYTES:], "<f8")
    return reg.copy(), raw[:MESH_HEADER_BYTES], data.reshape(ni, nj, nk, 3).copy()


def write_mesh(path, header, arr):
    with open(path, "wb") as fp:
        fp.write(header)
        fp.write(np.ascontiguousarray(arr, "<f8").tobytes())


def read_domain(path):
    with open(path, "rb") as fp:
        raw = fp.read()
    d = np.frombuffer(raw[:56], "<f8")
    ints = np.frombuffer(raw[56:104], "<i4")
    return {"h": d[0:3].copy(), "L": d[3:6].copy(), "tau": float(d[6]),
            "dmn_min": ints[0:3].copy(), "dmn_max": ints[3:6].copy(),
            "bc_min": ints[6:9].copy(), "bc_max": ints[9:12].copy()}


def read_diag(path):
    rows = []
    with open(path) as fp:
        for line in fp:
            parts = line.split()
            if len(parts) == 10:
                try:
                    rows.append([float(v) for v in parts])
                except ValueError:
                    pass
    return np.array(rows)


PROBE_SAMPLE = np.dtype([(k, "<f8") for k in ("t", "Ex", "Ey", "Ez", "Hx", "Hy", "Hz")])


def read_probe(raw):
    """A probe file (core/diag_probe.c:86-98, probe.h): probeHeader_t
    {char magic[8] = "probes", int i, j, k} then probeSample_t rows."""
    raw = bytes(raw)
    assert raw[:8] == b"probes\0\0", raw[:8]
    ijk = tuple(int(v) for v in np.frombuffer(raw[8:20], "<i4"))
    return ijk, np.frombuffer(raw[20:], "<f8").reshape(-1, 7)


TFSF_E_FACES = ("Ey_xMin", "Ez_xMin", "Ey_xMax", "Ez_xMax", "Ez_yMin", "Ex_yMin",
                "Ez_yMax", "Ex_yMax", "Ex_zMin", "Ey_zMin", "Ex_zMax", "Ey_zMax")
TFSF_H_FACES = ("Hz_xMin", "Hy_xMin", "Hz_xMax", "Hy_xMax", "Hx_yMin", "Hz_yMin",
                "Hx_yMax", "Hz_yMax", "Hy_zMin", "Hx_zMin", "Hy_zMax", "Hx_zMax")
TFSF_FACES = TFSF_E_FACES + TFSF_H_FACES      # core/em_TFSF.c:86-119


def read_tfsf_stream(raw):
    """A TF/SF face stream (core/em_TFSF.c:256-268, 565-594): reg_t header
    {min[3], max[3], cpu, barcode, wrap[3]} then frames of the region's
    values, the face's first tangential axis slowest.  Returns (header ints,
    frames (k, volume))."""
    raw = bytes(raw)
    head = np.frombuffer(raw[:44], "<i4")
    vol = int(np.prod(head[3:6] - head[0:3] + 1))
    return head, np.frombuffer(raw[44:], "<f8").reshape(-1, vol)


_WS = b" \t\n\r\x0b\x0c"


def read_mirror(raw, n):
    """A focused-laser mirror file (scpic/em_mirror.c:393-481) as core.out
    reads it: the title and dashes lines, nine "@ double" lines, one
    "@ int" line, the dashes line -- each fscanf whitespace directive also
    skipping the whitespace that follows -- then the E and H profiles,
    (n1-9)(n2-9) records of {y_cos, y_sin, z_cos, z_sin}.  Returns (nine
    values, direction, E (nodes, 4), H (nodes, 4))."""
    raw = bytes(raw)
    pos = 0

    def skip_ws(p):
        while p < len(raw) and raw[p:p + 1] in _WS:
            p += 1
        return p
    title = b"Mirror focused laser beam #"
    assert raw.startswith(title)
    pos = raw.index(b"\n") 
    pos = skip_ws(pos)
    dashes = b"-" * 39
    assert raw[pos:pos + 39] == dashes
    pos = skip_ws(pos + 39)
    vals = []
    for _ in range(9):
        assert raw[pos:pos + 1] == b"@"
        end = raw.index(b"\n", pos)
        vals.append(float(raw[pos + 1:end].split()[0]))
        pos = skip_ws(end)
    assert raw[pos:pos + 1] == b"@"
    end = raw.index(b"\n", pos)
    direction = int(raw[pos + 1:end].split()[0])
    pos = end + 1
    assert raw[pos:pos + 39] == dashes
    pos = skip_ws(pos + 39)
    nodes = (n[1] - 9) * (n[2] - 9)
    data = np.frombuffer(raw[pos:pos + 2 * nodes * 32], "<f8").reshape(2, nodes, 4)
    return vals, direction, data[0], data[1]


def read_chunks(raw):
    """A chunk file (type_CFile.c:112-370): the magic, then chunks of
    {INT64 size with header, int deleted, int name length, '\\n', name,
    '\\n', data}; returns [(name, deleted, data bytes)]."""
    raw = bytes(raw)
    magic = b"============\n Chunk file\n============\n"
    assert raw.startswith(magic)
    out, pos = [], len(magic)
    while pos < len(raw):
        size = int(np.frombuffer(raw[pos:pos + 8], "<i8")[0])
        deleted, l = (int(v) for v in np.frombuffer(raw[pos + 8:pos + 16], "<i4"))
        assert raw[pos + 16:pos + 17] == b"\n" and raw[pos + 17 + l:pos + 18 + l] == b"\n"
        name = raw[pos + 17:pos + 17 + l].decode()
        out.append((name, deleted, raw[pos + 18 + l:pos + size]))
        pos += size
    assert pos == len(raw)
    return out


def mesh_header(n, name, ghost=1, vector=True):
    """Header of a checkpoint mesh file for a one-rank run: the valid region
    (0,0,0)-(n) and the mesh_t struct of a mesh allocated over
    [-ghost, n+ghost] (type_mesh.h:67-84; pointers zeroed)."""
    lo = [-ghost] * 3
    hi = [v + ghost for v in n]
    w = [hi[a] - lo[a] + 1 for a in range(3)]
    node = 24 if vector else 8
    ints = [0, 0, 0, n[0], n[1], n[2],
            lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], 1 if vector else 0,
            w[2], w[1] * w[2], node * w[0] * w[1] * w[2]]
    raw = np.array(ints, "<i4").tobytes() + b"\0" * 16
    raw += name.encode().ljust(30, b"\0") + b"\0\0"
    assert len(raw) == MESH_HEADER_BYTES
    return raw


def write_checkpoint0(root, n, h, tau, bc_min, bc_max, E, H, markers, time=0.0):
    """The record-0 file set that core.out loads (what setup.out writes):
    domain.bin, sys.N, sys_000000.txt, file maps, E/H meshes, markers."""
    b = os.path.join(root, "binData")
    for d in ("binData", "output/logs", "tmp"):
        os.makedirs(os.path.join(root, d), exist_ok=True)
    with open(os.path.join(b, "domain.bin"), "wb") as fp:
        fp.write(np.array(list(h) + [n[a] * h[a] for a in range(3)] + [tau], "<f8").tobytes())
        fp.write(np.array([0, 0, 0] + list(n) + list(bc_min) + list(bc_max), "<i4").tobytes())
    with open(os.path.join(b, "sys.N"), "w") as fp:
        fp.write("@ 1\t  system check-point records written.\n")
    with open(os.path.join(b, "sys_000000.txt"), "w") as fp:
        fp.write("@ %.14e    time.\n@ 1       cpus total.\n@ 1       file map id.\n"
                 "That is checkpoint (record of the full system state) #0.\n" % time)
    for i in (0, 1):
        with open(os.path.join(b, "fileMap_%06d.txt" % i), "w") as fp:
            fp.write("1 cpus total.\n0: (0 0 0) - (%d %d %d)\n" % tuple(n))
    with open(os.path.join(b, "fileMap_start.txt"), "w") as fp:
        fp.write("@ 2 filemaps are generated by setup - keep them on the start of simulation.\n")
    with open(os.path.join(b, "fileMap.N"), "w") as fp:
        fp.write("@ 2 filemaps total is written.\n")
    # units.bin: the 15 doubles of units_save (misc_units.c:38-58) for a
    # 1-micron wavelength; core.out only logs them.
    c, m_e, e = 2.99792458e10, 9.1093826e-28, 4.8032044e-10
    lam = 1e-4
    t = lam / c
    om = 2 * np.pi / t
    A = m_e * c * om / e
    n_u = m_e * om ** 2 / (16 * np.pi ** 3 * e ** 2)
    wp = 2 * e * np.sqrt(np.pi * n_u / m_e) * t
    units = [lam, c, t, om, A / (2 * np.pi), 0.0, A, n_u, e * n_u,
             om ** 2 * m_e / (4 * np.pi * e ** 2), 0.0, 1e-4 / lam, 1e-15 / t, wp, 2 * np.pi / wp]
    with open(os.path.join(b, "units.bin"), "wb") as fp:
        fp.write(np.array(units, "<f8").tobytes())
    write_mesh(os.path.join(b, "sys_E_000000(000).bin"), mesh_header(n, "vec_E"), E)
    write_mesh(os.path.join(b, "sys_H_000000(000).bin"), mesh_header(n, "vec_H"), H)
    write_markers(os.path.join(b, "plasma_000000_000.bin"), markers)


def write_run_cfg(root, steps, full, stop=10 ** 8):
    with open(os.path.join(root, "run_mandor.cfg"), "w") as fp:
        fp.write("@ %d\ttotal steps\n@ %d\tcheckpoint period\n@ -1\ttecplot\n"
                 "@ 0\tcontinue\n@ %d\tstop-flag period\n@ -100\tspectral dumps\n"
                 % (steps, full, stop))


def deck_text(n, L_um, tau, bc_min, bc_max, lambda_um=1.0):
    """A minimal setup deck: units, mesh and boundary tags only."""
    lines = ["[units]", "@ %r\tlambda [microns]" % lambda_um, "",
             "[mesh]"]
    # Every value line carries a comment: cfg_readDouble's format
    # "@ %le %*[^\n] " (misc_cfgReader.c:62) would otherwise swallow the
    # next line as the comment.
    lines += ["@ %d\tcells" % v for v in n]
    lines += ["@ %.17g\tlength [microns]" % v for v in L_um]
    lines += ["@ %.17g\ttau" % tau, "", "[boundaryConditions]"]
    for a in range(3):
        lines += ["@ %d\tmin" % bc_min[a], "@ %d\tmax" % bc_max[a]]
    return "\n".join(lines) + "\n"


class RefRun:
    """One reference run directory."""

    def __init__(self, workdir=None):
        self.dir = workdir or tempfile.mkdtemp(prefix="mandor_ref_")
        for d in ("source", "binData", "output/logs", "tmp",
                  ".EM_sources/TFSF", ".EM_sources/laser"):
            os.makedirs(os.path.join(self.dir, d), exist_ok=True)
        stub = os.path.join(self.dir, "source", "import.pl")
        with open(stub, "w") as fp:
            fp.write("#!/bin/sh\necho BYE\n")
        os.chmod(stub, 0o755)

    def path(self, *p):
        return os.path.join(self.dir, *p)

    def setup(self, n, L_um, tau, bc_min, bc_max):
        with open(self.path("deck.input"), "w") as fp:
            fp.write(deck_text(n, L_um, tau, bc_min, bc_max))
        self._run("setup.out", "deck.input", "create")
        return read_domain(self.path("binData", "domain.bin"))

    def set_state(self, markers=None, E=None, H=None):
        if markers is not None:
            write_markers(self.path("binData", "plasma_000000_000.bin"), markers)
        for name, arr in (("E", E), ("H", H)):
            if arr is not None:
                f = self.path("binData", "sys_%s_000000(000).bin" % name)
                _, hdr, _ = read_mesh(f)
                write_mesh(f, hdr, arr)

    def set_gauss_spot(self, ampl, frequency, x, y, z, width, duration, front_offset, t_plateau, ey, ez):
        """.gaussSpot.cfg as setup/tag_gaussSpot.c:126-140 writes it (the
        order core/em_gaussSpot.c:46-56 reads)."""
        vals = [ampl, frequency, x, y, z, width, duration, front_offset, t_plateau]
        with open(self.path(".gaussSpot.cfg"), "w") as fp:
            for v in vals:
                fp.write("@ %.17e\tparameter\n" % v)
            fp.write("@ %d\tEy\n@ %d\tEz\n" % (ey, ez))

    def set_tfsf(self, box, mode, open_faces=None):
        """.EM_sources/TFSF/TFSF.cfg as setup/tag_TFSF.c:164-171 writes it
        (the order core/em_TFSF.c:157-166 reads), and openFaces.cfg
        (setup/tag_TFSFFaces.c) when faces are opened."""
        d = self.path(".EM_sources", "TFSF")
        with open(os.path.join(d, "TFSF.cfg"), "w") as fp:
            for v in box:
                fp.write("@ %5d       TFSF interface bounding box.\n" % v)
            fp.write("@ %5d       Interface regime.\n" % mode)
        if open_faces is not None:
            with open(os.path.join(d, "openFaces.cfg"), "w") as fp:
                for axis in range(3):
                    for top in range(2):
                        fp.write("@ %d\topen face flag\n" % open_faces[top][axis])

    def defrag(self):
        """The reference's TFSFdefrag on the recorded streams, no filter."""
        with open(self.path(".EM_sources", "TFSF", "filter.cfg"), "w") as fp:
            fp.write("@ % 5d       I0.\n@ % 5d       I1.\n@ % 5d       Shift frames.\n"
                     % (-10 ** 6, 10 ** 6, 0))
        self._run("TFSFdefrag.out")

    def run(self, steps, exe="core.out", timeout=3600):
        with open(self.path("run_mandor.cfg"), "w") as fp:
            fp.write("@ %d\ttotal steps\n@ %d\tcheckpoint period\n@ -1\ttecplot\n"
                     "@ 0\tcontinue\n@ %d\tstop-flag period\n@ -100\tspectral dumps\n"
                     % (steps, 10 ** 8, 10 ** 8))
        try:
            os.remove(self.path("tmp", "stop.flag"))
        except FileNotFoundError:
            pass
        out = self._run(exe, timeout=timeout)
        return out

    def final(self, record=1):
        m = read_markers(self.path("binData", "plasma_%06d_000.bin" % record))
        _, _, E = read_mesh(self.path("binData", "sys_E_%06d(000).bin" % record))
        _, _, H = read_mesh(self.path("binData", "sys_H_%06d(000).bin" % record))
        return m, E, H

    def diag(self):
        return read_diag(self.path("binData", "diag.dat"))

    def _run(self, exe, *args, timeout=3600):
        res = subprocess.run([os.path.join(REF_DIR, exe)] + list(args),
                             cwd=self.dir, stdout=subprocess.PIPE,
                             stderr=subprocess.STDOUT, timeout=timeout)
        text = res.stdout.decode(errors="replace")
        if res.returncode != 0:
            raise RuntimeError("%s failed (%d):\n%s" % (exe, res.returncode, text[-3000:]))
        return text

    def cleanup(self):
        shutil.rmtree(self.dir, ignore_errors=True)
