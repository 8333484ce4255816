"""Freezes the reference's output for every case of tests/cases.py.

Runs the reference setup.out / core.out (built from the reference sources by
oracle/Makefile into oracle/_ref) on each case's initial state and stores the
final markers, E, H and the diag.dat energy rows in tests/golden/<case>.npz;
for two cases also the Gauss-law rows of core_gauss.out in
tests/golden/gauss_<case>.npz, and the fields of an empty Mur box driven by
the hard gauss-spot source in tests/golden/gauss_spot.npz; the reference
placers, tecplot dumps, probes and spectral dumps, and TF/SF record and
play runs in place_*.npz, tecplot.npz, probes.npz and tfsf.npz.

    make -C oracle ref REF=/path/to/reference
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import cases  # noqa: E402
import refrun  # noqa: E402
import oracle_port  # noqa: E402
from refrun import RefRun, have_reference  # noqa: E402


def make(name):
    case = cases.CASES[name]
    n, L_um = cases.geometry(case)
    rr = RefRun()
    try:
        dom = rr.setup(n, L_um, -0.5, case["bc_min"], case["bc_max"])
        h, tau = dom["h"], dom["tau"]
        m0 = oracle_port.place(**cases.placer_args(case, h))
        E0, H0 = cases.initial_fields(case, h)
        rr.set_state(m0, E0, H0)
        rr.run(case["steps"])
        m, E, H = rr.final()
        diag = rr.diag()
        np.savez_compressed(os.path.join(HERE, name + ".npz"), h=h, tau=tau,
                            n_markers0=len(m0), markers=m.tobytes(), E=E, H=H, diag=diag)
        print("%-18s markers %d -> %d, diag rows %d" % (name, len(m0), len(m), len(diag)))
    finally:
        rr.cleanup()


def make_gauss(name):
    """The reference built with MC_GAUSS_TEST (core_gauss.out) on the case:
    its output/gauss_test.dat rows {t, deltaRho_J, deltaRho_E}."""
    case = cases.CASES[name]
    n, L_um = cases.geometry(case)
    rr = RefRun()
    try:
        dom = rr.setup(n, L_um, -0.5, case["bc_min"], case["bc_max"])
        h = dom["h"]
        m0 = oracle_port.place(**cases.placer_args(case, h))
        E0, H0 = cases.initial_fields(case, h)
        rr.set_state(m0, E0, H0)
        rr.run(case["steps"], exe="core_gauss.out")
        rows = np.loadtxt(rr.path("output", "gauss_test.dat"), skiprows=1, ndmin=2)
        np.savez_compressed(os.path.join(HERE, "gauss_" + name + ".npz"), rows=rows)
        print("%-18s gauss rows %d" % (name, len(rows)))
    finally:
        rr.cleanup()


GAUSS_CASES = ("periodic_thermal", "mur_mixed")

# Hard gauss-spot source in an empty Mur box (core/em_gaussSpot.c).
SPOT_N = (20, 16, 16)
SPOT_L_UM = (1.0, 0.8, 0.8)
SPOT_STEPS = 40


def spot_params(h):
    return dict(ampl=2.0, frequency=1.0, x=6 * h[0], y=0.4, z=0.4, width=0.2, duration=0.3,
                front_offset=0.4, t_plateau=0.1, ey=1, ez=-1)


def make_gauss_spot():
    rr = RefRun()
    try:
        dom = rr.setup(SPOT_N, SPOT_L_UM, -0.5, (2, 2, 2), (2, 2, 2))
        h, tau = dom["h"], dom["tau"]
        rr.set_state(np.zeros(0, dtype=oracle_port.MARKER_DTYPE))
        rr.set_gauss_spot(**spot_params(h))
        rr.run(SPOT_STEPS)
        m, E, H = rr.final()
        np.savez_compressed(os.path.join(HERE, "gauss_spot.npz"), h=h, tau=tau, E=E, H=H, diag=rr.diag())
        print("gauss_spot: E max %.3e" % np.max(np.abs(E)))
    finally:
        rr.cleanup()


# The reference placers (see make_placers).
FOIL = dict(n=(24, 8, 8), L_um=(1.2, 0.4, 0.4), bc=(2, 0, 0),
            spec=dict(x0=0.6, y0=0.2, z0=0.2, lx=1.0, ly=0.2, lz=0.0, width=0.2, shift=0.01,
                      profile=1, n1=-20.0, n2=-60.0, q=-1.0, M=1.0, nx=2, ny=2, nz=2))


def placer_deck(cfg):
    """A setup deck with one [DF:foil] tag (setup/tag_foil.c:60-100 order)."""
    from refrun import deck_text
    s = cfg["spec"]
    text = deck_text(cfg["n"], cfg["L_um"], -0.5, cfg["bc"], cfg["bc"])
    text += ("\n[DF:foil]\n@ %.17g\tx0\n@ %.17g\ty0\n@ %.17g\tz0\n@ %.17g\tlx\n@ %.17g\tly\n"
             "@ %.17g\tlz\n@ %.17g\twidth\n> %.17g\tshift\n@ %s\tprofile\n@ %.17g\tn1\n"
             "@ %.17g\tn2\n@ %.17g\tq\n@ %.17g\tM\n@ %d\tnx\n@ %d\tny\n@ %d\tnz\n"
             % (s["x0"], s["y0"], s["z0"], s["lx"], s["ly"], s["lz"], s["width"], s["shift"],
                "linear" if s["profile"] == 0 else "exponential", s["n1"], s["n2"], s["q"], s["M"],
                s["nx"], s["ny"], s["nz"]))
    return text


MAXWELL_SPECS = [dict(nx=2, ny=2, nz=1, layers=4, omega_pe2=1.5, qDivM=-1.0, ux=0.05, uy=0.1, uz=0.02,
                      tune_energy=1, uniform_weight=1),
                 dict(nx=1, ny=2, nz=3, layers=2, omega_pe2=0.7, qDivM=-1.0, ux=0.03, uy=0.03, uz=0.06,
                      tune_energy=0, uniform_weight=0)]


def make_placers():
    """[DF:foil] through setup.out; the Maxwell quiet-start pattern through
    oracle/_ref/maxwell_pattern.out (the reference's sampler and mapper):
    setup.out's own [plasma] + [DF:Maxwell] path cannot serve, because
    tag_plasma.c:109 (`cell[p].vx = p++`) reads and increments p without a
    sequence point, and under GCC the pattern index lands in the next marker."""
    import subprocess
    from refrun import read_markers, read_domain, REF_DIR
    rr = RefRun()
    try:
        with open(rr.path("deck.input"), "w") as fp:
            fp.write(placer_deck(FOIL))
        rr._run("setup.out", "deck.input", "create")
        dom = read_domain(rr.path("binData", "domain.bin"))
        m = read_markers(rr.path("binData", "plasma_000000_000.bin"))
        np.savez_compressed(os.path.join(HERE, "place_foil.npz"), h=dom["h"], tau=dom["tau"],
                            markers=m.tobytes())
        print("place_foil: %d markers" % len(m))
    finally:
        rr.cleanup()
    pats = []
    for s in MAXWELL_SPECS:
        args = [str(s[k]) for k in ("nx", "ny", "nz", "layers", "omega_pe2", "qDivM", "ux", "uy", "uz",
                                    "tune_energy", "uniform_weight")]
        out = subprocess.run([os.path.join(REF_DIR, "maxwell_pattern.out")] + args, stdout=subprocess.PIPE,
                             check=True).stdout.decode()
        pats.append(np.array([[float(v) for v in line.split()] for line in out.splitlines()]))
    np.savez_compressed(os.path.join(HERE, "place_maxwell.npz"), **{"pattern%d" % q: p for q, p in enumerate(pats)})
    print("place_maxwell: patterns of %s markers" % [len(p) for p in pats])


# Tecplot dumps: the reference core.out on the drop-in driver's case with a
# tecplot period of 4 steps (12 steps: records 1..3).
TEC_PERIOD = 4


def read_tecplot(root, num):
    """The arrays of tecplot record num: E, H, J, rho over [0, n]^3 and the
    binary record header {time, cpus, file map id}."""
    from refrun import read_mesh, MESH_HEADER_BYTES
    b = os.path.join(root, "binData")
    out = {}
    for f in ("E", "H", "J"):
        _, hdr, a = read_mesh(os.path.join(b, "tec_%s_%06d(000).bin" % (f, num)))
        out[f] = a
    raw = open(os.path.join(b, "tec_rho_%06d(000).bin" % num), "rb").read()
    out["rho"] = np.frombuffer(raw[MESH_HEADER_BYTES:], "<f8")
    info = open(os.path.join(b, "tec_%06d.txt" % num), "rb").read()
    out["time"] = np.frombuffer(info[:8], "<f8")[0]
    out["ids"] = np.frombuffer(info[8:16], "<i4")
    return out


def make_tecplot():
    import tempfile, shutil, refrun
    import test_driver
    root = tempfile.mkdtemp(prefix="mg_tec_")
    try:
        rr = RefRun(root)
        test_driver.prepare(root)
        with open(os.path.join(root, "run_mandor.cfg"), "w") as fp:
            fp.write("@ %d\ttotal\n@ %d\tfull\n@ %d\ttecplot\n@ 0\tcontinue\n@ %d\tstop\n@ -100\tspectr\n"
                     % (test_driver.CASE["steps"], 10 ** 6, TEC_PERIOD, 10 ** 6))
        rr._run("core.out")
        arrays = {}
        for num in (1, 2, 3):
            t = read_tecplot(root, num)
            for k, v in t.items():
                arrays["%s%d" % (k, num)] = v
        np.savez_compressed(os.path.join(HERE, "tecplot.npz"), **arrays)
        print("tecplot: records 1-3")
    finally:
        shutil.rmtree(root, ignore_errors=True)


# Probes and spectral dumps: the reference core.out on the drop-in driver's
# case with a probe deck (points, a repeat, one outside the domain, a line, a
# rectangle and a volume), spectral dumps every 5 steps and a tecplot dump at
# step 10 (steps 5 and 10: one dump alone, one beside a tecplot dump).
# Probe positions in cells (x h, the case's h is one value on all axes).
PROBE_GROUPS = [
    ("point", (5.3, 4.2, 7.6)),
    ("point", (5.6, 4.4, 7.9)),               # the same node again
    ("point", (12.2, 4.2, 7.6)),              # i = n: outside
    ("line", (0.2, 0.3, 0.1, 11.5, 9.6, 13.7), (3,)),
    ("rectangle", (1.2, 2.1, 3.3, 10.4, 2.1, 3.3, 1.2, 8.7, 3.3), (1, 0)),
    ("volume", (2.5, 1.5, 0.5, 9.5, 1.5, 0.5, 2.5, 7.5, 0.5, 2.5, 1.5, 12.5), (0, 0, 0)),
]


def probe_deck(h):
    lines = []
    for g in PROBE_GROUPS:
        lines.append("@ %s\t\tprobe group" % g[0])
        for q, v in enumerate(g[1]):
            lines.append("> %.9f\t\tcoordinate [micron]" % (v * h[q % 3]))
        for v in (g[2] if len(g) > 2 else ()):
            lines.append("> %d\t\tadditional points" % v)
    lines.append("@ end\t\tterminator")
    return "\n".join(lines) + "\n"
SPECTR_PERIOD = 5
PROBE_TEC_PERIOD = 10


def probe_run_cfg(steps):
    return ("@ %d\ttotal\n@ %d\tfull\n@ %d\ttecplot\n@ 0\tcontinue\n@ %d\tstop\n@ %d\tspectr\n"
            % (steps, 10 ** 6, PROBE_TEC_PERIOD, 10 ** 6, SPECTR_PERIOD))


def probe_files(root):
    """The probe and spectral-dump files of a run directory: name -> bytes."""
    out = {}
    for d in ("binData", "tmp", "output"):
        for f in sorted(os.listdir(os.path.join(root, d))):
            if (f.startswith("probe_") and f.endswith(".bin")) or f.startswith("spectrDump_") \
                    or f in ("spectr.N", "probe_locations.dat"):
                out[d + "/" + f] = open(os.path.join(root, d, f), "rb").read()
    return out


def make_probes():
    import tempfile, shutil
    import test_driver
    root = tempfile.mkdtemp(prefix="mg_probe_")
    try:
        rr = RefRun(root)
        test_driver.prepare(root)
        with open(os.path.join(root, "run_mandor.cfg"), "w") as fp:
            fp.write(probe_run_cfg(test_driver.CASE["steps"]))
        n, L_um = cases.geometry(test_driver.CASE)
        with open(os.path.join(root, "run_probes.cfg"), "w") as fp:
            fp.write(probe_deck([L_um[a] / n[a] for a in range(3)]))
        rr._run("core.out")
        files = probe_files(root)
        np.savez_compressed(os.path.join(HERE, "probes.npz"),
                            **{k: np.frombuffer(v, np.uint8) for k, v in files.items()})
        print("probes: %d files" % len(files))
    finally:
        shutil.rmtree(root, ignore_errors=True)


# TF/SF interface (core/em_TFSF.c): a record run (hard gauss spot inside
# the interface box of an empty Mur box), the reference TFSFdefrag on its
# streams, then play runs forward (with a warm electron cloud across the
# faces) and backward (empty) on the merged streams.
TFSF_N = (18, 14, 14)
TFSF_L_UM = (0.9, 0.7, 0.7)
TFSF_BOX = (5, 12, 5, 8, 5, 8)
TFSF_STEPS = 16


def tfsf_spot(h):
    sp = spot_params(h)
    sp.update(x=8 * h[0], y=0.325, z=0.325)
    return sp


def tfsf_plasma(h):
    return oracle_port.place(lo=(3, 3, 3), hi=(15, 11, 11), ppc=2, rho=-0.5, qDivM=-1.0, h=h,
                             uth=(0.1, 0.1, 0.1), seed=(1802, 9373))


def tfsf_files(d, suffix):
    return {k: open(os.path.join(d, "%s_%s.bin" % (k, suffix)), "rb").read()
            for k in refrun.TFSF_FACES}


def make_tfsf():
    import shutil, glob
    rec, plays = RefRun(), []
    out = {}
    try:
        dom = rec.setup(TFSF_N, TFSF_L_UM, -0.5, (2, 2, 2), (2, 2, 2))
        h = dom["h"]
        rec.set_state(np.zeros(0, dtype=oracle_port.MARKER_DTYPE))
        rec.set_gauss_spot(**tfsf_spot(h))
        rec.set_tfsf(TFSF_BOX, 1)
        rec.run(TFSF_STEPS)
        d = rec.path(".EM_sources", "TFSF")
        for k, v in tfsf_files(d, "000").items():
            out["rec/" + k] = v
        for f in ("consistencyCheck.dat", "TFSF_defrag.map", "lastFrameTime.bin"):
            out["rec/" + f] = open(os.path.join(d, f), "rb").read()
        rec.defrag()
        for k, v in tfsf_files(d, "99999").items():
            out["merged/" + k] = v
        out["merged/lastFrameTime.bin"] = open(os.path.join(d, "lastFrameTime.bin"), "rb").read()
        for mode, plasma in ((0, True), (2, False)):
            play = RefRun()
            plays.append(play)
            play.setup(TFSF_N, TFSF_L_UM, -0.5, (2, 2, 2), (2, 2, 2))
            play.set_state(tfsf_plasma(h) if plasma else np.zeros(0, dtype=oracle_port.MARKER_DTYPE))
            pd = play.path(".EM_sources", "TFSF")
            for f in glob.glob(os.path.join(d, "*_99999.bin")) + [os.path.join(d, "consistencyCheck.dat"),
                                                                 os.path.join(d, "lastFrameTime.bin")]:
                shutil.copy(f, pd)
            play.set_tfsf(TFSF_BOX, mode)
            play.run(TFSF_STEPS)
            m, E, H = play.final()
            out["play%d/E" % mode] = E.tobytes()
            if plasma:
                out["play%d/H" % mode] = H.tobytes()
                out["play%d/diag" % mode] = play.diag().tobytes()
        np.savez_compressed(os.path.join(HERE, "tfsf.npz"), h=np.array(h), tau=dom["tau"],
                            **{k: np.frombuffer(v, np.uint8) for k, v in out.items()})
        print("tfsf: %d entries" % len(out))
    finally:
        rec.cleanup()
        for p in plays:
            p.cleanup()


# Setup tags on the device (row f-4): [DF:two-stream] alone and followed by
# [velocity shift] through setup.out, and [DF:uniform] through the harness
# oracle/_ref/df_uniform.out (the reference tag on 1000 markers, with and
# without earlier rand () draws).
TS = dict(n=(8, 8, 10), L_um=(0.8, 0.8, 1.0), gamma=0.1, qDivM=-1.0, N=(4, 3, 5), m=(1, 2, 1),
          dv=(0.01, -0.02, 0.003))
DF_CASES = [dict(rho=-1.0, qDivM=-1.0, u=(0.01, 0.0, -0.02), du=(2.0, 1.0, 0.5), skip=0, lam=1.0),
            dict(rho=2.5, qDivM=1.0 / 1836, u=(0.0, 0.3, 0.0), du=(0.1, 0.2, 0.3), skip=7, lam=0.8)]
DF_MARKERS = 1000
DF_PPC = 4                      # fixed in oracle/df_uniform_main.c


def two_stream_deck(shift):
    from refrun import deck_text
    text = deck_text(TS["n"], TS["L_um"], -0.5, (0, 0, 0), (0, 0, 0))
    text += ("\n[DF:two-stream]\n@ %.17g\tgamma\n@ %.17g\tq/M\n@ %d\tNx\n@ %d\tNy\n@ %d\tNz\n"
             "@ %d\tmx\n@ %d\tmy\n@ %d\tmz\n" % ((TS["gamma"], TS["qDivM"]) + TS["N"] + TS["m"]))
    if shift:
        text += ("\n[velocity shift]\n@ %.17g\tdvx\n@ %.17g\tdvy\n@ %.17g\tdvz\n@ last\tcomponent\n"
                 % TS["dv"])
    return text


def df_deck(c):
    return "".join("@ %.17g\tvalue\n" % v for v in (c["rho"], c["qDivM"]) + c["u"] + c["du"])


def make_setup_tags():
    import subprocess, tempfile
    out = {}
    for shift in (0, 1):
        rr = RefRun()
        try:
            with open(rr.path("deck.input"), "w") as fp:
                fp.write(two_stream_deck(shift))
            rr._run("setup.out", "deck.input", "create")
            m = refrun.read_markers(rr.path("binData", "plasma_000000_000.bin"))
            out["two_stream%d" % shift] = np.frombuffer(m.tobytes(), np.uint8)
            out["domain"] = np.array(list(refrun.read_domain(rr.path("binData", "domain.bin"))["h"]) +
                                     list(refrun.read_domain(rr.path("binData", "domain.bin"))["L"]))
        finally:
            rr.cleanup()
    for q, c in enumerate(DF_CASES):
        with tempfile.NamedTemporaryFile("w", suffix=".cfg", delete=False) as fp:
            fp.write(df_deck(c))
        res = subprocess.run([os.path.join(refrun.REF_DIR, "df_uniform.out"), repr(c["lam"]), str(DF_MARKERS),
                              str(c["skip"]), fp.name], stdout=subprocess.PIPE, check=True)
        os.remove(fp.name)
        out["df%d" % q] = np.loadtxt(res.stdout.decode().splitlines()[-DF_MARKERS:])
    np.savez_compressed(os.path.join(HERE, "setup_tags.npz"), **out)
    print("setup tags: %s" % sorted(out))


# The reference's focused-laser soft source (scpic/em_mirror.c): setup.out
# computes the mirror profiles ([focused laser], setup/tag_laser.c) into
# .EM_sources/laser/mirror_00, core.out plays them in an empty Mur box;
# once along +x, once along -x.
MIRROR_N = (24, 20, 20)
MIRROR_L_UM = (1.2, 1.0, 1.0)
MIRROR_STEPS = 40


def mirror_deck(direction):
    from refrun import deck_text
    text = deck_text(MIRROR_N, MIRROR_L_UM, -0.5, (2, 2, 2), (2, 2, 2))
    text += ("\n[focused laser]\n@ -1.5\tamplitude\n@ 0.9\tf-number\n@ 0.6\tfocus x\n@ 0.5\tfocus y\n"
             "@ 0.5\tfocus z\n@ 2.0\tduration fs\n@ 3.0\tarrival fs\n@ 0.3\tphase\n@ 10.0\tratio\n"
             "@ %d\tdirection\n" % direction)
    return text


def make_mirror():
    out = {}
    for direction in (1, -1):
        rr = RefRun()
        try:
            with open(rr.path("deck.input"), "w") as fp:
                fp.write(mirror_deck(direction))
            rr._run("setup.out", "deck.input", "create")
            out["file%d" % direction] = np.frombuffer(open(rr.path(".EM_sources", "laser", "mirror_00"), "rb").read(),
                                                      np.uint8)
            out["units%d" % direction] = np.frombuffer(open(rr.path("binData", "units.bin"), "rb").read(), "<f8")
            dom = refrun.read_domain(rr.path("binData", "domain.bin"))
            out["h"], out["tau"] = dom["h"], dom["tau"]
            rr.set_state(np.zeros(0, dtype=oracle_port.MARKER_DTYPE))
            rr.run(MIRROR_STEPS)
            _, E, H = rr.final()
            out["E%d" % direction] = E
            out["H%d" % direction] = H
        finally:
            rr.cleanup()
    np.savez_compressed(os.path.join(HERE, "mirror.npz"), **out)
    print("mirror: E max %.3e / %.3e" % (np.abs(out["E1"]).max(), np.abs(out["E-1"]).max()))


# Runs at the benchmark configurations' sizes and the field-only runs of
# tests/cases.py.
def make_resonator():
    """The cavity eigenmode set up by the reference's own setup.out
    ([EMResonator] Yee_2nd_order) and run by core.out: the initial fields,
    the fields after the run and its diag.dat rows."""
    c = cases.RESONATOR
    rr = RefRun()
    try:
        with open(rr.path("deck.input"), "w") as fp:
            fp.write(cases.resonator_deck())
        rr._run("setup.out", "deck.input", "create")
        dom = refrun.read_domain(rr.path("binData", "domain.bin"))
        _, _, E0 = refrun.read_mesh(rr.path("binData", "sys_E_000000(000).bin"))
        _, _, H0 = refrun.read_mesh(rr.path("binData", "sys_H_000000(000).bin"))
        rr.set_state(np.zeros(0, dtype=oracle_port.MARKER_DTYPE))
        rr.run(c["steps"])
        _, E, H = rr.final()
        np.savez_compressed(os.path.join(HERE, "resonator.npz"), h=dom["h"], tau=dom["tau"], E0=E0, H0=H0,
                            E=E, H=H, diag=rr.diag())
        print("resonator: |E0| %.3e, |E| %.3e after %d steps" % (np.abs(E0).max(), np.abs(E).max(), c["steps"]))
    finally:
        rr.cleanup()


def _run_records(rr, steps, period):
    with open(rr.path("run_mandor.cfg"), "w") as fp:
        fp.write("@ %d\ttotal steps\n@ %d\tcheckpoint period\n@ -1\ttecplot\n@ 0\tcontinue\n"
                 "@ %d\tstop-flag period\n@ -100\tspectral dumps\n" % (steps, period, 10 ** 8))
    rr._run("core.out")


def make_mur_pulse():
    """The free pulse of cases.MUR_PULSE in an empty Mur box: the
    reference's E and H at every checkpoint and its diag.dat rows."""
    c = cases.MUR_PULSE
    n = c["n"]
    rr = RefRun()
    try:
        dom = rr.setup(n, [v * c["h"] for v in n], c["tau"], c["bc"], c["bc"])
        E0, H0 = cases.mur_pulse_fields()
        rr.set_state(np.zeros(0, dtype=oracle_port.MARKER_DTYPE), E0, H0)
        _run_records(rr, c["period"] * c["records"], c["period"])
        out = {}
        for q in range(1, c["records"] + 1):
            _, out["E%d" % q], out["H%d" % q] = rr.final(q)
        np.savez_compressed(os.path.join(HERE, "mur_pulse.npz"), h=dom["h"], tau=dom["tau"], diag=rr.diag(), **out)
        print("mur_pulse: |E| %s" % ["%.3e" % np.abs(out["E%d" % q]).max() for q in range(1, c["records"] + 1)])
    finally:
        rr.cleanup()


def make_thermal_c1():
    """BASELINE configuration 1 (cases.THERMAL_C1) through core.out: the
    diag.dat history of all 200 steps, every 64th marker by id, E and H at
    4096 seeded nodes and the shell power spectra of E and H at the end."""
    c = cases.THERMAL_C1
    n = c["n"]
    rr = RefRun()
    try:
        dom = rr.setup(n, [v * cases.H_LAMBDA for v in n], c["tau"], c["bc"], c["bc"])
        m0 = cases.thermal_c1_markers(dom["h"])
        z = np.zeros((n[0] + 1, n[1] + 1, n[2] + 1, 3))
        rr.set_state(m0, z, z)
        rr.run(c["steps"])
        m, E, H = rr.final()
        m = np.sort(m, order="id")
        keep = m[(m["id"] - 1) % c["sample_every"] == 0]
        nodes = cases.field_sample(n, 4096, 1)
        sel = tuple(nodes.T)
        np.savez_compressed(os.path.join(HERE, "thermal_c1.npz"), h=dom["h"], tau=dom["tau"], diag=rr.diag(),
                            n_markers=len(m), markers=keep.tobytes(), nodes=nodes, E=E[sel], H=H[sel],
                            spec_E=cases.shell_spectrum(E, n), spec_H=cases.shell_spectrum(H, n))
        print("thermal_c1: %d markers, %d sampled, diag rows %d" % (len(m), len(keep), len(rr.diag())))
    finally:
        rr.cleanup()


def make_foil_c2():
    """The grid and foil of BASELINE configuration 2 (cases.FOIL_C2),
    warm, through core.out for 10 steps: every 1024th marker by id, E and
    H at 8192 seeded nodes around the foil and 4096 anywhere, the diag.dat
    rows."""
    c = cases.FOIL_C2
    n = c["n"]
    rr = RefRun()
    try:
        dom = rr.setup(n, [v * c["h"] for v in n], c["tau"], c["bc"], c["bc"])
        m0 = cases.foil_c2_markers(dom["h"])
        rr.set_state(m0)
        rr.run(c["steps"])
        m, E, H = rr.final()
        m = np.sort(m, order="id")
        keep = m[(m["id"] - 1) % c["sample_every"] == 0]
        nodes = np.concatenate([cases.field_sample(n, 8192, 2, ((115, 0, 0), (135, n[1], n[2]))),
                                cases.field_sample(n, 4096, 3)])
        sel = tuple(nodes.T)
        np.savez_compressed(os.path.join(HERE, "foil_c2.npz"), h=dom["h"], tau=dom["tau"], diag=rr.diag(),
                            n_markers=len(m), markers=keep.tobytes(), nodes=nodes, E=E[sel], H=H[sel],
                            E_max=np.abs(E).max(axis=(0, 1, 2)), H_max=np.abs(H).max(axis=(0, 1, 2)))
        print("foil_c2: %d -> %d markers, %d sampled, |E| %.3e" % (len(m0), len(m), len(keep), np.abs(E).max()))
    finally:
        rr.cleanup()


CONFIG_RUNS = {"resonator": make_resonator, "mur_pulse": make_mur_pulse, "thermal_c1": make_thermal_c1,
               "foil_c2": make_foil_c2}


if __name__ == "__main__":
    if not have_reference():
        sys.exit("reference binaries missing: make -C oracle ref REF=<reference tree>")
    for name in (sys.argv[1:] or list(cases.CASES) + ["gauss_spot", "placers", "tecplot", "probes", "tfsf",
                                                 "setup_tags", "mirror"] + list(CONFIG_RUNS)):
        if name in CONFIG_RUNS:
            CONFIG_RUNS[name]()
            continue
        if name == "probes":
            make_probes()
            continue
        if name == "tfsf":
            make_tfsf()
            continue
        if name == "setup_tags":
            make_setup_tags()
            continue
        if name == "mirror":
            make_mirror()
            continue
        if name == "tecplot":
            make_tecplot()
            continue
        if name == "gauss_spot":
            make_gauss_spot()
            continue
        if name == "placers":
            make_placers()
            continue
        make(name)
        if name in GAUSS_CASES:
            make_gauss(name)
