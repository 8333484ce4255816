"""Throughput benchmark of the B200 PIC core.

Workload (default): the plain FP64 3D laser-foil interaction -- a 256x128x128
grid at 20 cells per wavelength (h = 0.05), Courant 0.5, Mur absorbing walls
on all six faces, an Ey-polarised Gaussian laser (lambda = 1, a0 = 3, waist
3 lambda, 10-cycle sin^2 envelope) injected at x-plane 5 and focused on the
front of a 30 n_cr, 0.5-lambda (10-cell) foil of electrons and protons at 16
markers per cell each (4.46e6 markers, uniform random in-cell positions from
ranmar seeds (1802, 9373), cold), run for 2000 steps: W warm-up steps, then
K timed steps of the same run.  Data are synthetic (no benchmark suite).

One JSON line on rank 0:
  value      particle-steps/s over all ranks, device-resident state, CUDA
             events on the run's stream around K graph-replayed steps;
  e2e        the same metric through the C ABI from pinned host buffers:
             upload of markers and fields, K steps with the energy rows read
             back, download of markers and fields, all inside the timed region;
  roofline   the push kernel (the largest kernel of the step): algorithmic
             bytes per launch (100 B per marker: x and u read and written in
             FP64, the weight read) over its mean launch time, against the
             measured HBM copy bandwidth;
  cpu_baseline  the reference core.out (built from the reference sources,
             oracle/_ref/core_fast.out) on a bounded sample of the same
             workload on this host's cores.

--impl reference times that reference path alone on rank 0 and prints the
same metric.  Under torchrun every rank runs an independent replica (the
path has no data-parallel exchange: replicas only, weak scaling).
"""
import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CR = 4 * math.pi ** 2
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def workload(name="laser_foil"):
    if name == "weibel":
        return weibel()
    if name.startswith("weibel_") and name[7:].isdigit():
        return weibel(int(name[7:]))
    if name != "laser_foil":
        raise SystemExit("unknown workload %r" % name)
    n = (256, 128, 128)
    h = (0.05, 0.05, 0.05)
    tau = 0.5 / math.sqrt(sum(1.0 / v ** 2 for v in h))
    bc = (2, 2, 2)
    ppc = 16
    foil = ((120, 5, 5), (130, 123, 123))           # 10 cells, 5-cell wall margins
    n_each = (foil[1][0] - foil[0][0]) * (foil[1][1] - foil[0][1]) * (foil[1][2] - foil[0][2]) * ppc
    species = [
        dict(lo=foil[0], hi=foil[1], ppc=ppc, rho=-30 * N_CR / ppc, qDivM=-1.0,
             drift=(0, 0, 0), uth=(0, 0, 0), seed=(1802, 9373), skip=0, id0=1),
        dict(lo=foil[0], hi=foil[1], ppc=ppc, rho=30 * N_CR / ppc, qDivM=1.0 / 1836,
             drift=(0, 0, 0), uth=(0, 0, 0), seed=(1802, 9373), skip=7 * n_each, id0=1 + n_each),
    ]
    laser = dict(a0=3.0, waist=3.0, x_focus=foil[0][0] * h[0], duration=10.0, t_start=0.0,
                 phase=0.0, plane=5, margin=5)
    return dict(name="laser_foil_fp64_256x128x128", n=n, h=h, tau=tau, bc=bc, species=species,
                laser=laser, markers=2 * n_each, total_steps=2000, precision=0, dtype="f64",
                bytes_per_marker=100.0)


def weibel(side=256):
    """Counter-streaming electron beams (two-stream/Weibel), precision form:
    256^3 periodic cells, h = 0.05 c/omega_p at the total density n_cr,
    Courant 0.5, beams at u_x = +-0.2 (gamma v = 0.2/sqrt(1 - 0.04)) with
    32 markers per cell each, thermal spread 0.01, 500 steps.  Workload
    "weibel_<side>" is the same plasma on side^3 cells (smaller cases for
    profiling).  The markers are re-sorted every 24 steps (on 128^3, steps
    every 8/16/24/32/48: 5.02/4.87/4.78/4.80/5.03 ms with the sort's cost
    spread over its interval)."""
    n = (side, side, side)
    hh = 0.05 / (2 * math.pi)
    h = (hh, hh, hh)
    tau = 0.5 / math.sqrt(3 / hh ** 2)
    ppc = 32
    each = n[0] * n[1] * n[2] * ppc
    u = 0.2 / math.sqrt(1 - 0.04)
    species = [
        dict(lo=(0, 0, 0), hi=n, ppc=ppc, rho=-0.5 * N_CR / ppc, qDivM=-1.0,
             drift=(u, 0, 0), uth=(0.01, 0.01, 0.01), seed=(1802, 9373), skip=0, id0=1),
        dict(lo=(0, 0, 0), hi=n, ppc=ppc, rho=-0.5 * N_CR / ppc, qDivM=-1.0,
             drift=(-u, 0, 0), uth=(0.01, 0.01, 0.01), seed=(1802, 9373), skip=7 * each,
             id0=1 + each),
    ]
    return dict(name="weibel_fp32_%dcubed" % side, n=n, h=h, tau=tau, bc=(0, 0, 0), species=species,
                laser=None, markers=2 * each, total_steps=500, precision=1, dtype="f32",
                bytes_per_marker=60.0, sort_every=24)


def make_run(w, device):
    import mandor3_b200 as mg
    r = mg.Run(w["n"], w["h"], w["tau"], w["bc"], w["bc"], device=device, capacity=w["markers"],
               precision=w["precision"], sort_every=w.get("sort_every", 0))
    z = np.zeros(r.field_shape())
    r.set_fields(z, z)
    if w["laser"]:
        r.set_laser(**w["laser"])
    for s in w["species"]:
        r.place_uniform(**s)
    r.init()
    return r


class Clocks:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def hbm_peak():
    try:
        with open(PEAKS_FILE) as fp:
            return float(json.load(fp)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(w, markers):
    """DRAM bytes per push launch from the committed ncu summary of the
    workload's push kernel, if any: the summary's bytes per marker (captured
    on the same kernel, scaled by markers) or its bytes per launch."""
    name = "push64_laser_foil.md" if w["precision"] == 0 else "push32_weibel.md"
    try:
        text = open(os.path.join(ROOT, "profiles", name)).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_marker:\s*([0-9.eE+]+)", text)
    if m:
        return float(m.group(1)) * markers
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", text)
    return float(m.group(1)) if m and w["name"].startswith("laser_foil") else None


# ---------------------------------------------------------------------------
# Reference CPU path (the reference core.out built from its sources).
# ---------------------------------------------------------------------------
def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_sample(w, steps, procs=None):
    """Runs the reference core_fast.out on the workload's grid and markers
    for `steps` steps as `procs` independent single-rank processes at once
    (default: one per host core, fewer if host memory is short).  The
    reference's only parallelism is MPI domain decomposition and no MPI
    library exists on these hosts, so independent copies are the way it
    uses every core.  Returns a dict: aggregate particle-steps/s (all
    copies' work over the slowest copy's main loop, the reference's own
    timer core/main.c:479-480), the slowest copy's seconds, the marker
    count, the number of copies and the median copy's own rate; or None
    without the reference binaries."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_port
    from refrun import RefRun, have_reference
    exe = os.path.join(ROOT, "oracle", "_ref", "core_fast.out")
    if not have_reference() or not os.path.exists(exe):
        return None
    m = np.concatenate([oracle_port.place(h=w["h"], **s) for s in w["species"]])
    if procs is None:
        procs = host_cores()
        try:
            import psutil
            per = 3.0 * (m.nbytes + 12 * 8 * int(np.prod([v + 5 for v in w["n"]])))
            procs = max(1, min(procs, int(0.7 * psutil.virtual_memory().available / per)))
        except ImportError:
            pass
    base = RefRun(tempfile.mkdtemp(prefix="mandor_bench_ref_"))
    runs = []
    try:
        L_um = [w["n"][a] * w["h"][a] for a in range(3)]
        base.setup(w["n"], L_um, -0.5, w["bc"], w["bc"])
        base.set_state(m)
        big = ("plasma_000000_000.bin", "sys_E_000000(000).bin", "sys_H_000000(000).bin")
        for q in range(procs):
            rr = RefRun(tempfile.mkdtemp(prefix="mandor_bench_ref%d_" % q))
            for f in os.listdir(base.path("binData")):
                src, dst = base.path("binData", f), rr.path("binData", f)
                if f in big:
                    os.link(src, dst)          # read only by core.out
                else:
                    with open(src, "rb") as a, open(dst, "wb") as b:
                        b.write(a.read())
            with open(rr.path("run_mandor.cfg"), "w") as fp:
                fp.write("@ %d\ttotal steps\n@ %d\tcheckpoint period\n@ -1\ttecplot\n@ 0\tcontinue\n"
                         "@ %d\tstop-flag period\n@ -100\tspectral dumps\n" % (steps, 10 ** 8, 10 ** 8))
            runs.append(rr)
        procs_ = [subprocess.Popen([exe], cwd=rr.dir, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
                  for rr in runs]
        secs = []
        for p in procs_:
            out, _ = p.communicate(timeout=1800)
            text = out.decode(errors="replace")
            if p.returncode != 0:
                raise RuntimeError("reference core_fast.out failed:\n" + text[-2000:])
            secs.append(float(re.search(r"main loop have taken ([0-9.eE+-]+) sec", text).group(1)))
    finally:
        base.cleanup()
        for rr in runs:
            rr.cleanup()
    rate = procs * len(m) * steps / max(secs)
    desc = ("reference core.out (-O3, single-rank MPI shim) as %d independent processes at once, one per "
            "host core, each on the laser-foil grid and markers for %d steps from t=0; aggregate "
            "particle-steps over the slowest process's main-loop time; laser source omitted (the "
            "reference has no analytic sin^2 source; the source plane is O(n^2) work)" % (procs, steps))
    return {"value": rate, "seconds": max(secs), "markers": len(m), "procs": procs,
            "per_process": len(m) * steps / statistics.median(secs), "sample": desc}


# ---------------------------------------------------------------------------
def dist_setup(backend="nccl"):
    """One process per GPU (replicas: each rank runs its own copy of the
    workload, no data-path collective); the process group only carries the
    timing reductions.  backend "gloo" runs the same logic on CPU."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def _reduce(v, world, op):
    import torch
    import torch.distributed as dist
    on_gpu = dist.get_backend() == "nccl"
    t = torch.tensor([float(v)], device="cuda" if on_gpu else "cpu", dtype=torch.float64)
    dist.all_reduce(t, op=op)
    return float(t.item())


def dist_max(v, world):
    if world == 1:
        return v
    import torch.distributed as dist
    return _reduce(v, world, dist.ReduceOp.MAX)


def replica_value(units, ms, world):
    """Whole-job throughput of replicas: the units all ranks processed over
    the slowest rank's time (ms)."""
    return dist_sum(units, world) / (dist_max(ms, world) / 1e3)


def dist_sum(v, world):
    if world == 1:
        return v
    import torch.distributed as dist
    return _reduce(v, world, dist.ReduceOp.SUM)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference_arm(args, w, world, rank):
    if rank != 0:
        return
    steps = args.ref_steps
    res = reference_sample(w, steps)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference binaries not built (make -C oracle ref REF=<reference root>)"}))
        return
    rate = res["value"]
    line = {"metric": "particle-steps/s", "value": rate, "unit": "particle-steps/s",
            "impl": "reference", "n_gpus": args.gpus, "steps": steps, "warmup": 0,
            "requested": {"steps": args.steps, "warmup": args.warmup},
            "ms_per_step": 1e3 * res["seconds"] / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": w["name"], "markers": res["markers"], "grid": list(w["n"]),
                       "bc": "mur x6", "courant": 0.5, "laser": "omitted (no sin^2 source in the reference)",
                       "copies": res["procs"]},
            "cpu_baseline": {"value": rate, "unit": "particle-steps/s", "cores": res["procs"],
                             "kind": "reference", "sample": res["sample"],
                             "per_process": res["per_process"]},
            "e2e": {"value": rate, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Many solves on one GPU: a batch of 256 runs, and a served request stream.
# ---------------------------------------------------------------------------
def batch_specs(count=256, steps=300, seed=1802):
    """256 independent runs drawn from one seed: half periodic thermal
    plasmas, half laser-foil runs; sides U{16..96} cells per axis, 4-32
    markers per cell, foil densities U(5, 50) n_cr, a0 U(0.5, 5), foils
    0.25 wavelength thick; precision form, `steps` steps each."""
    from mandor3_b200 import scan, FP32_OFFSET
    rng = np.random.default_rng(seed)
    out = []
    for q in range(count):
        n = tuple(int(v) for v in rng.integers(16, 97, size=3))
        ppc = int(rng.integers(4, 33))
        if q % 2 == 0:
            out.append(scan.PeriodicSolve(n, ppc, 0.01 + 0.04 * rng.random(), steps,
                                          precision=FP32_OFFSET, seed=(1802, 9373 + q)))
        else:
            n = (max(n[0], 24),) + n[1:]
            out.append(scan.FoilSolve(n, max(1, ppc // 2), float(rng.uniform(0.5, 5.0)), 0.25,
                                      float(rng.uniform(5.0, 50.0)), steps, precision=FP32_OFFSET,
                                      seed=(1802, 9373 + q)))
    return out


def serve_specs(count=24, seed=9373, step_scale=1.0):
    """Laser-foil scan solves of mixed size: grids (64, 32, 32) x U{1..4},
    4-16 markers per cell, a0 U(1, 10), foil thickness U(0.1, 2) wavelengths,
    density U(10, 100) n_cr, U{1000..3000} steps (times step_scale)."""
    from mandor3_b200 import scan, FP32_OFFSET
    rng = np.random.default_rng(seed)
    out = []
    for q in range(count):
        k = int(rng.integers(1, 5))
        out.append(scan.FoilSolve((64 * k, 32 * k, 32 * k), int(rng.integers(4, 17)),
                                  float(rng.uniform(1, 10)), float(rng.uniform(0.1, 2.0)),
                                  float(rng.uniform(10, 100)),
                                  max(10, int(rng.integers(1000, 3001) * step_scale)),
                                  precision=FP32_OFFSET, seed=(1802, 9373 + q)))
    return out


def batch_bench(args):
    """Throughput of 256 runs stepped by one graph launch per step, against
    the same runs stepped one at a time (both device-resident)."""
    import torch
    import mandor3_b200 as mg
    from mandor3_b200 import scan
    specs = batch_specs(steps=args.steps or 300)
    tuner = scan.Tuner(steps=6, sorts=(8, 16))
    t = time.perf_counter()
    choice = [tuner.choose(s) for s in specs]
    tune_s = time.perf_counter() - t
    runs = [s.build(0, tile=c[0], sort_every=c[1], warps=c[2]) for s, c in zip(specs, choice)]
    markers = sum(r.marker_count() for r in runs)
    b = mg.Batch(runs)
    b.step(args.warmup)
    with Clocks(0) as clocks:
        torch.cuda.synchronize()
        t = time.perf_counter()
        b.step(specs[0].steps)
        torch.cuda.synchronize()
        batch_s = time.perf_counter() - t
    b.close()
    for r in runs:
        r.close()
    # Same runs, one at a time.
    alone_s = 0.0
    for s, c in zip(specs, choice):
        r = s.build(0, tile=c[0], sort_every=c[1], warps=c[2])
        r.step(args.warmup)
        torch.cuda.synchronize()
        t = time.perf_counter()
        r.step(s.steps)
        alone_s += time.perf_counter() - t
        r.close()
    steps = specs[0].steps
    value = markers * steps / batch_s
    print(json.dumps({
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": 1,
        "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * batch_s / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "batch_256_runs", "runs": len(specs), "markers": markers,
                   "sides": "U{16..96} per axis", "ppc": "4-32", "kinds": "half periodic thermal, half laser foil",
                   "precision": "int cell + FP32 offset", "tuned": sorted(set(map(str, tuner.table.values()))),
                   "tuning_seconds": tune_s},
        "clocks": clocks.summary(),
        "alone": {"value": markers * steps / alone_s, "seconds": alone_s},
        "batch_over_alone": alone_s / batch_s,
    }))


def serve_measure(requests=24, step_scale=1.0, chaos=True):
    """A Poisson stream (200 requests/s) of laser-foil scan solves served
    with continuous batching in the precision form, against the same solves
    run one at a time in the plain FP64 form (queued in arrival order).
    Accuracy: per solve, the served total-energy history against the FP64
    solve's, next to its conditioning floor -- the FP64 solve against
    itself with the laser amplitude moved by 2^-24 (single-precision
    rounding of one input), which bounds how closely any form carrying
    single-precision state can follow FP64 on these strongly driven
    solves."""
    import torch
    from mandor3_b200 import scan, FP64
    import dataclasses
    specs = serve_specs(count=requests, step_scale=step_scale)
    stream = scan.poisson_stream(specs, 200.0)
    tuner = scan.Tuner(steps=6, sorts=(8, 16))
    t = time.perf_counter()
    for s in specs:
        tuner.choose(s)
    tune_s = time.perf_counter() - t
    srv = scan.Server(chunk=100, tuner=tuner)
    with Clocks(0) as clocks:
        torch.cuda.synchronize()
        t = time.perf_counter()
        res = srv.serve(stream)
        served_s = time.perf_counter() - t
    tot = lambda a: a[:, 1] + a[:, 2] + a[:, 3:6].sum(1)
    done, lat, fp64_s, err, floor = 0.0, [], 0.0, [], []
    for (arr, s), r in zip(stream, res):
        plain = dataclasses.replace(s, precision=FP64)
        rows, count, sec = scan.run_alone(plain)
        fp64_s += sec
        done = max(done, arr) + sec
        lat.append(done - arr)
        scale = np.max(np.abs(tot(rows)))
        err.append(float(np.max(np.abs(tot(r.rows) - tot(rows))) / scale))
        if chaos:
            nudged = dataclasses.replace(plain, a0=plain.a0 * (1 + 2.0 ** -24))
            rows2, _, _ = scan.run_alone(nudged)
            floor.append(float(np.max(np.abs(tot(rows2) - tot(rows))) / scale))
    psteps = sum(s.markers() * s.steps for s in specs)
    out = {
        "workload": "serve_laser_foil_scan", "requests": len(specs), "rate_per_s": 200.0,
        "grids": "(64,32,32) x U{1..4}", "ppc": "4-16", "a0": "U(1,10)", "thickness": "U(0.1,2) lambda",
        "density": "U(10,100) n_cr", "steps": "U{1000..3000} x %g" % step_scale,
        "precision": "int cell + FP32 offset (served) vs plain FP64 (one at a time)",
        "admission": "device footprint", "budget_bytes": srv.budget, "peak_admitted_bytes": srv.peak_used,
        "server_host_seconds": srv.stats, "tuning_seconds": tune_s,
        "clocks": clocks.summary(),
        "solves_per_s": len(specs) / served_s,
        "served": {"seconds": served_s, "particle_steps_per_s": psteps / served_s,
                   "latency_p50_s": scan.percentile([r.latency for r in res], 50),
                   "latency_p99_s": scan.percentile([r.latency for r in res], 99)},
        "plain_fp64_one_at_a_time": {"seconds": fp64_s, "solves_per_s": len(specs) / fp64_s,
                                     "latency_p50_s": scan.percentile(lat, 50),
                                     "latency_p99_s": scan.percentile(lat, 99)},
        "throughput_over_plain": fp64_s / served_s,
        "total_energy_error_vs_fp64": {"max": max(err), "median": scan.percentile(err, 50),
                                       "per_solve": err},
    }
    if chaos:
        ratio = [e / f for e, f in zip(err, floor)]
        out["conditioning_floor"] = {"max": max(floor), "median": scan.percentile(floor, 50), "per_solve": floor,
                                     "error_over_floor_max": max(ratio),
                                     "note": "FP64 solve against itself with a0 x (1 + 2^-24): max over the "
                                             "history of |W_total difference| / max |W_total|"}
    return out


def serve_bench(args):
    m = serve_measure(args.requests, args.step_scale)
    steps = None
    print(json.dumps({
        "metric": "scan solves/s", "value": m["solves_per_s"], "unit": "solves/s", "n_gpus": 1,
        "steps": steps, "warmup": 0, "ms_per_step": None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {k: m[k] for k in ("workload", "requests", "rate_per_s", "grids", "ppc",
                                                          "a0", "thickness", "density", "steps", "admission",
                                                          "budget_bytes", "peak_admitted_bytes")},
        "clocks": m["clocks"], "serve": m}))


def precision_form_measure(device, warmup=3):
    """BASELINE configuration 3 at full size (256^3 periodic two-stream
    plasma, 2 x 32 markers per cell = 1.07e9 markers) in the precision form:
    W warm-up steps, then one sort interval (24 steps, one sort inside) timed
    with CUDA events on the run's stream; roofline of the tiled push (60 B
    per marker) and of the whole step (60 B per marker + 72 B per cell);
    then both forms from t = 0 over the same 24 steps for the energy-history
    error against FP64."""
    import torch
    w = weibel()
    t = time.perf_counter()
    r = make_run(w, device)
    build_s = time.perf_counter() - t
    r.step(warmup)
    steps = w["sort_every"]
    n0 = r.marker_count()
    stream = torch.cuda.ExternalStream(r.stream(), device=device)
    r.profile(True)
    torch.cuda.synchronize()
    with Clocks(device) as clocks:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r.step_async(steps)
        e1.record(stream)
        r.synchronize()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    push_ms, step_ms = r.last_timing()
    launches = r.kernels_per_step()
    r.close()
    peak, peak_kind = hbm_peak()
    cells = w["n"][0] * w["n"][1] * w["n"][2]
    push_bytes = w["bytes_per_marker"] * n0
    step_bytes = push_bytes + 72.0 * cells
    achieved = push_bytes / (push_ms / 1e3) / 1e9
    step_achieved = step_bytes / (ms / steps / 1e3) / 1e9
    out = {"workload": w["name"], "markers": n0, "grid": list(w["n"]), "dtype": "f32",
           "precision": "int cell + FP32 offset, FP32 u/E/H/J, FP64 reductions",
           "steps": steps, "warmup": warmup, "sort_every": w["sort_every"], "sorts_in_window": 1,
           "ms_per_step": ms / steps, "value": n0 * steps / (ms / 1e3), "unit": "particle-steps/s",
           "build_seconds": build_s, "clocks": clocks.summary(), "gpu_launches_per_step": launches,
           "roofline": {"bound": "hbm", "kernel": "k_push32_tiles", "achieved": achieved, "peak": peak,
                        "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                        "traffic": ncu_traffic(w, n0), "push_ms": push_ms,
                        "algorithmic_bytes_per_launch": push_bytes},
           "step_roofline": {"achieved": step_achieved, "peak": peak, "unit": "GB/s", "frac": step_achieved / peak,
                             "algorithmic_bytes_per_step": step_bytes,
                             "note": "60 B per marker + 72 B per cell over the whole step, its sort included"}}
    out["fp64_comparison"] = compare_fp64(w, device, steps)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="laser_foil")
    ap.add_argument("--ref-steps", type=int, default=12)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the precision-form (configuration 3) and serving sub-objects of the default line")
    ap.add_argument("--requests", type=int, default=24, help="serve workload: solves in the stream")
    ap.add_argument("--step-scale", type=float, default=1.0, help="serve workload: scale of the solves' steps")
    ap.add_argument("--compare-fp64", type=int, default=0, metavar="K",
                    help="precision-form workloads: also run K steps in both forms from t = 0 and report the "
                         "energy-history error of each quantity against the FP64 form")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("at least 3 warm-up steps")
    if args.workload in ("yee", "yee_fp32"):
        yee_bench(args)
        return
    if args.workload in ("batch", "serve"):
        import torch
        torch.cuda.set_device(0)
        (batch_bench if args.workload == "batch" else serve_bench)(args)
        return

    w = workload(args.workload)
    if args.steps is None:
        args.steps = w["total_steps"] - args.warmup
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference_arm(args, w, world, rank)
        barrier(world)
        return

    import mandor3_b200 as mg
    import torch

    device = local
    torch.cuda.set_device(device)
    r = make_run(w, device)
    r.step(args.warmup)
    launches_per_step = r.kernels_per_step()
    n_before = r.marker_count()
    stream = torch.cuda.ExternalStream(r.stream(), device=device)

    # Timed region: K graph-replayed steps, events on the run's stream.
    r.profile(True)
    barrier(world)
    torch.cuda.synchronize()
    with Clocks(device) as clocks:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r.step_async(args.steps)
        e1.record(stream)
        r.synchronize()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    push_ms, step_ms = r.last_timing()
    n_after = r.marker_count()
    r.close()
    n_avg = 0.5 * (n_before + n_after)
    ms_max = dist_max(ms, world)
    value = replica_value(n_avg * args.steps, ms, world)

    # End to end through the C ABI from pinned host buffers.
    e2e = None
    if not args.no_e2e:
        e2e = end_to_end(w, device, args.steps, args.warmup, world)

    peak, peak_kind = hbm_peak()
    algo_bytes = w["bytes_per_marker"] * n_avg
    achieved = algo_bytes / (push_ms / 1e3) / 1e9 if push_ms > 0 else None
    roofline = {"bound": "hbm", "kernel": "k_push64" if w["precision"] == 0 else "k_push32_tiles",
                "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s",
                "frac": achieved / peak if achieved else None,
                "traffic": ncu_traffic(w, n_avg), "push_ms": push_ms, "step_ms": step_ms,
                "algorithmic_bytes_per_launch": algo_bytes}

    compare = None
    if args.compare_fp64 > 0 and w["precision"] != 0:
        compare = compare_fp64(w, device, args.compare_fp64)

    # The other north-star forms, on rank 0 of a single-GPU run: the
    # precision form at configuration 3's full size and the served scan.
    extras = {}
    if world == 1 and w["precision"] == 0 and not args.no_extras:
        for key, fn in (("precision_form", lambda: precision_form_measure(device)),
                        ("serve", lambda: serve_measure(args.requests, args.step_scale))):
            t = time.perf_counter()
            try:
                extras[key] = fn()
            except Exception as e:                      # report, keep the headline line
                extras[key] = {"error": "%s: %s" % (type(e).__name__, e)}
            extras[key]["wall_seconds"] = time.perf_counter() - t
            torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        res = reference_sample(w, args.ref_steps)
        if res:
            cpu = {"value": res["value"], "unit": "particle-steps/s", "cores": res["procs"],
                   "kind": "reference", "sample": res["sample"], "per_process": res["per_process"]}
    barrier(world)
    if rank != 0:
        return
    line = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": w["dtype"], "data": "synthetic",
            "config": config_of(w, world),
            "clocks": clocks.summary(), "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps, "roofline": roofline,
            "cpu_baseline": cpu}
    if compare:
        line["fp64_comparison"] = compare
    line.update(extras)
    print(json.dumps(line), flush=True)


def yee_bench(args):
    """Field-only Yee solver: a 256^3 box with Mur walls on all faces and an
    initial Gaussian E pulse, no markers; cell-updates/s and the fraction of
    the measured HBM bandwidth for 96 B (FP64) / 48 B (FP32) per cell update
    (read E, H; write E, H)."""
    import torch
    import mandor3_b200 as mg
    fp32 = args.workload == "yee_fp32"
    n = (256, 256, 256)
    h = (0.05, 0.05, 0.05)
    tau = 0.5 / math.sqrt(sum(1.0 / v ** 2 for v in h))
    r = mg.Run(n, h, tau, (2, 2, 2), (2, 2, 2), precision=mg.FP32_OFFSET if fp32 else mg.FP64)
    x = np.arange(n[0] + 1)[:, None, None, None]
    E = np.zeros(r.field_shape())
    E[..., 1] = np.exp(-((x - 128) * h[0] / 1.0) ** 2)[..., 0]
    r.set_fields(E, np.zeros(r.field_shape()))
    r.init()
    steps = args.steps or 200
    r.step(max(args.warmup, 3))
    stream = torch.cuda.ExternalStream(r.stream(), device=0)
    torch.cuda.synchronize()
    with Clocks(0) as clocks:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r.step_async(steps)
        e1.record(stream)
        r.synchronize()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    cells = n[0] * n[1] * n[2]
    bpc = 48.0 if fp32 else 96.0
    peak, peak_kind = hbm_peak()
    achieved = cells * bpc / (ms / 1e3) / 1e9
    traffic = None
    try:
        text = open(os.path.join(ROOT, "profiles", "launches_yee.md")).read()
        m = re.search(r"traffic_bytes_per_launch_%s:\s*([0-9.eE+]+)" % ("fp32" if fp32 else "fp64"), text)
        traffic = float(m.group(1)) if m else None
    except OSError:
        pass
    r.close()
    print(json.dumps({
        "metric": "Yee cell-updates/s", "value": cells / (ms / 1e3), "unit": "cell-updates/s", "n_gpus": 1,
        "steps": steps, "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if fp32 else "f64", "data": "synthetic",
        "config": {"workload": "yee_%s_256cubed" % ("fp32" if fp32 else "fp64"), "grid": list(n),
                   "bc": "mur x6", "markers": 0, "l2": "inputs larger than L2 (fields %.1f GB)"
                   % (12 * (n[0] + 5) ** 3 * (4 if fp32 else 8) / 1e9)},
        "clocks": clocks.summary(),
        "roofline": {"bound": "hbm", "kernel": "whole step (one pass k_yee_tile, E shell, walls)",
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "traffic_of": None if traffic is None else "k_yee_tile, one launch (ncu)",
                     "algorithmic_bytes_per_step": cells * bpc}}), flush=True)


def compare_fp64(w, device, steps):
    """The workload's energy history over `steps` steps from t = 0 in the
    precision form and in the plain FP64 form (same markers: the same
    placer draws), one run after the other; per quantity, the largest
    difference over the history relative to the FP64 quantity's largest
    magnitude."""
    hist = {}
    for prec in (w["precision"], 0):
        r = make_run(dict(w, precision=prec), device)
        hist[prec] = r.step(steps)
        r.close()
    a, b = hist[w["precision"]], hist[0]
    def err(qa, qb):
        return float(np.max(np.abs(qa - qb)) / max(np.max(np.abs(qb)), 1e-300))
    tot = lambda h: h[:, 1] + h[:, 2] + h[:, 3:6].sum(1)
    return {"steps": steps, "W_E": err(a[:, 1], b[:, 1]), "W_M": err(a[:, 2], b[:, 2]),
            "W_T": err(a[:, 3:6].sum(1), b[:, 3:6].sum(1)), "W_total": err(tot(a), tot(b)),
            "note": "max over the history of |precision form - FP64| / max |FP64| per quantity"}


def config_of(w, world):
    if w["precision"] == 0:
        return {"workload": w["name"], "markers": w["markers"], "grid": list(w["n"]),
                "bc": "mur x6", "courant": 0.5, "laser": "a0=3 w0=3 sin^2 10 cycles",
                "foil": "30 n_cr, 10 cells, e- and p+ at 16 ppc",
                "parallelism": "replicas x%d" % world,
                "l2": "inputs larger than L2 (fields 0.34 GB + markers 0.27 GB per step)"}
    return {"workload": w["name"], "markers": w["markers"], "grid": list(w["n"]), "bc": "periodic",
            "courant": 0.5, "beams": "u_x = +-0.2c, 32 ppc each, u_th 0.01",
            "precision": "int cell + FP32 offset, FP32 u/E/H/J, FP64 reductions",
            "sort_every": w.get("sort_every", 16),
            "parallelism": "replicas x%d" % world,
            "l2": "inputs larger than L2 (43 GB of markers per step)"}


def end_to_end(w, device, steps, warmup, world):
    """Host buffers in, host buffers out, through the reference-facing ABI."""
    import mandor3_b200 as mg
    import torch
    # The initial state as host data (what core.out would load from binData).
    r0 = make_run(w, device)
    markers = r0.markers()
    r0.close()
    shape = (w["n"][0] + 1, w["n"][1] + 1, w["n"][2] + 1, 3)
    pin = lambda nbytes: torch.empty(nbytes, dtype=torch.uint8, pin_memory=True).numpy()
    hm = pin(markers.nbytes).view(mg.MARKER_DTYPE)
    hm[:] = markers
    hE = pin(8 * int(np.prod(shape))).view("<f8").reshape(shape)
    hH = pin(8 * int(np.prod(shape))).view("<f8").reshape(shape)
    hE[:] = 0
    hH[:] = 0
    rows = pin(8 * 6 * steps).view("<f8").reshape(steps, 6)
    out_m = pin(markers.nbytes).view(mg.MARKER_DTYPE)
    r = mg.Run(w["n"], w["h"], w["tau"], w["bc"], w["bc"], device=device, capacity=len(markers),
               precision=w["precision"], sort_every=w.get("sort_every", 0))
    if w["laser"]:
        r.set_laser(**w["laser"])
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    marks = [t0]
    r.set_fields(hE, hH)
    r.set_markers(hm)
    r.init()
    marks.append(time.perf_counter())
    lib = mg.load()
    rc = lib.mg_run_step(r.ptr, steps, rows.ctypes.data)
    if rc:
        raise mg.MandorError(rc, lib.mg_last_error().decode())
    marks.append(time.perf_counter())
    import ctypes
    got = ctypes.c_longlong()
    rc = lib.mg_run_get_markers(r.ptr, out_m.ctypes.data, len(out_m), ctypes.byref(got))
    if rc:
        raise mg.MandorError(rc, lib.mg_last_error().decode())
    rc = lib.mg_run_get_fields(r.ptr, hE.ctypes.data, hH.ctypes.data)
    if rc:
        raise mg.MandorError(rc, lib.mg_last_error().decode())
    sec = time.perf_counter() - t0
    marks.append(t0 + sec)
    phases = {k: round(b - a, 4) for k, a, b in zip(("upload_init_s", "steps_s", "download_s"), marks, marks[1:])}
    r.close()
    sec = dist_max(sec, world)
    ps = dist_sum(0.5 * (len(markers) + got.value) * steps, world)
    h2d = markers.nbytes + hE.nbytes + hH.nbytes
    d2h = got.value * 64 + hE.nbytes + hH.nbytes + rows.nbytes
    return {"value": ps / sec, "unit": "particle-steps/s",
            "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h / steps,
            "seconds": sec, "phases": phases,
            "note": "wall clock, max over ranks; upload + %d steps + download" % steps}


if __name__ == "__main__":
    main()
