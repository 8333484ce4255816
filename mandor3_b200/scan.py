"""Parameter scans on one GPU: solve specifications, an autotuner for the
precision form's tile shape and sort interval, and a continuous-batching
server.

None of this has a counterpart in the reference, which runs one simulation
per `core.out` process (core/main.c:195-480); a scan there is a sequence of
runs.  Here many solves share the device:

* `Tuner` picks tile shape, block size and sort interval per class of solve;
* `Batch` (C ABI `mg_batch_*`) steps a fixed set of runs with one graph
  launch per step;
* `Server` admits solves from a request stream while memory allows (each
  run's footprint from `mg_estimate_bytes`), keeps their state on the device
  and steps every admitted run in rounds of batched graph launches, so the
  work of solves that arrived at different times overlaps on the GPU;
  finished solves leave and free their memory for queued ones.

A solve's result is its energy history (rows {t, W_E, W_M, W_Tx, W_Ty, W_Tz},
the arguments of wDensity_addPoint, core/diag_WDensity.c:136-147) and its
final marker count.
"""
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import (FP32_OFFSET, FP64, BC_OPEN, BC_PERIODIC, Batch, MandorError, Run, estimate_bytes,
               load)

ERR_ADMISSION = -8               # MG_ERR_ADMISSION (include/mandor_b200.h)

N_CR = 4 * math.pi ** 2          # critical density in code units


@dataclass
class FoilSolve:
    """Laser on a foil of electrons and protons: Mur walls on all sides, an
    Ey-polarised sin^2 Gaussian laser injected at x-plane 5 and focused on the
    foil front, foil `thickness` wavelengths thick near x = 0.6 L, `density`
    n_cr, `ppc` markers per cell per species, cold, h = 0.05 wavelengths,
    Courant 0.5."""
    n: tuple
    ppc: int
    a0: float
    thickness: float
    density: float
    steps: int
    precision: int = FP32_OFFSET
    seed: tuple = (1802, 9373)
    h: float = 0.05

    def geometry(self):
        """Grid and foil box [lo, hi): behind the laser plane 5 and at least
        two cells from the far wall (the foil is thinned on short grids)."""
        n = tuple(int(v) for v in self.n)
        cells = min(max(1, int(round(self.thickness / self.h))), n[0] - 9)
        x0 = max(6, min(int(0.6 * n[0]), n[0] - 2 - cells))
        m = [max(2, n[1] // 8), max(2, n[2] // 8)]
        lo, hi = (x0, m[0], m[1]), (x0 + cells, n[1] - m[0], n[2] - m[1])
        return n, lo, hi

    def markers(self):
        _, lo, hi = self.geometry()
        return 2 * self.ppc * (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2])

    def tau(self):
        return 0.5 / math.sqrt(3 / self.h ** 2)

    def params(self):
        n = tuple(int(v) for v in self.n)
        return dict(n=n, h=(self.h,) * 3, tau=self.tau(), bc_min=(BC_OPEN,) * 3,
                    bc_max=(BC_OPEN,) * 3)

    def build(self, device=0, tile=(0, 0, 0), sort_every=0, warps=0):
        n, lo, hi = self.geometry()
        p = self.params()
        r = Run(p["n"], p["h"], p["tau"], p["bc_min"], p["bc_max"], precision=self.precision,
                device=device, capacity=self.markers(), sort_every=sort_every, tile=tile,
                tile_warps=warps)
        # Fields start at zero (mg_run_create clears them).
        waist = 0.25 * min(n[1], n[2]) * self.h
        r.set_laser(a0=self.a0, waist=waist, x_focus=lo[0] * self.h, duration=10.0, t_start=0.0,
                    phase=0.0, plane=5, margin=3)
        each = self.markers() // 2
        rho = self.density * N_CR / self.ppc
        r.place_uniform(lo, hi, self.ppc, -rho, -1.0, seed=self.seed, id0=1)
        r.place_uniform(lo, hi, self.ppc, rho, 1.0 / 1836, seed=self.seed, skip=7 * each,
                        id0=1 + each)
        r.init()
        return r


@dataclass
class PeriodicSolve:
    """Periodic thermal electron plasma at `density` n_cr over an immobile
    neutralising background (not modelled: the system is not neutral, as in
    the reference's electron-only decks), h = 0.05 c/omega_p, Courant 0.5."""
    n: tuple
    ppc: int
    uth: float
    steps: int
    density: float = 1.0
    precision: int = FP32_OFFSET
    seed: tuple = (1802, 9373)

    def markers(self):
        return self.ppc * int(np.prod(self.n))

    def params(self):
        hh = 0.05 / (2 * math.pi)
        n = tuple(int(v) for v in self.n)
        return dict(n=n, h=(hh,) * 3, tau=0.5 / math.sqrt(3 / hh ** 2), bc_min=(BC_PERIODIC,) * 3,
                    bc_max=(BC_PERIODIC,) * 3)

    def build(self, device=0, tile=(0, 0, 0), sort_every=0, warps=0):
        p = self.params()
        r = Run(p["n"], p["h"], p["tau"], p["bc_min"], p["bc_max"], precision=self.precision,
                device=device, capacity=self.markers(), sort_every=sort_every, tile=tile,
                tile_warps=warps)
        # Fields start at zero (mg_run_create clears them).
        r.place_uniform((0, 0, 0), p["n"], self.ppc, -self.density * N_CR / self.ppc, -1.0,
                        uth=(self.uth,) * 3, seed=self.seed)
        r.init()
        return r


def footprint(spec):
    """Device bytes a solve holds while admitted (mg_estimate_bytes)."""
    p = spec.params()
    return estimate_bytes(p["n"], p["h"], p["tau"], p["bc_min"], p["bc_max"], spec.markers(),
                          spec.precision)


class Tuner:
    """Picks the tile shape, the block size of the tiled push (warps per
    block, i.e. markers of a tile pushed at once / 32) and the sort interval
    of precision-form solves by timing each candidate for a few steps on a
    solve of the same class (grid-size and markers-per-cell bucket) and
    keeping the fastest, one knob after the other; FP64 solves have nothing
    to tune."""

    TILES = ((8, 8, 4), (4, 4, 4), (8, 8, 8))
    WARPS = (8, 4, 16)
    SORTS = (4, 8, 16)

    def __init__(self, device=0, steps=12, tiles=TILES, sorts=SORTS, warps=WARPS):
        self.device = device
        self.steps = steps
        self.tiles = tiles
        self.sorts = sorts
        self.warps = warps
        self.table = {}

    @staticmethod
    def key(spec):
        cells = int(np.prod(spec.n))
        return (type(spec).__name__, spec.precision, int(math.log2(max(cells, 1))) // 2,
                int(math.log2(max(spec.markers() / max(cells, 1), 1))))

    def _time(self, spec, steps, which, **kw):
        r = spec.build(self.device, **kw)
        r.step(2)
        r.profile(True)
        r.step(steps)
        push, step = r.last_timing()
        r.close()
        return push if which == "push" else step

    def choose(self, spec):
        """(tile, sort_every, warps) for this solve."""
        if spec.precision == FP64:
            return (0, 0, 0), 0, 0
        k = self.key(spec)
        if k not in self.table:
            every0 = min(self.sorts)
            tile = min(self.tiles, key=lambda t: self._time(spec, self.steps, "push", tile=t,
                                                            sort_every=every0, warps=self.warps[0]))
            warps = min(self.warps, key=lambda w: self._time(spec, self.steps, "push", tile=tile,
                                                             sort_every=every0, warps=w))
            every = min(self.sorts, key=lambda e: self._time(spec, max(self.steps, 2 * e), "step",
                                                             tile=tile, sort_every=e, warps=warps))
            self.table[k] = (tile, every, warps)
        return self.table[k]


@dataclass
class Result:
    index: int
    arrival: float          # seconds after the start of the stream
    admitted: float
    finished: float
    rows: np.ndarray
    markers: int
    latency: float = field(init=False)

    def __post_init__(self):
        self.latency = self.finished - self.arrival


class Server:
    """Continuous batching of solves on one GPU.

    `serve(stream)` takes (arrival seconds, spec) pairs and returns the
    results in request order.  Between rounds it admits queued solves in
    arrival order while their footprints fit `budget` bytes and retires the
    finished ones.  A round steps every admitted solve by the same number of
    steps (at most `chunk`, and no more than the closest solve to its end
    still needs) through one `Batch`: one CUDA graph launch per step for all
    admitted solves, rebuilt whenever the set of solves changes.
    """

    def __init__(self, device=0, budget=None, chunk=100, tuner=None):
        import torch
        self.device = device
        self.chunk = chunk
        self.tuner = tuner
        if budget is None:
            free, _ = torch.cuda.mem_get_info(device)
            budget = int(0.85 * free)
        self.budget = budget
        self.peak_used = 0
        # Host seconds spent admitting (building runs), rebuilding batches and
        # stepping rounds.
        self.stats = dict(admit_s=0.0, batch_s=0.0, step_s=0.0, retire_s=0.0, idle_s=0.0, rounds=0)

    def serve(self, stream):
        pending = sorted(((float(t), i, s) for i, (t, s) in enumerate(stream)), key=lambda x: (x[0], x[1]))
        queue, active, results = [], [], {}
        batch = None
        used = 0
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        while pending or queue or active:
            while pending and pending[0][0] <= now():
                queue.append(pending.pop(0))
            # Admission in arrival order while the footprints fit.
            changed = False
            while queue:
                arrival, i, spec = queue[0]
                need = footprint(spec)
                if need > self.budget:
                    raise MandorError(ERR_ADMISSION, "solve %d needs %d bytes of device memory, more than "
                                      "the whole admission budget of %d bytes" % (i, need, self.budget))
                if used + need > self.budget:
                    break
                queue.pop(0)
                ta = time.perf_counter()
                tile, every, warps = self.tuner.choose(spec) if self.tuner else ((0, 0, 0), 0, 0)
                run = spec.build(self.device, tile=tile, sort_every=every, warps=warps)
                self.stats["admit_s"] += time.perf_counter() - ta
                active.append(dict(i=i, spec=spec, run=run, rows=[], done=0, need=need,
                                   arrival=arrival, admitted=now()))
                used += need
                self.peak_used = max(self.peak_used, used)
                changed = True
            if not active:
                if pending:
                    ti = time.perf_counter()
                    time.sleep(max(0.0, min(0.05, pending[0][0] - now())))
                    self.stats["idle_s"] += time.perf_counter() - ti
                continue
            if changed or batch is None:
                tb = time.perf_counter()
                if batch is not None:
                    batch.close()
                batch = Batch([a["run"] for a in active])
                self.stats["batch_s"] += time.perf_counter() - tb
            k = min([self.chunk] + [a["spec"].steps - a["done"] for a in active])
            ts = time.perf_counter()
            rows = batch.step(k)
            self.stats["step_s"] += time.perf_counter() - ts
            self.stats["rounds"] += 1
            tr = time.perf_counter()
            still = []
            for a, rw in zip(active, rows):
                a["rows"].append(rw)
                a["done"] += k
                if a["done"] < a["spec"].steps:
                    still.append(a)
                    continue
                results[a["i"]] = Result(a["i"], a["arrival"], a["admitted"], now(),
                                         np.concatenate(a["rows"]), a["run"].marker_count())
                used -= a["need"]
            if len(still) != len(active):
                batch.close()
                batch = None
                for a in active:
                    if a["done"] >= a["spec"].steps:
                        a["run"].close()
            active = still
            self.stats["retire_s"] += time.perf_counter() - tr
        if batch is not None:
            batch.close()
        return [results[i] for i in range(len(stream))]


def run_alone(spec, device=0, tile=(0, 0, 0), sort_every=0, warps=0):
    """One solve on its own: (energy rows, final marker count, seconds)."""
    import torch
    torch.cuda.synchronize(device)
    t = time.perf_counter()
    r = spec.build(device, tile=tile, sort_every=sort_every, warps=warps)
    rows = r.step(spec.steps)
    count = r.marker_count()
    r.close()
    return rows, count, time.perf_counter() - t


def poisson_stream(specs, rate, seed=1802):
    """Arrival times of a Poisson stream with `rate` requests per second."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=len(specs)))
    return list(zip(t - t[0], specs))


def percentile(values, q):
    return float(np.percentile(np.asarray(values, dtype=float), q))
