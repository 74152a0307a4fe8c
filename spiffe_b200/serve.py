"""Many independent spiffe problems on one GPU: a batched parameter scan and
a request server with HBM-budget admission.

spiffe runs one problem per process (spiffe.c:85-365).  A design scan or a
stream of requests is many small problems, each of which alone leaves most
of a B200 idle, so they run concurrently: every instance keeps its own CUDA
stream and device state and the kernels of different instances overlap.

* ``draw_requests`` draws the scan's instances: mesh log-uniform between
  80 x 120 and 400 x 1500 nodes (nr x nz), pillbox or 1.6-cell gun (50/50),
  10k-500k macroparticles (log-uniform), RF phase U(0, 90 deg), peak field
  U(60, 120) MV/m, bunch charge log-U(0.05, 2) nC, solenoid peak U(0, 0.3) T
  (the gun), parameter seed 1234 and emission seed 987654321 + index.
* ``build`` turns a request into a ready instance: the pillbox emits its
  bunch from a cathode at the drawn RF phase; the gun starts from its bunch
  already emitted by the drawn cathode field, with the drawn solenoid.
* ``run_scan`` advances a set of instances together through the library's
  native scheduler (``spiffe_gpu_batch_run``).
* ``Server`` admits requests that arrive as a Poisson process while the sum
  of the running requests' device footprints stays within a budget: first
  come first served, with backfill (a later request that fits may start
  while the head of the queue waits for memory, unless the head has already
  been passed over ``max_bypass`` times); it reports each request's latency
  (arrival to result) and their percentiles.

Each instance's arithmetic does not depend on what else runs: a result is
the same alone and in the mix (tests/test_serve.py).
"""
from __future__ import annotations

import dataclasses
import math
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import abi, workloads

# device bytes of an instance: a fixed part (allocation granularity, solver
# scratch), per mesh node (split form: FP32 E/B and imposed fields, int64
# current and particle charge, FP64 Psi/PsiImposed/Q, flags, update mask,
# FP64 staging, and the multigrid levels: FP32 correction and residual on
# the mesh, ten coefficient planes and two arrays a quarter the size on the
# next level, a sixteenth on the one after, padded rows) and per particle
# slot (the split particle layout, a second
# copy for the cell sort, sort keys, transfer staging).  An upper estimate:
# on a B200 the measured use of eight scan instances (18k-273k nodes,
# 39k-610k slots, a screen as large as the beam) lay 5-55 % below it.
FIXED_BYTES = 16 << 20
NODE_BYTES = {"split32": 200, "f64": 260}
PARTICLE_BYTES = {"split32": 360, "f64": 460}
RECORD_BYTES = 112  # one screen record slot


@dataclasses.dataclass
class ScanRequest:
    index: int
    kind: str           # "pillbox" or "gun"
    nz: int
    nr: int
    n_macro: int
    phase_deg: float    # RF phase of the emission
    peak_field: float   # V/m
    charge: float       # C
    solenoid: float     # T (gun only)
    steps: int
    seed: int           # emission seed

    @property
    def nodes(self):
        return (self.nz + 1) * (self.nr + 1)

    @property
    def capacity(self):
        return int(self.n_macro * 1.25) + 4096


def draw_requests(n, steps=5000, seed=1234, size_scale=1.0, particle_scale=1.0):
    """n scan instances.  size_scale and particle_scale shrink meshes and
    bunches for tests and short benchmark samples (1.0 = the scan as
    specified)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nz = int(round(math.exp(rng.uniform(math.log(120), math.log(1500))) * size_scale))
        nr = int(round(math.exp(rng.uniform(math.log(80), math.log(400))) * size_scale))
        kind = "pillbox" if rng.random() < 0.5 else "gun"
        n_macro = int(math.exp(rng.uniform(math.log(1e4), math.log(5e5))) * particle_scale)
        phase = float(rng.uniform(0.0, 90.0))
        field = float(rng.uniform(60e6, 120e6))
        charge = float(math.exp(rng.uniform(math.log(0.05e-9), math.log(2e-9))))
        sol = float(rng.uniform(0.0, 0.3))
        out.append(ScanRequest(i, kind, max(nz, 40), max(nr, 30), max(n_macro, 256), phase, field, charge, sol,
                               steps, 987654321 + i))
    return out


def footprint_bytes(req, precision="split32"):
    """Device bytes an instance of this request occupies (an upper estimate)."""
    return FIXED_BYTES + req.nodes * NODE_BYTES[precision] + req.capacity * (PARTICLE_BYTES[precision] +
                                                                            RECORD_BYTES)


def _precision(name):
    from . import gpu

    return gpu.PRECISION_SPLIT32 if name == "split32" else gpu.PRECISION_F64


def build(req, precision="split32"):
    """A GpuInstance of the request, after run_begin; returns (instance, config)."""
    from . import geometry, gpu

    push = abi.push_options(abi.COMPACT_SWAP, abi.SCREEN_PARTICLE)
    if req.kind == "pillbox":
        cfg = workloads.PillboxConfig(nz=req.nz, nr=req.nr, E0=-req.peak_field, charge=req.charge,
                                      n_macro=req.n_macro, seed=req.seed)
        f_rf = 2.405 * workloads.C_MKS / (2 * math.pi * cfg.R)
        cfg.t_centre = max(req.phase_deg / 360.0 / f_rf, 4 * cfg.sigma_t)
        f = geometry.fields_for(cfg.nz, cfg.nr, cfg.zmin, cfg.zmax, cfg.rmax, cfg.geo_text(),
                                modes=abi.FL_TM_FIELDS | abi.FL_RADIAL_INTERP | abi.FL_LONGIT_INTERP |
                                abi.FL_SPACE_CHARGE)
        f.mesh.dt = cfg.dt
        f["Ez"] = cfg.initial_ez()
        g = gpu.GpuInstance(f, capacity=req.capacity, precision=_precision(precision))
        g.add_screen(cfg.screen_z(), capacity=req.capacity)
        g.add_cathode(cfg.cathode_options())
        g.configure_run(space_charge=1, push=push)
    else:
        e_emit = req.peak_field * max(math.cos(math.radians(req.phase_deg)), 0.2)
        cfg = workloads.Gun16Config(nz=req.nz, nr=req.nr, n_macro=req.n_macro, charge=req.charge,
                                    E_cathode=e_emit, B_peak=req.solenoid, seed=req.seed)
        f, b = cfg.state()
        g = gpu.GpuInstance(f, capacity=req.capacity, precision=_precision(precision))
        g.upload_beam(b)
        g.add_screen(cfg.screen_z(), 1, capacity=req.capacity)
        g.configure_run(space_charge=1, push=push, poisson=cfg.poisson())
    g.run_begin()
    return g, cfg


def collect(g, req):
    """The request's result: its exit-screen records and particle count."""
    from . import moments

    rec = g.screen(0, capacity=req.capacity).records()
    np_end, _ = g.counts()
    work = g.work_counters()
    return {"moments": moments.exit_moments(rec), "records": len(rec["q"]), "np": np_end,
            "particle_steps": int(work["particle_steps"]), "cell_updates": int(req.nz * req.nr * work["fdtd_steps"])}


def run_scan(requests, precision="split32", workers=16, chunk=20):
    """Builds every request's instance, advances them together with the
    native scheduler and returns (results, done_ms, build_s)."""
    from . import gpu

    t0 = time.perf_counter()
    insts = [build(r, precision)[0] for r in requests]
    build_s = time.perf_counter() - t0
    for g in insts:
        g.synchronize()
    done = gpu.batch_run(insts, [r.steps for r in requests], workers=workers, chunk=chunk)
    results = [collect(g, r) for g, r in zip(insts, requests)]
    for g in insts:
        g.close()
    return results, done, build_s


def percentile(xs, p):
    """Nearest-rank percentile (p in [0, 100]) of a non-empty sequence."""
    s = sorted(xs)
    k = max(0, min(len(s) - 1, int(math.ceil(p / 100.0 * len(s))) - 1))
    return s[k]


class Server:
    """Admits requests under a device-memory budget and runs each on a worker
    thread (its own instance and stream).

    ``execute(request) -> result`` does the work (default: build, run the
    request's steps, collect, close); ``footprint(request) -> bytes`` sizes
    it.  Both can be replaced, so the admission logic is testable without a
    GPU."""

    def __init__(self, budget_bytes, workers=16, precision="split32", backfill=True, max_bypass=8,
                 execute=None, footprint=None):
        self.budget = float(budget_bytes)
        self.workers = int(workers)
        self.precision = precision
        self.backfill = backfill
        self.max_bypass = int(max_bypass)
        self.execute = execute or self._execute
        self.footprint = footprint or (lambda r: footprint_bytes(r, precision))

    def _execute(self, req):
        g, _ = build(req, self.precision)
        g.run_steps(req.steps)
        out = collect(g, req)
        g.close()
        return out

    def _pick(self, queue, in_use, bypassed):
        """Index in `queue` of the request to start next, or None."""
        if not queue:
            return None
        head = queue[0]
        if in_use + self.footprint(head) <= self.budget:
            return 0
        if not self.backfill or bypassed.get(head.index, 0) >= self.max_bypass:
            return None
        for k in range(1, len(queue)):
            if in_use + self.footprint(queue[k]) <= self.budget:
                bypassed[head.index] = bypassed.get(head.index, 0) + 1
                return k
        return None

    def serve(self, requests, rate, seed=1234):
        """Releases the requests as a Poisson process of the given rate
        (req/s, seeded) and serves them; returns one dict per request with
        arrival, start and end times (s from the first arrival), latency,
        the peak budget in use, and the result."""
        rng = np.random.default_rng(seed)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, len(requests)))
        arrivals -= arrivals[0]
        for r in requests:
            if self.footprint(r) > self.budget:
                raise ValueError(f"request {r.index} needs more than the whole budget")
        lock = threading.Condition()
        queue, running = [], [0]
        in_use = [0.0]
        peak = [0.0]
        bypassed = {}
        out = {}
        t0 = time.perf_counter()

        def done(req, fp, t_start, fut):
            with lock:
                in_use[0] -= fp
                running[0] -= 1
                exc = fut.exception()
                out[req.index] = {"arrival": float(arrivals[order[req.index]]), "start": t_start,
                                  "end": time.perf_counter() - t0, "error": repr(exc) if exc else None,
                                  "result": None if exc else fut.result()}
                lock.notify_all()

        order = {r.index: k for k, r in enumerate(requests)}
        nxt = 0
        with ThreadPoolExecutor(max_workers=self.workers) as pool:
            with lock:
                while len(out) < len(requests):
                    now = time.perf_counter() - t0
                    while nxt < len(requests) and arrivals[nxt] <= now:
                        queue.append(requests[nxt])
                        nxt += 1
                    while running[0] < self.workers:
                        k = self._pick(queue, in_use[0], bypassed)
                        if k is None:
                            break
                        req = queue.pop(k)
                        fp = self.footprint(req)
                        in_use[0] += fp
                        peak[0] = max(peak[0], in_use[0])
                        running[0] += 1
                        t_start = time.perf_counter() - t0
                        fut = pool.submit(self.execute, req)
                        fut.add_done_callback(lambda f, r=req, fp=fp, ts=t_start: done(r, fp, ts, f))
                    wait = None
                    if nxt < len(requests):
                        wait = max(0.0, arrivals[nxt] - (time.perf_counter() - t0))
                    if len(out) < len(requests):
                        lock.wait(timeout=wait if wait is not None else 1.0)
        rows = []
        for r in requests:
            o = out[r.index]
            o["latency"] = o["end"] - o["arrival"]
            o["index"] = r.index
            o["peak_in_use"] = peak[0]
            rows.append(o)
        return rows
