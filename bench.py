#!/usr/bin/env python
"""Benchmark of spiffe's per-timestep PIC loop on one B200 (or N replicas).

Workload: the 1.6-cell RF gun -- 3001 x 821 nodes at 50 um, 1,000,000
macroparticles of a 1 nC, 2 ps bunch, solenoid, Poisson correction every 20
steps (spiffe_b200.workloads.Gun16Config).  One step is one pass of the
perform_integration loop body (integrate.c:136-193): J zero and deposit,
Poisson correction when due, FDTD, gather and push with wall losses and the
exit screen.  The metric is active particles pushed per second (with cell
updates per second beside it), measured on the device with CUDA events on
the library's stream, maximum over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--impl reference times the reference spiffe's own CPU code (compiled from
its sources into oracle/_ref) on the same state, with all host threads.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s & cell-updates/s per B200 at ≤0.5% moment error vs FP64; p50/p99"
UNIT = "particle-steps/s"
QoMC = -1.602176634e-19 / (9.1093837015e-31 * 2.99792458e8)

# algorithmic bytes per unit: the compulsory traffic of each phase in each form
BYTES = {
    "f64": {
        "fdtd": 74.0,     # per node-step: read Ez,Er,Bphi,Jz,Jr (40) + flags (2); write Ez,Er,Bphi,Bphi2 (32)
        "push": 144.0,    # per particle-step: read 9 doubles + status (80); write 8 doubles (64)
        "deposit": 80.0,  # per particle-step: z, r, v, Q, status for Jz and again for Jr
        "sor": 13.0,      # per node and half-sweep: read Psi, rhs, flags; write half of Psi
        "correction": 110.0,  # per node and correction: two flux passes, rhs scaling, gradient update
    },
    "split32": {
        "fdtd": 29.0,     # per node-step: read Ez,Er,Bphi (12) + mask (1); write Ez,Er,Bphi,Bphi2 (16); the int64
                          # current is read and cleared only on the rows the deposition touched
        "push": 86.0,     # per particle-step: read cell,fz,fr,pz,pr,r_pphi,Q,status,4 extrema (45); write all
                          # but Q (41); the next step's deposition is fused in (its J traffic stays in L2)
        "deposit": 29.0,  # per particle-step (first step only): cell, offsets, momenta, Q, status
        "sor": 7.0,       # per node and half-sweep: FP32 d and r0 (the bands live in shared memory)
        "mg": 180.0,      # per node and V-cycle: FP64 residual (25) and fold (20), four red-black sweeps on the
                          # mesh (56), transfers (12), the nine-point levels below (about 67)
        "correction": 90.0,  # per node and correction: flux passes, charge combine, rhs scaling, FP64 r0 and fold
    },
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=600)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--precision", default="split32", choices=["split32", "f64"],
                   help="split32: FP32 fields/push, split positions, fixed-point current (the form the metric is "
                        "quoted on); f64: the plain FP64 drop-in")
    p.add_argument("--f64-steps", type=int, default=200,
                   help="steps of the plain FP64 form timed on the same state for comparison (0: skip)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true", help="skip the end-to-end run (profiling captures)")
    p.add_argument("--cpu-steps", type=int, default=20, help="reference steps timed for the CPU baseline")
    p.add_argument("--workload", default="gun16", choices=["gun16", "dcgun", "scan", "serve"],
                   help="gun16: the benchmark (config 2); dcgun: the DC gun (config 3), both forms; scan: a sample "
                        "of the batched scan (config 4) run together; serve: a sample of the request stream "
                        "(config 5) at several arrival rates")
    p.add_argument("--instances", type=int, default=64, help="scan: instances drawn from the scan distribution")
    p.add_argument("--scan-steps", type=int, default=500, help="scan/serve: integration steps per instance")
    p.add_argument("--workers", type=int, default=4, help="scan/serve: host threads driving instances")
    p.add_argument("--requests", type=int, default=48, help="serve: requests per arrival rate")
    p.add_argument("--rates", default="5,10,20", help="serve: arrival rates in requests/s")
    p.add_argument("--budget-gb", type=float, default=150.0, help="serve: device-memory admission budget")
    p.add_argument("--scale", type=int, default=1,
                   help="coarsen the mesh by this factor and the beam by its square (small profiling cases)")
    return p.parse_args()


def combine_ranks(dist, ms, e2e_ms, psteps, e2e_psteps, device):
    """The job's figures from every rank's (replicas: each GPU runs the whole
    workload): the slowest rank's times and the sum of the work.  dist is
    torch.distributed with an initialised group, or None for one process."""
    if not dist:
        return ms, e2e_ms, float(psteps), float(e2e_psteps)
    import torch

    t = torch.tensor([ms, e2e_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    w = torch.tensor([psteps, e2e_psteps], dtype=torch.float64, device=device)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return float(t[0]), float(t[1]), float(w[0]), float(w[1])


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100", "-f", self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) < 9:
                        continue
                    try:
                        sm.append(float(parts[1]))
                        mx = float(parts[2])
                    except ValueError:
                        continue
                    for n, v in zip(names, parts[5:9]):
                        if v.lower() == "active":
                            reasons.add(n)
            os.unlink(self.path)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "samples": len(sm),
                "reasons": sorted(reasons)}


def build_state(cfg):
    """Mesh flags from the product's define_geometry, the analytic field, the
    solenoid and the beam, as abi containers."""
    return cfg.state()


def pinned_like(arr):
    import torch

    t = torch.empty(arr.shape, dtype=getattr(torch, str(arr.dtype).replace("uint64", "int64")), pin_memory=True)
    out = t.numpy().view(arr.dtype)
    out[...] = arr
    return out, t


def reference_sample(cfg, steps, warmup=1, threads=None):
    """The reference's own perform_integration loop body (integrate.c:136-193,
    compiled from its sources) on the same state; returns timing per step."""
    from oracle import pyoracle
    from spiffe_b200 import abi, workloads

    threads = threads or os.cpu_count()
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "gun.geo"), "w") as fgeo:
        fgeo.write(cfg.geo_text())
    geom = workloads.geometry_command(cfg.nz, cfg.nr, cfg.zmin, cfg.zmax, cfg.rmax, "gun.geo")
    pc = workloads.namelist("poisson_correction", step_interval=cfg.step_interval, accuracy=1e-6,
                            maximum_iterations=1000)
    scr = workloads.namelist("define_screen", filename="exit", z_position=cfg.screen_z())
    modes = abi.FL_TM_FIELDS | abi.FL_RADIAL_INTERP | abi.FL_LONGIT_INTERP | abi.FL_SPACE_CHARGE
    flags_prog = [("command", geom), ("get_flags",)]
    flags = pyoracle.run_reference(flags_prog, cwd=d, threads=threads)[0]
    arrays = cfg.beam_arrays()
    n = len(arrays["z"])
    bz, br = cfg.solenoid()
    prog = [("command", geom), ("command", pc), ("command", scr), ("set_time", cfg.dt, 0.0, 0, modes),
            ("set_field", "Ez", cfg.initial_ez(flags)), ("set_field", "BzImposed", bz), ("set_field", "BrImposed", br),
            ("set_beam", (n, n, 0, n + 1), (QoMC, 1.0), arrays), ("call", "ref_calculate_areas_and_setup"),
            ("call", "ref_compute_imposed_Efield", 1), ("call", "ref_add_poisson_correction", 1),
            ("time_steps", warmup, 1, -1.0), ("time_steps", steps, 1, -1.0)]
    res = pyoracle.run_reference(prog, cwd=d, capacity=int(n * 1.25), threads=threads, timeout=3600)
    timed = res[-1]
    secs = sum(t for t, _ in timed)
    psteps = sum(a for _, a in timed)
    return {"seconds": secs, "particle_steps": psteps, "steps": steps, "threads": threads,
            "value": psteps / secs if secs else 0.0,
            "cell_updates_per_s": cfg.nz * cfg.nr * steps / secs if secs else 0.0}


def scaled_config(scale):
    from spiffe_b200 import workloads

    if scale <= 1:
        return workloads.Gun16Config()
    return workloads.Gun16Config(nz=3000 // scale + 1, nr=820 // scale + 1, n_macro=1_000_000 // scale ** 2)


def e2e_phase(f, host_f, host_b, b, cfg, push, mesh_w, prec, K, dist):
    """The same K steps end to end through the public API from pinned host
    buffers: state upload, K single-step calls each followed by a read-back of
    that step's particle count into pinned memory (queued, no per-step stall),
    state download.  Returns (ms, particle-steps, state bytes)."""
    import numpy as np
    import torch

    from spiffe_b200 import gpu

    # pinned copies: the caller's post-warm-up state stays as it is
    host_f, host_b = host_f.copy(), host_b.copy()
    pin = {}
    for k, v in host_f.a.items():
        host_f.a[k], pin[k] = pinned_like(v)
    for k, v in host_b.a.items():
        host_b.a[k], pin["b" + k] = pinned_like(v)
    counts = pinned_like(np.zeros((K, 2), np.int64))
    pin["counts"] = counts[1]
    counts = counts[0]
    g2 = gpu.GpuInstance(f, capacity=b.capacity, precision=prec)
    g2.add_screen(cfg.screen_z(), 1, capacity=b.capacity)
    g2.configure_run(space_charge=1, push=push, poisson=cfg.poisson())
    g2.set_mesh(mesh_w)
    stream2 = torch.cuda.ExternalStream(g2.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    state_bytes = sum(v.nbytes for v in host_f.a.values()) + sum(
        v[: host_b.np].nbytes for v in host_b.a.values()) + host_b.np * (4 + 2 + 8)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream2)
    g2.upload_fields(host_f)
    g2.upload_beam(host_b)
    wb0 = g2.work_counters()
    for k in range(K):
        g2.run_steps(1)
        g2.counts_async(counts[k])  # this step's particle count, read back without a stall
    g2.synchronize()
    wb1 = g2.work_counters()
    g2.download_beam(host_b)
    g2.download_fields(host_f)
    e1.record(stream2)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    assert tuple(counts[-1]) == g2.counts(), "per-step count read back"
    g2.close()
    return ms, wb1["particle_steps"] - wb0["particle_steps"], state_bytes


def gpu_arm(args):
    import torch

    from spiffe_b200 import abi, gpu, workloads

    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    gpu.select_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as td

        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = td
    cfg = scaled_config(args.scale)
    f, b = build_state(cfg)
    K, W = args.steps, args.warmup
    push = abi.push_options(compaction=abi.COMPACT_SWAP, screen_momentum=abi.SCREEN_PARTICLE)
    prec = gpu.PRECISION_SPLIT32 if args.precision == "split32" else gpu.PRECISION_F64
    nbytes = BYTES[args.precision]

    # --- device-resident throughput
    g = gpu.GpuInstance(f, capacity=b.capacity, precision=prec)
    g.upload_beam(b)
    g.add_screen(cfg.screen_z(), 1, capacity=b.capacity)
    g.configure_run(space_charge=1, push=push, poisson=cfg.poisson())
    g.run_begin()
    g.run_steps(W)
    g.synchronize()
    # host copy of the post-warm-up state, for the end-to-end run
    host_f, host_b = f.copy(), abi.Beam(b.capacity)
    g.download_fields(host_f)
    g.download_beam(host_b)
    mesh_w = g.get_mesh()
    stream = torch.cuda.ExternalStream(g.stream_handle())
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    g.set_profiling(True)
    w0 = g.work_counters()
    l0 = gpu.launch_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0.record(stream)
    g.run_steps(K)
    ev1.record(stream)
    ev1.synchronize()
    clk = clocks.stop()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = gpu.launch_count() - l0
    w1 = g.work_counters()
    phases = g.phase_times()
    g.set_profiling(False)
    psteps = w1["particle_steps"] - w0["particle_steps"]
    halfsweeps = w1["sor_halfsweeps"] - w0["sor_halfsweeps"]
    solves = w1["sor_solves"] - w0["sor_solves"]
    cycles = w1["mg_cycles"] - w0["mg_cycles"]
    np_end, _ = g.counts()
    g.close()

    # --- end to end through the public API from pinned host buffers, right
    # after the timed run (before the FP64 comparison, whose FP64-heavy
    # instance would otherwise precede it)
    e2e_ms, e2e_psteps, state_bytes = 0.0, 0, 0
    if not args.no_e2e:
        e2e_ms, e2e_psteps, state_bytes = e2e_phase(f, host_f, host_b, b, cfg, push, mesh_w, prec, K, dist)

    f64_form = None
    if prec == gpu.PRECISION_SPLIT32 and args.f64_steps > 0:
        # the plain FP64 drop-in on the same post-warm-up state, same GPU, same run
        g3 = gpu.GpuInstance(f, capacity=b.capacity, precision=gpu.PRECISION_F64)
        g3.add_screen(cfg.screen_z(), 1, capacity=b.capacity)
        g3.configure_run(space_charge=1, push=push, poisson=cfg.poisson())
        g3.upload_fields(host_f)
        g3.upload_beam(host_b)
        g3.set_mesh(mesh_w)
        s3 = torch.cuda.ExternalStream(g3.stream_handle())
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        K3 = args.f64_steps
        g3.run_steps(2)
        g3.synchronize()
        x0 = g3.work_counters()
        f0.record(s3)
        g3.run_steps(K3)
        f1.record(s3)
        f1.synchronize()
        x1 = g3.work_counters()
        f64_val = (x1["particle_steps"] - x0["particle_steps"]) / (f0.elapsed_time(f1) / 1e3)
        f64_form = {"value": round(f64_val, 1), "unit": UNIT, "steps": K3,
                    "ms_per_step": round(f0.elapsed_time(f1) / K3, 4),
                    "how": "plain FP64 drop-in on the same post-warm-up state and GPU, right after the split-form "
                           "run; its K steps hold the same share of Poisson corrections (one per 20 steps)"}
        g3.close()
    # --- totals over ranks (max time, summed work)
    ms, e2e_ms, psteps_all, e2e_all = combine_ranks(dist, ms, e2e_ms, psteps, e2e_psteps, "cuda")
    sec = ms / 1e3
    value = psteps_all / sec
    cells = cfg.nz * cfg.nr * K * world / sec

    # --- roofline of the dominant phase
    nodes = (cfg.nz + 1) * (cfg.nr + 1)
    sor_nodes = cfg.nz * (cfg.nr - 1)
    work_bytes = {
        "fdtd": nbytes["fdtd"] * nodes * phases["fdtd"][1],
        "push": nbytes["push"] * psteps,
        "deposit": nbytes["deposit"] * psteps if prec == gpu.PRECISION_F64 else nbytes["deposit"] * cfg.n_macro * phases["deposit"][1],
        "poisson": nbytes["sor"] * sor_nodes * halfsweeps + nbytes.get("mg", 0.0) * nodes * cycles +
                   nbytes["correction"] * nodes * solves,
        "emission": 0.0,
    }
    total_ms = sum(v[0] for v in phases.values()) or 1.0
    peak, peak_kind = measured_peak()
    breakdown = {k: {"ms": round(v[0], 3), "launches": v[1], "share": round(v[0] / total_ms, 4),
                     "gbs": round(work_bytes[k] / (v[0] / 1e3) / 1e9, 1) if v[0] > 0 else None,
                     "frac": round(work_bytes[k] / (v[0] / 1e3) / 1e9 / peak, 3) if v[0] > 0 else None}
                 for k, v in phases.items()}
    breakdown["poisson"]["solves"] = solves
    breakdown["poisson"]["halfsweeps_per_solve"] = round(halfsweeps / solves, 1) if solves else 0
    breakdown["poisson"]["vcycles_per_solve"] = round(cycles / solves, 2) if solves else 0
    dom = max(phases, key=lambda k: phases[k][0])
    dom_units = {"fdtd": phases["fdtd"][1], "push": phases["push"][1], "deposit": phases["deposit"][1],
                 "poisson": max(solves, 1), "emission": 1}[dom]
    achieved = work_bytes[dom] / (phases[dom][0] / 1e3) / 1e9 if phases[dom][0] > 0 else 0.0
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.json")) as ft:
            traffic = json.load(ft).get(dom)
    except (OSError, ValueError):
        pass
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": traffic, "bytes_per_launch": round(work_bytes[dom] / max(dom_units, 1)),
                "avg_launch_ms": round(phases[dom][0] / max(dom_units, 1), 4)}

    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": round(ms / K, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if prec == gpu.PRECISION_SPLIT32 else "f64", "data": "synthetic",
        "config": {"workload": "1.6-cell RF gun, 3001x821 nodes at 50um, 1,000,000 macroparticles, "
                               "Poisson correction every 20 steps, solenoid",
                   "form": ("split precision: FP32 fields and push, cell+FP32-offset positions, 64-bit fixed-point "
                            "current, FP32 multigrid in FP64 iterative refinement") if prec == gpu.PRECISION_SPLIT32
                   else "plain FP64 (bit-faithful to the reference)",
                   "field": "stand-in: an analytic pi-mode standing wave, 100 MV/m on the cathode, in place of the "
                            "30,000-step antenna build-up and reload",
                   "beam": "stand-in: the 1 nC, 2 ps rms bunch generated already emitted (positions from uniform "
                           "acceleration by the cathode field), so the timed steps hold no emission",
                   "particles": cfg.n_macro, "nodes": cfg.nz * cfg.nr, "steps_timed": K,
                   "poisson_solver": ("multigrid (FP32 V-cycles in FP64 refinement)" if prec == gpu.PRECISION_SPLIT32
                                      else "the reference's red-black SOR"),
                   "l2": ("no flush: each step streams the 1M-particle beam (%d MB read and written) and the fields; "
                          "the split form keeps its ~%d MB of FP32 TM fields in an L2 persisting window on purpose, "
                          "as it does in production" % (cfg.n_macro * 86 // 2 ** 20,
                                                        16 * (cfg.nz + 1) * ((cfg.nr + 1 + 31) // 32 * 32) // 2 ** 20))
                         if prec == gpu.PRECISION_SPLIT32 else
                         "no flush: the resident state (fields ~%d MB, beam ~%d MB) exceeds the 126 MB L2"
                         % (sum(v.nbytes for v in f.a.values()) // 2 ** 20, sum(v.nbytes for v in b.a.values()) // 2 ** 20),
                   "parallelism": "replicas" if world > 1 else "single"},
        "cell_updates_per_s": round(cells, 1),
        "particles_end": np_end,
        "phases": breakdown,
        "roofline": roofline,
        "gpu_launches": launches,
        "clocks": clk,
        "e2e": None if args.no_e2e else {"value": round(e2e_all / (e2e_ms / 1e3), 1), "unit": UNIT,
                "h2d_bytes_per_step": int(state_bytes / K), "d2h_bytes_per_step": int((state_bytes + 8 * K) / K),
                "how": "public API from pinned host buffers: state upload, K single-step calls each followed by a "
                       "queued read-back of that step's particle count into pinned memory, state download"},
    }
    if f64_form:
        f64_form["split_over_f64"] = round(value / f64_form["value"], 3) if f64_form["value"] else None
        line["f64_form"] = f64_form
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            s = reference_sample(cfg, args.cpu_steps)
            line["cpu_baseline"] = {"value": round(s["value"], 1), "unit": UNIT, "cores": s["threads"],
                                    "kind": "reference",
                                    "sample": "%d perform_integration steps of the reference (one Poisson interval) "
                                              "on the same 1M-particle state, after 1 warm-up step, %.1f s"
                                              % (s["steps"], s["seconds"])}
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                                    "sample": "unavailable: %s" % str(e)[:200]}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def reference_arm(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    from oracle import pyoracle
    from spiffe_b200 import workloads

    if not pyoracle.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libspiffe_ref.so was not built"}))
        return
    cfg = scaled_config(args.scale)
    steps = min(args.steps, args.cpu_steps)
    s = reference_sample(cfg, steps, warmup=max(1, min(args.warmup, 1)))
    line = {
        "impl": "reference", "metric": METRIC, "value": round(s["value"], 1), "unit": UNIT, "n_gpus": world,
        "steps": steps, "warmup": 1, "ms_per_step": round(1e3 * s["seconds"] / steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "1.6-cell RF gun, 3001x821 nodes at 50um, 1,000,000 macroparticles, "
                               "Poisson correction every 20 steps, solenoid",
                   "form": "reference spiffe CPU code (OpenMP push)", "steps_timed": steps},
        "cell_updates_per_s": round(s["cell_updates_per_s"], 1),
        "cpu_baseline": {"value": round(s["value"], 1), "unit": UNIT, "cores": s["threads"], "kind": "reference",
                         "sample": "%d perform_integration steps (a bounded sample of the K requested)" % steps},
        "e2e": {"value": round(s["value"], 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def dcgun_arm(args):
    """The DC gun (1501 x 1001 nodes, 4M particles, a Poisson correction
    every step): --steps timed steps of the split form and half as many of
    the FP64 form, on the same state after --warmup steps each."""
    import torch

    from spiffe_b200 import abi, gpu, workloads

    torch.cuda.set_device(0)
    cfg = workloads.DcGunConfig()
    f, b = cfg.state()
    push = abi.push_options(compaction=abi.COMPACT_SWAP, screen_momentum=abi.SCREEN_PARTICLE)
    nodes = (cfg.nz + 1) * (cfg.nr + 1)
    legs = {}
    clk = None
    for name, prec, K in (("split32", gpu.PRECISION_SPLIT32, args.steps),
                          ("f64", gpu.PRECISION_F64, max(args.steps // 2, 3))):
        g = gpu.GpuInstance(f, capacity=b.capacity, precision=prec)
        g.upload_beam(b)
        g.add_screen(cfg.screen_z(), 1, capacity=b.capacity)
        g.configure_run(space_charge=1, push=push, poisson=cfg.poisson())
        g.run_begin()
        g.run_steps(args.warmup)
        g.synchronize()
        stream = torch.cuda.ExternalStream(g.stream_handle())
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clocks = ClockSampler(0)
        g.set_profiling(True)
        w0 = g.work_counters()
        torch.cuda.synchronize()
        clocks.start()
        ev0.record(stream)
        g.run_steps(K)
        ev1.record(stream)
        ev1.synchronize()
        c = clocks.stop()
        clk = clk or c
        ms = ev0.elapsed_time(ev1)
        w1 = g.work_counters()
        phases = g.phase_times()
        np_end, _ = g.counts()
        g.close()
        ps = w1["particle_steps"] - w0["particle_steps"]
        legs[name] = {"steps": K, "ms_per_step": round(ms / K, 4), "particle_steps_per_s": round(ps / (ms / 1e3), 1),
                      "cell_updates_per_s": round(nodes * K / (ms / 1e3), 1),
                      "sor_halfsweeps_per_step": round((w1["sor_halfsweeps"] - w0["sor_halfsweeps"]) / K, 1),
                      "particles_end": np_end,
                      "phases_ms_per_step": {k: round(v[0] / K, 4) for k, v in phases.items() if v[1]}}
    line = {"metric": "particle-steps/s & cell-updates/s of the DC gun (config 3)",
            "value": legs["split32"]["particle_steps_per_s"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": legs["split32"]["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "DC gun, 1501x1001 nodes at 20um, 300 kV gap of 10 mm, 4,000,000 macroparticles "
                                   "(0.5 nC, 100 ps flat top, already emitted), Poisson correction every step",
                       "form": "split precision; plain FP64 leg on the same state"},
            "cell_updates_per_s": legs["split32"]["cell_updates_per_s"], "legs": legs,
            "split_over_f64": round(legs["f64"]["ms_per_step"] / legs["split32"]["ms_per_step"], 3), "clocks": clk}
    print(json.dumps(line), flush=True)


def scan_arm(args):
    """A sample of the batched scan: --instances drawn from its distribution,
    --scan-steps each, advanced together by the native scheduler on
    --workers threads, then the same instances one at a time."""
    import torch

    from spiffe_b200 import serve

    torch.cuda.set_device(0)
    serve.run_scan(serve.draw_requests(2, steps=5, size_scale=0.25, particle_scale=0.02), workers=2)  # warm-up
    reqs = serve.draw_requests(args.instances, steps=args.scan_steps)
    clocks = ClockSampler(0)
    clocks.start()
    res, done, build_s = serve.run_scan(reqs, workers=args.workers, chunk=20)
    clk = clocks.stop()
    seq, seq_done, _ = serve.run_scan(reqs, workers=1, chunk=0)
    wall = max(done) / 1e3
    ps = sum(r["particle_steps"] for r in res)
    cu = sum(r["cell_updates"] for r in res)
    assert [r["moments"] for r in res] == [r["moments"] for r in seq], "a result changed in the mix"
    line = {"metric": "particle-steps/s & cell-updates/s of a batched scan (config 4 sample)", "value": round(ps / wall, 1),
            "unit": UNIT, "n_gpus": 1, "steps": args.scan_steps, "warmup": 0, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "%d scan instances (pillbox or 1.6-cell gun, 80x120..400x1500 nodes, "
                                   "10k..500k macroparticles, seeds 1234 / 987654321+i), %d steps each"
                                   % (args.instances, args.scan_steps),
                       "form": "split precision", "workers": args.workers, "chunk": 20},
            "cell_updates_per_s": round(cu / wall, 1), "wall_s": round(wall, 3), "build_s": round(build_s, 3),
            "completion_ms": {"p50": round(statistics.median(done), 1),
                              "p99": round(sorted(done)[max(0, math.ceil(0.99 * len(done)) - 1)], 1)},
            "one_at_a_time": {"wall_s": round(max(seq_done) / 1e3, 3),
                              "value": round(ps / (max(seq_done) / 1e3), 1)},
            "results_identical_alone_and_in_the_mix": True, "clocks": clk}
    print(json.dumps(line), flush=True)


def serve_arm(args):
    """A sample of the request stream: --requests per rate from the scan
    distribution, --scan-steps each, Poisson arrivals, admission within
    --budget-gb of device memory, --workers concurrent requests."""
    import torch

    from spiffe_b200 import serve

    torch.cuda.set_device(0)
    serve.run_scan(serve.draw_requests(2, steps=5, size_scale=0.25, particle_scale=0.02), workers=2)  # warm-up
    rates = [float(x) for x in args.rates.split(",") if x]
    out = {}
    for k, rate in enumerate(rates):
        reqs = serve.draw_requests(args.requests, steps=args.scan_steps, seed=1234 + k)
        srv = serve.Server(args.budget_gb * 1e9, workers=args.workers)
        rows = srv.serve(reqs, rate=rate, seed=4321 + k)
        lat = [r["latency"] for r in rows]
        errs = [r["error"] for r in rows if r["error"]]
        span = max(r["end"] for r in rows)
        out["%g" % rate] = {"p50_s": round(serve.percentile(lat, 50), 4), "p99_s": round(serve.percentile(lat, 99), 4),
                            "served_per_s": round(len(rows) / span, 2), "errors": len(errs),
                            "peak_budget_gb": round(rows[0]["peak_in_use"] / 1e9, 3),
                            "particle_steps_per_s": round(sum(r["result"]["particle_steps"] for r in rows
                                                              if r["result"]) / span, 1)}
    worst = max(out.values(), key=lambda v: v["p99_s"])
    line = {"metric": "request latency p50/p99 under Poisson arrivals (config 5 sample)", "value": worst["p99_s"],
            "unit": "s (p99, highest rate)", "n_gpus": 1, "steps": args.scan_steps, "warmup": 0,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "%d requests per rate from the scan distribution, %d steps each, Poisson "
                                   "arrivals, %.0f GB admission budget" % (args.requests, args.scan_steps,
                                                                          args.budget_gb),
                       "form": "split precision", "workers": args.workers},
            "rates": out}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    elif args.workload == "dcgun":
        dcgun_arm(args)
    elif args.workload == "scan":
        scan_arm(args)
    elif args.workload == "serve":
        serve_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
