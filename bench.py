"""Benchmark: particle RK4 steps/s of Emu's evolution path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl emu|reference]
                    [--workload c2|c3|c5] [--precision fp64|mixed]

A step is one RK4 step (4 stages: deposit, interpolate, -i[H,rho], stage
update; then wrap, Renormalize and compute_dt on the device) over every
particle of the workload.  Default workload: C2, the fast-flavor 1D case
(2 flavors, 1x1x128 cells, 80 Fibonacci directions per cell, 10,240
particles, FP64).  Inputs are synthetic (seeded initial conditions).

Timing: W untimed warm-up steps, then K steps, each bracketed by CUDA events
on the launching stream with an L2 flush (512 MB write) before every step;
the reported time is the sum of the K step durations, max over ranks.  With
torchrun (N > 1) every rank runs an independent replica of the workload on
its own GPU (weak scaling).

--impl reference times the reference's per-particle arithmetic on the host
cores (oracle/_ref: Emu's generated kernel bodies in the restated AMReX
loops; the oracle port when _ref is absent) on the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from emu_b200 import api  # noqa: E402
from emu_b200 import workloads as W  # noqa: E402

METRIC = "particle RK4 steps/s on 1 B200: mixed vs FP64 at stated err; % of HBM peak"


def workload(name, precision, cells=None, fused=None, resort=None, ranks=1):
    """cells overrides the cell count (z cells for c2/c3, cells per side for
    c5) to run a smaller case of the same workload (profiling).  With ranks
    > 1 every cell gets ranks times the directions, so that each rank's
    shard (every ranks-th particle) has the single-GPU particle count."""
    if name == "c2":
        p = W.c2_fast_flavor_1d(ncell_z=cells or 128, ndirs=80 * ranks)
        desc = "C2 fast-flavor 1D: 2 flavors, 1x1x%d cells over %g cm, %d Fibonacci directions/cell" % (
            p.ncell[2], p.Lz, 80 * ranks)
    elif name == "c4":
        p = W.c4_adjoint()
        desc = ("C4 adjoint: C2 sizes (2 flavors, 1x1x%d cells, 80 directions/cell), %d RK4 steps, "
                "checkpoints every 25 steps" % (p.ncell[2], p.nsteps))
    elif name == "c3":
        p = W.c3_three_flavor_1d(ncell_z=cells or 1024)
        desc = "C3 3-flavor 1D: 1x1x%d cells, 378 ring directions/cell" % p.ncell[2]
        if ranks > 1:
            p.direction_generator, p.ndirections = 1, 378 * ranks
            desc = "C3 3-flavor 1D: 1x1x%d cells, %d Fibonacci directions/cell" % (p.ncell[2], 378 * ranks)
    elif name == "c5":
        p = W.c5_3d(n=cells or 64, ndirs=96 * ranks)
        desc = "C5 3-flavor 3D: %d^3 cells x %d Fibonacci directions" % (p.ncell[0], 96 * ranks)
    else:
        raise SystemExit("unknown workload " + name)
    if precision:
        p.precision = api.PREC_MIXED if precision == "mixed" else api.PREC_FP64
    if fused:
        p.fused = fused
    if resort is not None:
        p.resort_interval = resort
    return p, desc


def algorithmic_bytes_per_particle_step(nf, mixed):
    """Compulsory HBM bytes per particle per RK4 step of the fused
    one-pass-per-stage design (S = static fields per pass, F64 = 2 NF^2 FP64
    flavor reals, Fs = stage-state width, E4 = L, Lbar read + pos, time
    written): plain 4S + 16 F64 + E4, mixed 4S + 10 F64 + 6 Fs + E4."""
    F64 = 2 * nf * nf * 8
    E4 = 48
    if mixed:
        S = 48
        Fs = 2 * nf * nf * 4
        return 4 * S + 10 * F64 + 6 * Fs + E4
    S = 72
    return 4 * S + 16 * F64 + E4


def mesh_bytes_per_step(p, nf):
    ncells = p.ncell[0] * p.ncell[1] * p.ncell[2]
    return 4 * 2 * ncells * 8 * nf * nf * 8


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for i, n in enumerate(names):
                if r[5 + i].strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def cpu_baseline(p, recs, budget_s, nthreads):
    """The reference arithmetic on host cores: run whole steps of the
    workload until the time budget is spent; particle-steps/s."""
    from oracle.oracle import Oracle, RefHarness, have_ref
    kind = "reference" if have_ref(p.nflavors) else "port"
    o = RefHarness(p) if kind == "reference" else Oracle(p)
    parts = np.array(recs, copy=True)
    vmax = o.vvac_max(parts)
    mesh = o.deposit(parts, nthreads)
    dt, _ = o.compute_dt(mesh, vmax)
    steps = 0
    t0 = time.perf_counter()
    while True:
        mesh, _, _ = o.rk_step(parts, dt, nthreads=nthreads)
        dt, _ = o.compute_dt(mesh, vmax)
        steps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or steps >= 100000:
            break
    return {"value": len(parts) * steps / el, "unit": "particle-steps/s", "cores": nthreads, "kind": kind,
            "sample": "%d full RK4 steps of the workload (%d particles), %.1f s" % (steps, len(parts), el)}


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference(args):
    ws, rank, local = dist_setup(args)
    if rank != 0:
        return
    # the emu arm's configuration (with N ranks: N times the directions)
    p, desc = workload(args.workload, args.precision, args.cells, args.fused, args.resort,
                       ws if args.workload != "c4" else 1)
    recs = api.init_particles(p)
    nthreads = os.cpu_count() or 1
    from oracle.oracle import Oracle, RefHarness, have_ref
    kind = "reference" if have_ref(p.nflavors) else "port"
    o = RefHarness(p) if kind == "reference" else Oracle(p)
    # bounded sample: at most ~2 minutes of host time in total
    parts = np.array(recs, copy=True)
    vmax = o.vvac_max(parts)
    mesh = o.deposit(parts, nthreads)
    dt, _ = o.compute_dt(mesh, vmax)
    for _ in range(args.warmup):
        mesh, _, _ = o.rk_step(parts, dt, nthreads=nthreads)
        dt, _ = o.compute_dt(mesh, vmax)
    t0 = time.perf_counter()
    steps = 0
    for _ in range(args.steps):
        mesh, _, _ = o.rk_step(parts, dt, nthreads=nthreads)
        dt, _ = o.compute_dt(mesh, vmax)
        steps += 1
        if time.perf_counter() - t0 > 120:
            break
    el = time.perf_counter() - t0
    value = len(parts) * steps / el
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "particle-steps/s",
           "n_gpus": ws, "steps": steps, "warmup": args.warmup, "ms_per_step": el / steps * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic",
           "config": {"workload": desc, "particles": len(parts), "nflavors": p.nflavors,
                      "cells": list(p.ncell)},
           "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": nthreads, "kind": kind,
                            "sample": "%d RK4 steps of the full workload" % steps},
           "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def run_emu(args):
    import torch
    ws, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    if ws > 1 or args.sharded:
        import datetime
        import torch.distributed as dist
        if ws == 1:
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            os.environ.setdefault("MASTER_PORT", "29533")
            os.environ.setdefault("RANK", "0")
            os.environ.setdefault("WORLD_SIZE", "1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    multi = (ws > 1 or args.sharded) and args.workload != "c4"
    p, desc = workload(args.workload, args.precision, args.cells, args.fused, args.resort, ws if multi else 1)
    mixed = p.precision == api.PREC_MIXED
    nf = p.nflavors
    recs = api.init_particles(p)
    stream = torch.cuda.Stream()
    ctx = api.Context(p)
    ctx.set_stream(stream.cuda_stream)
    if multi:
        # particle sharding: this rank's particles, replicated mesh summed
        # over the ranks by an NCCL all-reduce after every deposit
        from emu_b200 import sharding
        sharding.attach(ctx, rank, ws)
        recs = sharding.shard(recs, rank, ws)
    n = recs.shape[0]
    ctx.load_particles(recs)
    # the library's automatic re-sort interval (resort_interval < 0)
    eff_resort = p.resort_interval
    if eff_resort < 0:
        eff_resort = 1 if sum(1 for c in p.ncell if c > 1) == 3 and p.shape_order >= 2 else 16
    total_steps = args.warmup + args.steps + args.profile_steps + 8
    ctx.evolve_begin(0.0, float("inf"), total_steps)
    flush_bytes = 512 << 20
    flush = torch.zeros(flush_bytes // 8, dtype=torch.float64, device="cuda")
    for _ in range(args.warmup):
        ctx.flush_l2(flush.data_ptr(), flush_bytes)
        ctx.evolve_steps(1)
    ctx.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = ClockSampler(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ else local)
    sampler.start()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    for i in range(args.steps):
        ctx.flush_l2(flush.data_ptr(), flush_bytes)
        evs[i][0].record(stream)
        ctx.evolve_steps(1)
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    wall = time.perf_counter() - wall0
    clocks = sampler.stop()
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if ws > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    total_ms = float(t.item())
    info = ctx.evolve_end()
    if info.status != 0:
        raise SystemExit("device status %d during the benchmark: %s" % (info.status, api.last_error(ctx.h)))
    value = n * args.steps * ws / (total_ms * 1e-3)

    # roofline of the stage kernel: per-kernel CUDA events on the stream
    ctx.evolve_begin(0.0, float("inf"), args.profile_steps + 2)
    kms = []
    for _ in range(args.profile_steps):
        ctx.flush_l2(flush.data_ptr(), flush_bytes)
        kms.append(ctx.profile_step())
    kms = np.array(kms)
    per_pstep = algorithmic_bytes_per_particle_step(nf, mixed)
    coop = kms.shape[1] == 1
    split = nf == 2 and p.ncell[0] == 1 and p.ncell[1] == 1 and not mixed   # species-split kernels
    if coop:
        # one cooperative kernel per step: the whole step is the launch
        kernel = "k_rk4_step_coop%s<%d>" % ("_split" if split else "", nf)
        stage_ms = float(kms[:, 0].mean())
        bytes_per_launch = per_pstep * n + mesh_bytes_per_step(p, nf)
    else:
        kernel = "k_rk4_stage%s<%d>" % ("_mixed" if mixed else ("_split" if split else ""), nf)
        stage_idx = [1, 3, 5, 7] if mixed else [0, 1, 2, 3]
        stage_ms = float(kms[:, stage_idx].mean())
        bytes_per_launch = (per_pstep * n + mesh_bytes_per_step(p, nf)) / 4.0
    peak, peak_kind = load_peaks()
    achieved = bytes_per_launch / (stage_ms * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_%s_%s.json" % (args.workload, "mixed" if mixed else "fp64"))
    if os.path.exists(tpath) and args.cells is None:
        with open(tpath) as f:
            tj = json.load(f)
        # DRAM bytes per launch of this kernel from the ncu capture (scaled
        # from the captured case's particle count when it was a smaller one)
        if tj.get("kernel", "").split("<")[0] == kernel.split("<")[0]:
            traffic = tj.get("bytes_per_launch")

    # end to end through the C ABI with host buffers: every step uploads its
    # particles from pinned host memory, runs one device step and downloads
    # the state.  One GPU: `--e2e-pipes` independent batches, each with its
    # own context, stream and host thread, so that one batch's copies overlap
    # another's compute (PCIe copies in both directions run concurrently).
    e2e = None
    if not args.no_e2e:
        import threading
        # (pinned host buffers of all batches within 32 GB)
        # (automatic: 16 small batches in flight, 8 large ones, whose copies
        # already fill PCIe and contend beyond that)
        want = args.e2e_pipes if args.e2e_pipes > 0 else (16 if recs.nbytes < 16e6 else 8)
        pipes = max(1, min(want, int(32e9 // (2 * recs.nbytes)))) if ws == 1 else 1
        ne = min(args.steps, args.e2e_steps)
        lanes = []
        for k in range(pipes):
            if k == 0:
                c, s_ = ctx, stream
            else:
                s_ = torch.cuda.Stream()
                c = api.Context(p)
                c.set_stream(s_.cuda_stream)
            lanes.append((c, torch.from_numpy(recs).pin_memory(), torch.empty_like(torch.from_numpy(recs)).pin_memory()))

        def lane(c, pin_in, pin_out, count):
            for _ in range(count):
                c.load_particles_ptr(pin_in.data_ptr(), n)
                c.evolve_begin(0.0, float("inf"), 1)
                c.evolve_steps(1)
                c.get_particles_ptr(pin_out.data_ptr(), n)

        for c, pi, po in lanes:      # untimed: graphs and buffers of every lane
            lane(c, pi, po, 2)
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        threads = [threading.Thread(target=lane, args=(c, pi, po, ne)) for c, pi, po in lanes]
        e0 = time.perf_counter()
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        el = time.perf_counter() - e0
        t = torch.tensor([el], dtype=torch.float64, device="cuda")
        if ws > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        for c, _, _ in lanes[1:]:
            c.close()
        bytes_rec = n * api.nreal(nf) * 8
        e2e = {"value": n * ne * pipes * ws / float(t.item()), "unit": "particle-steps/s",
               "h2d_bytes_per_step": bytes_rec, "d2h_bytes_per_step": bytes_rec, "batches_in_flight": pipes,
               "note": "per step of a batch: emu_load_particles from pinned host memory, emu_evolve_begin "
                       "(deposit + compute_dt), one device step, emu_get_particles to pinned host memory; "
                       "%d batches with their own contexts and host threads run concurrently" % pipes}
        # its bound: pinned copies of the batch size, both directions at once
        pc = pcie_copy_rate(bytes_rec, pipes)
        pc["frac"] = e2e["value"] / n * bytes_rec / 1e9 / pc["concurrent_gbs_per_direction"]
        e2e["pcie"] = pc

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(p, recs, args.cpu_budget, os.cpu_count() or 1)

    kernels_per_step = 1 if coop else (8 if mixed else 4)
    resorts = (args.steps // eff_resort) if eff_resort > 0 else 0
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "particle-steps/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "mixed(f32/i64/f64)" if mixed else "f64",
        "data": "synthetic",
        "config": {"workload": desc, "particles": n, "nflavors": nf, "cells": list(p.ncell),
                   "precision": "mixed" if mixed else "fp64", "integrator": "RK4",
                   "l2": "flushed (512 MB write) before every timed step",
                   "parallelism": ("particles sharded over %d GPUs, replicated mesh, NCCL all-reduce of "
                                   "every deposit" % ws) if multi else ("replica per GPU" if ws > 1 else "1 GPU"),
                   "resort_interval": eff_resort},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": kernel,
                     "kernel_ms": stage_ms, "algorithmic_bytes_per_launch": bytes_per_launch,
                     "peak_source": peak_kind},
        "e2e": e2e,
        "cpu_baseline": cpu,
        # per step: the step kernels + the L2 flush; per re-sort: keys,
        # radix-sort histogram + scan + one pass per 8 key bits, gather
        "gpu_launches": args.steps * kernels_per_step + args.steps +
                        resorts * (4 + (int(np.ceil(np.log2(max(int(np.prod(p.ncell)), 2)))) + 7) // 8),
        "clocks": clocks,
        "wall_s": wall,
        "kernel_ms_per_step": [float(x) for x in kms.mean(axis=0)],
    }
    if args.workload == "c4" and ws == 1:
        out["adjoint"] = run_adjoint(ctx, recs, p, stream, total_ms / args.steps, int(p.nsteps), 25)
    elif args.adjoint and ws == 1 and not multi:
        # the adjoint differentiates the FP64 step: its own FP64 context
        # (the benchmark's context is released first)
        ctx.close()
        del flush
        torch.cuda.empty_cache()
        pa = api.EmuParams.from_buffer_copy(p)
        pa.precision = api.PREC_FP64
        ctx = api.Context(pa)
        ctx.set_stream(stream.cuda_stream)
        out["adjoint"] = run_adjoint(ctx, recs, pa, stream, None, args.adjoint_steps or int(p.nsteps),
                                     args.adjoint_interval)
    ctx.close()
    if rank == 0:
        print(json.dumps(out))
    if torch.distributed.is_initialized():
        torch.distributed.destroy_process_group()


def pcie_copy_rate(nbytes, nbuf, reps=10):
    """GB/s of pinned host <-> device copies of nbytes (at most 256 MB),
    nbuf copies per direction in flight: host to device alone, device to host
    alone, and both at once on separate streams (per direction), the bound of
    an end-to-end step that uploads and downloads a batch."""
    import torch
    nb = int(min(nbytes, 256 << 20))
    nbuf = max(1, min(nbuf, int(1e9 // max(nb, 1))))
    hs = [torch.empty(nb, dtype=torch.uint8).pin_memory() for _ in range(nbuf)]
    hd = [torch.empty(nb, dtype=torch.uint8).pin_memory() for _ in range(nbuf)]
    ds = [torch.empty(nb, dtype=torch.uint8, device="cuda") for _ in range(nbuf)]
    dd = [torch.empty(nb, dtype=torch.uint8, device="cuda") for _ in range(nbuf)]
    sa, sb = torch.cuda.Stream(), torch.cuda.Stream()

    def run(h2d, d2h):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            for i in range(nbuf):
                if h2d:
                    with torch.cuda.stream(sa):
                        ds[i].copy_(hs[i], non_blocking=True)
                if d2h:
                    with torch.cuda.stream(sb):
                        hd[i].copy_(dd[i], non_blocking=True)
        torch.cuda.synchronize()
        return nb * nbuf * reps / (time.perf_counter() - t0) / 1e9

    run(True, True)   # warm-up
    return {"h2d_gbs": run(True, False), "d2h_gbs": run(False, True),
            "concurrent_gbs_per_direction": run(True, True), "bytes_per_copy": nb, "copies_in_flight": nbuf}


def run_adjoint(ctx, recs, p, stream, fwd_ms_per_step, nsteps, interval):
    """Recorded forward run (checkpoints) + J + backward sweep, device time
    with CUDA events on the context's stream, against the plain forward step
    time of the same context.  Storage is reserved and every code path run
    once (a shorter recorded run) before the timed run."""
    import torch
    ctx.load_particles(recs)
    nbytes, stage_store, sub = ctx.adjoint_reserve(nsteps, interval)
    kw = min(nsteps, 2 * interval)
    ctx.adjoint_forward(kw, interval)                # warm-up: every kernel once
    J, lf, lN = ctx.adjoint_objective()
    ctx.adjoint_backward(lf, lN)
    # plain forward under the same conditions (back-to-back steps, no L2 flush)
    ctx.load_particles(recs)
    nplain = min(nsteps, 50)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.evolve(nplain)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1) / nplain
    ctx.load_particles(recs)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record(stream)
    ctx.adjoint_forward(nsteps, interval)
    ev[1].record(stream)
    J, lf, lN = ctx.adjoint_objective()
    ev[2].record(stream)
    g, gN = ctx.adjoint_backward(lf, lN)
    ev[3].record(stream)
    torch.cuda.synchronize()
    rec_ms = ev[0].elapsed_time(ev[1])
    bwd_ms = ev[2].elapsed_time(ev[3])
    return {"steps": nsteps, "checkpoint_interval": interval, "precision": "fp64", "J": J,
            "device_bytes": nbytes, "stage_states_stored": stage_store, "sub_checkpoint_interval": sub,
            "record_ms_per_step": rec_ms / nsteps, "backward_ms_per_step": bwd_ms / nsteps,
            "forward_ms_per_step": plain_ms, "forward_ms_per_step_l2_flushed": fwd_ms_per_step,
            "backward_over_forward": bwd_ms / nsteps / plain_ms,
            "record_plus_backward_over_forward": (rec_ms + bwd_ms) / nsteps / plain_ms,
            "grad_max_abs": float(np.abs(g).max()),
            "note": "record = forward run with checkpoints; backward = per segment a forward recompute "
                    "from its checkpoint (stage states stored per segment, or per step with the stages "
                    "recomputed; sub-checkpoints when memory is short), then the adjoint sweep (dt of each "
                    "step held at its recorded value)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000, help="timed steps (C2's run length by default)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="emu", choices=["emu", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c2", "c3", "c4", "c5"])
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"])
    ap.add_argument("--cells", type=int, default=None, help="smaller case of the workload (cells per side)")
    ap.add_argument("--fused", type=int, default=None, choices=[1, 2],
                    help="RK4 kernels: 1 one fused kernel per stage in a CUDA graph (default), 2 one "
                         "cooperative launch per step when it fits")
    ap.add_argument("--resort", type=int, default=None,
                    help="steps between on-device cell re-sorts (0 never; default the workload's)")
    ap.add_argument("--sharded", action="store_true",
                    help="particle-sharded path even on one GPU (a one-rank communicator)")
    ap.add_argument("--profile-steps", type=int, default=10)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--e2e-pipes", type=int, default=0,
                    help="batches in flight for the end-to-end figure (one GPU; 0 = 16 for batches under "
                         "16 MB, else 8)")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--adjoint", action="store_true",
                    help="also time the checkpointed adjoint (FP64) on this workload (always on for c4)")
    ap.add_argument("--adjoint-steps", type=int, default=None, help="recorded steps (default: the workload's)")
    ap.add_argument("--adjoint-interval", type=int, default=25, help="checkpoint interval")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_emu(args)


if __name__ == "__main__":
    main()
