"""Benchmark: particle RK4 steps/s of Emu's evolution path on B200, mixed
precision against the plain FP64 path of the same code, with the error of
the flavor-conversion observables between them.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl emu|reference]
                    [--workload c5|c3|c2|c4] [--precision mixed|fp64]

A step is one RK4 step (4 stages: deposit, interpolate, -i[H,rho], stage
update; then wrap, Renormalize, compute_dt and the cell re-sort on the
device) over every particle of the workload.  Default workload: C5, the 3D
scale case (3 flavors, 64^3 periodic cells x 96 Fibonacci directions =
25,165,824 particles, 27-cell TSC stencils), mixed precision; the same
initial particles are then run through the FP64 path (`fp64` keys) and the
observables of both runs after the same steps are compared (`mixed_vs_fp64`).
Inputs are synthetic (seeded initial conditions, no datasets exist).

Timing: W untimed warm-up steps, then K steps between CUDA events on the
launching stream, max over ranks.  Workloads whose particle state exceeds
the 126 MB L2 (C3, C5) run the K steps back to back; smaller ones (C2, C4)
flush L2 (512 MB write) before every step and time each step alone.

With N > 1 (torchrun, or `--gpus N`, which re-launches itself under
torchrun) the particles of N times the directions are sharded over the
ranks (every rank keeps the single-GPU particle count: weak scaling) and
every deposit is summed over the ranks by an NCCL all-reduce.

--impl reference times the reference's per-particle arithmetic on the host
cores (oracle/_ref: Emu's generated kernel bodies in the restated AMReX
loops; the oracle port when _ref is absent) on a bounded sample of the same
workload; it never loads the CUDA library.
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

# (api and workloads are plain Python: the CUDA library is loaded only by the
# emu arm's first device call)
from emu_b200 import api  # noqa: E402
from emu_b200 import workloads as W  # noqa: E402

METRIC = "particle RK4 steps/s on 1 B200: mixed vs FP64 at stated err; % of HBM peak"
L2_BYTES = 126 << 20


def default_precision(name):
    return "mixed" if name in ("c3", "c5") else "fp64"


def workload(name, precision, cells=None, fused=None, resort=None, ranks=1):
    """EmuParams and a description.  cells overrides the cell count (z cells
    for c2/c3, cells per side for c5) to run a smaller case of the same
    workload (profiling, CPU samples).  With ranks > 1 every cell gets ranks
    times the directions, so that each rank's shard (every ranks-th particle)
    has the single-GPU particle count."""
    precision = precision or default_precision(name)
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
        desc = "C5 3-flavor 3D: %d^3 cells x %d Fibonacci directions, TSC" % (p.ncell[0], 96 * ranks)
    else:
        raise SystemExit("unknown workload " + name)
    p.precision = api.PREC_MIXED if precision == "mixed" else api.PREC_FP64
    if fused:
        p.fused = fused
    if resort is not None:
        p.resort_interval = resort
    return p, desc


def n_particles(p):
    return (p.ncell[0] * p.ncell[1] * p.ncell[2] * p.nppc[0] * p.nppc[1] * p.nppc[2] *
            (p.ndirections if p.direction_generator == 1 else _ring_count(p.nphi_equator)))


def _ring_count(nphi):
    from oracle import ic
    return ic.uniform_sphere_xyz(nphi).shape[0]


def config_dict(name, p, desc, ws, multi, eff_resort):
    """The `config` object of both arms."""
    return {"workload": desc, "particles": n_particles(p), "nflavors": p.nflavors, "cells": list(p.ncell),
            "precision": "mixed" if p.precision == api.PREC_MIXED else "fp64", "integrator": "RK4",
            "shape_order": p.shape_order,
            "l2": ("inputs larger than L2 (%.1f GB of particle state), steps back to back"
                   % (n_particles(p) * api.nreal(p.nflavors) * 8 / 1e9)) if large_state(p)
            else "flushed (512 MB write) before every timed step",
            "parallelism": ("particles sharded over %d GPUs, replicated mesh, NCCL all-reduce of every deposit"
                            % ws) if multi else "1 GPU",
            "resort_interval": eff_resort}


def large_state(p):
    return n_particles(p) * api.nreal(p.nflavors) * 8 > 2 * L2_BYTES


def effective_resort(p):
    r = p.resort_interval
    if r < 0:
        r = 1 if sum(1 for c in p.ncell if c > 1) == 3 and p.shape_order >= 2 else 16
    return r


def cpu_sample(name):
    """The bounded sample of a workload that the host-core legs run: the
    whole workload where one step takes a fraction of a second on the host
    (C2, C3, C4); for C5 a periodic 12^3-cell box with the same cell size,
    directions and physics (165,888 particles: the same per-particle work,
    27-cell stencils, 3 flavors)."""
    if name == "c5":
        p, _ = workload("c5", "fp64", cells=12)
        return p, "a periodic 12^3-cell box of the C5 workload (same cell size, 96 directions, 165,888 particles)"
    p, _ = workload(name, "fp64")
    return p, "the full workload"


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
        return d.get("hbm_gbs", 6650.0), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons of one GPU, sampled every
    100 ms between start() and stop()."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        self.gpu = vis.split(",")[local_rank].strip() if vis else str(local_rank)
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu, "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # the first sample is written before the timed region starts
        t0 = time.time()
        while time.time() - t0 < 5.0 and os.path.getsize(self.f.name) == 0:
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [v for v in (num(r[1]) for r in rows) if v is not None]
        mx = [v for v in (num(r[2]) for r in rows) if v is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for i, n in enumerate(names):
                if r[5 + i].strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def observable_sums(parts, nf):
    """Partial sums of the flavor-conversion observables over a particle
    set: sum |rho_emu| (neutrinos), sum |rho_emu| (antineutrinos), the
    N-weighted sums of Re and Im rho_emu, and the particle count."""
    nh = nf * nf
    f01 = 3 + 11
    fb01 = 3 + 12 + nh + 1
    N = parts[:, 3 + 8]
    return np.array([np.hypot(parts[:, f01], parts[:, f01 + 1]).sum(),
                     np.hypot(parts[:, fb01], parts[:, fb01 + 1]).sum(),
                     (parts[:, f01] * N).sum(), (parts[:, f01 + 1] * N).sum(), float(parts.shape[0])])


def observables(sums):
    """mean |rho_emu| of the neutrinos and of the antineutrinos, and |N_emu|
    of the whole domain (the N-weighted sum of rho_emu over particles)"""
    return {"mean_abs_rho_emu": float(sums[0] / sums[4]), "mean_abs_rho_emu_bar": float(sums[1] / sums[4]),
            "domain_abs_N_emu": float(np.hypot(sums[2], sums[3]))}


def sum_over_ranks(v, ws):
    import torch
    if ws == 1:
        return v
    t = torch.tensor(v, dtype=torch.float64, device="cuda")
    torch.distributed.all_reduce(t)
    return t.cpu().numpy()


def cpu_run(p, recs, steps, warmup, budget_s, nthreads):
    """The reference arithmetic on host cores: warm-up steps, then up to
    `steps` RK4 steps of the sample (or until budget_s); (particle-steps/s,
    steps, seconds, kind)."""
    from oracle.oracle import Oracle, RefHarness, have_ref
    kind = "reference" if have_ref(p.nflavors) else "port"
    o = RefHarness(p) if kind == "reference" else Oracle(p)
    parts = np.array(recs, copy=True)
    vmax = o.vvac_max(parts)
    mesh = o.deposit(parts, nthreads)
    dt, _ = o.compute_dt(mesh, vmax)
    for _ in range(warmup):
        mesh, _, _ = o.rk_step(parts, dt, nthreads=nthreads)
        dt, _ = o.compute_dt(mesh, vmax)
    done = 0
    t0 = time.perf_counter()
    while done < steps:
        mesh, _, _ = o.rk_step(parts, dt, nthreads=nthreads)
        dt, _ = o.compute_dt(mesh, vmax)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return len(parts) * done / el, done, el, kind


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference(args):
    """--impl reference: rank 0 times the reference's CPU arithmetic on a
    bounded sample of the emu arm's workload, with every host core."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    multi = ws > 1 and args.workload != "c4"
    p, desc = workload(args.workload, args.precision, args.cells, args.fused, args.resort, ws if multi else 1)
    sp, sdesc = cpu_sample(args.workload)
    from oracle import ic
    recs = ic.init_particles(sp)
    nthreads = os.cpu_count() or 1
    value, done, el, kind = cpu_run(sp, recs, args.steps, args.warmup, args.cpu_budget_ref, nthreads)
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "particle-steps/s",
           "n_gpus": ws, "steps": done, "warmup": args.warmup, "ms_per_step": el / done * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic",
           "config": config_dict(args.workload, p, desc, ws, multi, effective_resort(p)),
           "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": nthreads, "kind": kind,
                            "sample": "%d RK4 steps (after %d warm-up) of %s, FP64, %.1f s" % (
                                done, args.warmup, sdesc, el)},
           "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "note": "the reference's CPU path (its generated kernel bodies in restated AMReX loops, FP64, "
                   "OpenMP over particles) on the host cores; ms_per_step is for the sample"}
    print(json.dumps(out), flush=True)


class Timed:
    """K device steps of a context between CUDA events on its stream: back
    to back for large states, each after an L2 flush otherwise."""

    def __init__(self, ctx, stream, flush):
        self.ctx, self.stream, self.flush = ctx, stream, flush

    def warm(self, w):
        for _ in range(w):
            if self.flush is not None:
                self.ctx.flush_l2(self.flush.data_ptr(), self.flush.numel() * 8)
            self.ctx.evolve_steps(1)
        self.ctx.synchronize()

    def run(self, k):
        import torch
        if self.flush is None:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(self.stream)
            self.ctx.evolve_steps(k)
            b.record(self.stream)
            b.synchronize()
            return a.elapsed_time(b)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        for i in range(k):
            self.ctx.flush_l2(self.flush.data_ptr(), self.flush.numel() * 8)
            evs[i][0].record(self.stream)
            self.ctx.evolve_steps(1)
            evs[i][1].record(self.stream)
        evs[-1][1].synchronize()
        return sum(x.elapsed_time(y) for x, y in evs)


def max_over_ranks(v, ws):
    import torch
    if ws == 1:
        return v
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    import torch
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()


def make_context(p, stream, multi, rank, ws):
    from emu_b200 import sharding
    ctx = api.Context(p)
    ctx.set_stream(stream.cuda_stream)
    if multi:
        sharding.attach(ctx, rank, ws)
    return ctx


def run_emu(args):
    import torch
    ws, rank, local = dist_env()
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
    all_recs = api.init_particles(p)
    recs = all_recs
    if multi:
        from emu_b200 import sharding
        recs = sharding.shard(all_recs, rank, ws)
    n = recs.shape[0]
    eff_resort = effective_resort(p)
    stream = torch.cuda.Stream()
    flush = None if large_state(p) else torch.zeros((512 << 20) // 8, dtype=torch.float64, device="cuda")
    ctx = make_context(p, stream, multi, rank, ws)
    ctx.load_particles(recs)
    total_steps = args.warmup + args.steps + args.profile_steps + 8
    ctx.evolve_begin(0.0, float("inf"), total_steps)
    T = Timed(ctx, stream, flush)
    T.warm(args.warmup)
    sampler = ClockSampler(local)
    sampler.start()
    barrier(ws)
    wall0 = time.perf_counter()
    total_ms = T.run(args.steps)
    barrier(ws)
    wall = time.perf_counter() - wall0
    clocks = sampler.stop()
    total_ms = max_over_ranks(total_ms, ws)
    info = ctx.evolve_end()
    if info.status != 0:
        raise SystemExit("device status %d during the benchmark: %s" % (info.status, api.last_error(ctx.h)))
    value = n * args.steps * ws / (total_ms * 1e-3)
    ms_per_step = total_ms / args.steps
    sums_mixed = observable_sums(ctx.get_particles(), nf) if (mixed and not args.no_fp64) else None
    t_mixed = info.time

    # per-kernel CUDA events of separately launched steps, attributed to the
    # graph-timed step in proportion (the graph's programmatic launches
    # overlap a kernel's prologue with its predecessor's tail)
    ctx.evolve_begin(t_mixed, float("inf"), args.profile_steps + 2)
    kms = []
    for _ in range(args.profile_steps):
        if flush is not None:
            ctx.flush_l2(flush.data_ptr(), flush.numel() * 8)
        kms.append(ctx.profile_step())
    ctx.evolve_end()
    width = max(len(k) for k in kms)
    kms = np.array([k + [0.0] * (width - len(k)) for k in kms])
    per_kernel = kms.mean(axis=0)
    serial_step = float(per_kernel.sum())
    scale = min(1.0, ms_per_step / serial_step) if serial_step > 0 else 1.0
    per_pstep = algorithmic_bytes_per_particle_step(nf, mixed)
    coop = kms.shape[1] == 1
    split = nf == 2 and p.ncell[0] == 1 and p.ncell[1] == 1 and not mixed   # species-split kernels
    if coop:
        kernel = "k_rk4_step_coop%s<%d>" % ("_split" if split else "", nf)
        stage_serial = float(kms[:, 0].mean())
        bytes_per_launch = per_pstep * n + mesh_bytes_per_step(p, nf)
    else:
        kernel = "k_rk4_stage%s<%d>" % ("_mixed" if mixed else ("_split" if split else ""), nf)
        stage_idx = [1, 3, 5, 7] if mixed else [0, 1, 2, 3]
        stage_serial = float(kms[:, stage_idx].mean())
        bytes_per_launch = (per_pstep * n + mesh_bytes_per_step(p, nf)) / 4.0
    stage_ms = stage_serial * scale
    peak, peak_kind = load_peaks()
    achieved = bytes_per_launch / (stage_ms * 1e-3) / 1e9
    step_bytes = per_pstep * n + mesh_bytes_per_step(p, nf)
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_%s_%s.json" % (args.workload, "mixed" if mixed else "fp64"))
    if os.path.exists(tpath) and args.cells is None and not multi:
        with open(tpath) as f:
            tj = json.load(f)
        if tj.get("kernel", "").split("<")[0] == kernel.split("<")[0]:
            traffic = tj.get("bytes_per_launch")

    # the FP64 path of the same code on the same particles and steps
    fp64 = None
    if mixed and not args.no_fp64:
        pd = api.EmuParams.from_buffer_copy(p)
        pd.precision = api.PREC_FP64
        cd = make_context(pd, stream, multi, rank, ws)
        cd.load_particles(recs)
        cd.evolve_begin(0.0, float("inf"), args.warmup + args.steps + 2)
        Td = Timed(cd, stream, flush)
        Td.warm(args.warmup)
        barrier(ws)
        d_ms = max_over_ranks(Td.run(args.steps), ws)
        barrier(ws)
        dinfo = cd.evolve_end()
        if dinfo.status != 0:
            raise SystemExit("device status %d in the FP64 run: %s" % (dinfo.status, api.last_error(cd.h)))
        sums_fp64 = observable_sums(cd.get_particles(), nf)
        cd.close()
        om = observables(sum_over_ranks(sums_mixed, ws))
        od = observables(sum_over_ranks(sums_fp64, ws))
        err = {k: abs(om[k] - od[k]) / abs(od[k]) for k in od}
        err["time"] = abs(t_mixed - dinfo.time) / dinfo.time
        fp64 = {"value": n * args.steps * ws / (d_ms * 1e-3), "ms_per_step": d_ms / args.steps,
                "mixed_over_fp64": (d_ms / args.steps) / ms_per_step,
                "mixed_vs_fp64": {"after_steps": args.warmup + args.steps, "relative_error": err,
                                  "fp64": od, "mixed": om,
                                  "note": "same initial particles and step count; each run takes its dt from its "
                                          "own stage-4 mesh (compute_dt), so the times differ by 'time'"}}

    # end to end through the C ABI with host buffers, one batch: every step
    # uploads the particle records from pinned host memory, deposits and
    # computes dt (emu_evolve_begin), runs one device step and downloads the
    # records into pinned host memory
    e2e = None
    if not args.no_e2e:
        pin_in = torch.from_numpy(recs).pin_memory()
        pin_out = torch.empty_like(pin_in).pin_memory()

        def e2e_step():
            ctx.load_particles_ptr(pin_in.data_ptr(), n)
            ctx.evolve_begin(0.0, float("inf"), 1)
            ctx.evolve_steps(1)
            ctx.get_particles_ptr(pin_out.data_ptr(), n)

        for _ in range(2):      # untimed: graphs and buffers
            e2e_step()
        barrier(ws)
        ne = max(1, min(args.steps, args.e2e_steps))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(ne):
            e2e_step()
        b.record(stream)
        b.synchronize()
        el = max_over_ranks(a.elapsed_time(b) * 1e-3, ws)
        bytes_rec = n * api.nreal(nf) * 8
        e2e = {"value": n * ne * ws / el, "unit": "particle-steps/s", "h2d_bytes_per_step": bytes_rec,
               "d2h_bytes_per_step": bytes_rec, "steps": ne, "batches_in_flight": 1,
               "note": "per step: emu_load_particles from pinned host memory (records of the whole workload), "
                       "emu_evolve_begin (deposit + compute_dt), one device RK4 step, emu_get_particles to "
                       "pinned host memory; CUDA events on the context stream around the steps"}
        # its bound: the step's upload and download at the measured copy rates
        pc = pcie_copy_rate(bytes_rec)
        pc["bound_s_per_step"] = bytes_rec / 1e9 / pc["h2d_gbs"] + bytes_rec / 1e9 / pc["d2h_gbs"]
        pc["frac"] = pc["bound_s_per_step"] / (el / ne)
        e2e["pcie"] = pc
        del pin_in, pin_out

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        sp, sdesc = cpu_sample(args.workload)
        from oracle import ic
        v, done, el, kind = cpu_run(sp, ic.init_particles(sp), 1 << 30, 1, args.cpu_budget, os.cpu_count() or 1)
        cpu = {"value": v, "unit": "particle-steps/s", "cores": os.cpu_count() or 1, "kind": kind,
               "sample": "%d RK4 steps of %s, FP64, %.1f s" % (done, sdesc, el)}

    kernels_per_step = 1 if coop else (8 if mixed else 4)
    widths = [1 if c <= 1 else (3 if p.shape_order >= 2 else (2 if p.shape_order == 1 else 1)) for c in p.ncell]
    resorts = (args.steps // eff_resort) if eff_resort > 0 else 0
    key_bits = int(np.ceil(np.log2(max(int(np.prod(list(p.ncell))) + 1, 2))))
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "particle-steps/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "mixed(f32/i64/f64)" if mixed else "f64",
        "data": "synthetic (seeded initial conditions of the workload's shape)",
        "config": config_dict(args.workload, p, desc, ws, multi, eff_resort),
        "fp64": fp64,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": kernel,
                     "kernel_ms": stage_ms, "kernel_ms_serial": stage_serial,
                     "algorithmic_bytes_per_launch": bytes_per_launch, "peak_source": peak_kind,
                     "step": {"algorithmic_bytes": step_bytes, "achieved": step_bytes / (ms_per_step * 1e-3) / 1e9,
                              "frac": step_bytes / (ms_per_step * 1e-3) / 1e9 / peak},
                     "note": "kernel_ms: per-kernel CUDA events of separately launched steps "
                             "(kernel_ms_serial) scaled by the graph-timed step over the sum of the "
                             "separately timed kernels (%.3f); algorithmic bytes %d per particle-step "
                             "plus the mesh term, a quarter per stage launch" % (scale, per_pstep)},
        "e2e": e2e,
        "cpu_baseline": cpu,
        # per step: the step kernels (+ the L2 flush for small states); per
        # re-sort: radix sort (histogram, scan, one pass per 8 key bits),
        # the keys (a kernel of their own unless stage 3 of a mixed step
        # with 3D stencils stores them) and the gather (FP64), or the
        # inversion of the permutation and the deposit of the sorted state
        # (mixed: stage 4 stores the state in cell order); per
        # emu_evolve_steps call of the mixed path: the stage-4 mesh control
        "gpu_launches": args.steps * kernels_per_step + (args.steps if flush is not None else 0) +
                        resorts * (4 + (key_bits + 7) // 8 + (1 if mixed and widths == [1, 1, 3] else 0)) +
                        ((args.steps if flush is not None else 1) if mixed else 0),
        "clocks": clocks,
        "wall_s": wall,
        "kernel_ms_per_step": [float(x) for x in per_kernel],
    }
    if mixed:
        out["path"] = ("mixed precision: FP32 interpolation and right-hand side (one FP32 commutator per species, "
                       "the vacuum + matter Hamiltonian rounded in), FP64 state accumulation and renormalisation, "
                       "int64 fixed-point deposits in the combined self-interaction layout; inside one "
                       "emu_evolve_steps call the stage-4 mesh keeps the combined layout and the diagonal N_ii "
                       "that compute_dt reads, and the call's last step deposits it in full (the mesh a caller "
                       "reads); results do not depend on how a run is split into calls")
    if args.workload == "c4" and ws == 1:
        out["adjoint"] = run_adjoint(ctx, recs, p, stream, ms_per_step, int(p.nsteps), 25)
    elif args.adjoint and ws == 1 and not multi:
        # the adjoint differentiates the FP64 step: its own FP64 context
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
        print(json.dumps(out), flush=True)
    if torch.distributed.is_initialized():
        torch.distributed.destroy_process_group()


def pcie_copy_rate(nbytes, reps=4):
    """GB/s of pinned host <-> device copies of one batch (at most 1 GB):
    host to device, device to host, one direction at a time."""
    import torch
    nb = int(min(nbytes, 1 << 30))
    h = torch.empty(nb, dtype=torch.uint8).pin_memory()
    d = torch.empty(nb, dtype=torch.uint8, device="cuda")

    def run(h2d):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            if h2d:
                d.copy_(h, non_blocking=True)
            else:
                h.copy_(d, non_blocking=True)
        torch.cuda.synchronize()
        return nb * reps / (time.perf_counter() - t0) / 1e9

    run(True)
    return {"h2d_gbs": run(True), "d2h_gbs": run(False), "bytes_per_copy": nb}


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


def relaunch_under_torchrun(args):
    """`--gpus N` without a torchrun environment: run this command as N
    ranks (one per GPU) under torch.distributed.run on 127.0.0.1."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="emu", choices=["emu", "reference"])
    ap.add_argument("--workload", default="c5", choices=["c2", "c3", "c4", "c5"])
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"],
                    help="default: mixed for c3 and c5, fp64 for c2 and c4")
    ap.add_argument("--cells", type=int, default=None, help="smaller case of the workload (cells per side)")
    ap.add_argument("--fused", type=int, default=None, choices=[1, 2],
                    help="RK4 kernels: 1 one fused kernel per stage in a CUDA graph (default), 2 one "
                         "cooperative launch per step when it fits")
    ap.add_argument("--resort", type=int, default=None,
                    help="steps between on-device cell re-sorts (0 never; default the workload's)")
    ap.add_argument("--sharded", action="store_true",
                    help="particle-sharded path even on one GPU (a one-rank communicator)")
    ap.add_argument("--profile-steps", type=int, default=4)
    ap.add_argument("--e2e-steps", type=int, default=6)
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of the emu arm's cpu_baseline")
    ap.add_argument("--cpu-budget-ref", type=float, default=150.0,
                    help="at most this many seconds of timed steps in the reference arm")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 run of a mixed workload")
    ap.add_argument("--adjoint", action="store_true",
                    help="also time the checkpointed adjoint (FP64) on this workload (always on for c4)")
    ap.add_argument("--adjoint-steps", type=int, default=None, help="recorded steps (default: the workload's)")
    ap.add_argument("--adjoint-interval", type=int, default=25, help="checkpoint interval")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch_under_torchrun(args))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_emu(args)


if __name__ == "__main__":
    main()
