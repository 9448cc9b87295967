"""Rank body of the gloo multi-process tests (tests/test_sharding_cpu.py):
the sharded algorithm (per-rank deposit, all-reduce, per-rank
interpolation and RK4) run with the oracle on each rank's particles."""
import os

import numpy as np
import torch
import torch.distributed as dist

from emu_b200 import api, sharding
from emu_b200 import workloads as W
from oracle.oracle import Oracle

A = (0.5, 0.5, 1.0)
B = (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0)


def _allreduce(x, op=dist.ReduceOp.SUM):
    t = torch.from_numpy(np.ascontiguousarray(x))
    dist.all_reduce(t, op=op)
    return t.numpy()


def sharded_rk4_step(o, parts, dt):
    """one RK4 step of this rank's particles with a replicated mesh:
    deposit(local) -> all-reduce -> interpolate(local), positions frozen
    during the stages, then wrap + Renormalize (main.cpp:129-203)"""
    Ks = []
    Y = parts.copy()
    for s in range(4):
        if s > 0:
            Y = parts.copy()
            Y[:, 3:] = parts[:, 3:] + (A[s - 1] * dt) * Ks[-1][:, 3:]
        mesh = _allreduce(o.deposit(Y))
        Ks.append(o.interpolate_rhs(mesh, Y))
    new = parts.copy()
    new[:, 3:] = parts[:, 3:] + dt * sum(b * K[:, 3:] for b, K in zip(B, Ks))
    return new, mesh


def run(rank, nranks, port, outdir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=nranks)
    try:
        p = W.c2_fast_flavor_1d(ncell_z=8, ndirs=6)
        full = api.init_particles(p)
        mine = sharding.shard(full, rank, nranks)
        o = Oracle(p)
        # replicated mesh = full deposit
        mesh = _allreduce(o.deposit(mine))
        ref = o.deposit(full)
        np.save(os.path.join(outdir, "mesh_%d.npy" % rank), np.stack([mesh, ref]))
        # global scalars
        vmax = _allreduce(np.array([o.vvac_max(mine)]), dist.ReduceOp.MAX)[0]
        np.save(os.path.join(outdir, "vmax_%d.npy" % rank), np.array([vmax, o.vvac_max(full)]))
        # two sharded RK4 steps (the oracle's wrap + Renormalize on the
        # local particles after each), gathered, against the oracle's step
        dt = 0.5 * o.compute_dt(ref, o.vvac_max(full))[0]
        q = mine.copy()
        for _ in range(2):
            q, _ = sharded_rk4_step(o, q, dt)
            o.finish_step(q)
        got = sharding.gather_records(q, rank, nranks)
        if rank == 0:
            want = full.copy()
            for _ in range(2):
                o.rk_step(want, dt)
            np.save(os.path.join(outdir, "step.npy"), np.stack([got, want]))
    finally:
        dist.destroy_process_group()
