"""Particle sharding over GPUs (one process per GPU), with torch.distributed
only as the plumbing that hands the NCCL communicator id to every rank.

Each rank owns a disjoint, strided subset of the particles (every nranks-th
record, so every rank has particles in every cell) and a full copy of the
mesh; the library sums every deposit over the ranks before a stage reads it
(include/emu_b200.h, emu_attach_comm).
"""
import numpy as np

from . import api


def shard(records, rank, nranks):
    """the records rank `rank` of `nranks` owns"""
    return np.ascontiguousarray(records[rank::nranks])


def unshard(shards):
    """inverse of shard(): interleave the per-rank record blocks"""
    nranks = len(shards)
    n = sum(s.shape[0] for s in shards)
    out = np.empty((n, shards[0].shape[1]), dtype=shards[0].dtype)
    for r, s in enumerate(shards):
        out[r::nranks] = s
    return out


def attach(ctx, rank, nranks):
    """attach ctx to a communicator over the torch.distributed world (call on
    every rank, before load_particles)"""
    import torch.distributed as dist
    obj = [api.comm_id() if rank == 0 else None]
    dist.broadcast_object_list(obj, src=0)
    ctx.attach_comm(obj[0], rank, nranks)


def gather_records(local, rank, nranks):
    """all ranks' records in global order (torch.distributed all_gather)"""
    import torch.distributed as dist
    parts = [None] * nranks
    dist.all_gather_object(parts, local)
    return unshard(parts)
