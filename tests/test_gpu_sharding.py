"""The sharded device path (NCCL all-reduce of every deposit, captured in
the step graph) with a one-rank communicator: the same results as the
unsharded context -- bit-identical for the mixed path's int64 mesh, within
FP64 deposit-order rounding for the plain path.

The same schedule with two and three ranks on one GPU (a local group: the
ranks are contexts of this process, each driven from its own thread, the
library's own exchange in place of NCCL's): each rank loads every nranks-th
particle; Vvac_max and the fixed-point scales are reduced over the ranks at
load and every deposit is summed over the ranks.  Against the unsharded
context: FP64 within deposit-order rounding (1e-11 after the steps); mixed
within FP32 rounding (each rank's CTAs sum different particles in FP32
before the exact int64 sum), and every rank holds the bit-identical mesh.
The algorithm of the schedule is also covered on CPU with gloo ranks
(tests/test_sharding_cpu.py)."""
import threading

import numpy as np
import pytest

from emu_b200 import api
from emu_b200 import sharding
from emu_b200 import workloads as W
from tests.helpers import colwise_rel, flavor_cols

pytestmark = pytest.mark.gpu


def _run(p, parts, nsteps, comm):
    with api.Context(p) as c:
        if comm:
            c.attach_comm(api.comm_id(), 0, 1)
        c.load_particles(parts)
        info = c.evolve(nsteps)
        return c.get_particles(), c.get_mesh(), info


@pytest.mark.parametrize("fused", [1, 2])
def test_one_rank_comm_fp64_matches_unsharded(fused):
    p = W.c2_fast_flavor_1d(ncell_z=16, ndirs=20)
    p.fused = fused
    parts = api.init_particles(p)
    a, ma, ia = _run(p, parts, 12, True)
    b, mb, ib = _run(p, parts, 12, False)
    assert ia.status == 0 and ia.steps_done == 12
    assert abs(ia.time - ib.time) <= 1e-12 * ib.time
    assert colwise_rel(a, b) < 1e-11


def test_one_rank_comm_mixed_is_bit_identical():
    p = W.c3_three_flavor_1d(ncell_z=16, nphi_equator=4)
    parts = api.init_particles(p)
    a, ma, ia = _run(p, parts, 8, True)
    b, mb, ib = _run(p, parts, 8, False)
    assert ia.time == ib.time
    assert np.array_equal(a, b)
    assert np.array_equal(ma, mb)


def test_comm_with_generic_integrator_and_errors():
    p = W.c2_fast_flavor_1d(ncell_z=8, ndirs=6)
    p.integration_type = 0   # forward Euler: unfused deposit + RHS
    parts = api.init_particles(p)
    outs = []
    for comm in (True, False):
        with api.Context(p) as c:
            if comm:
                c.attach_comm(api.comm_id(), 0, 1)
            c.load_particles(parts)
            dt, _ = c.compute_dt()
            for _ in range(3):
                c.step(dt)
            outs.append(c.get_particles())
    assert colwise_rel(outs[0], outs[1]) < 1e-12
    with api.Context(p) as c:
        c.load_particles(parts)
        with pytest.raises(api.EmuError):
            c.attach_comm(api.comm_id(), 0, 1)    # after load
    q = W.c2_fast_flavor_1d(ncell_z=8, ndirs=6)
    with api.Context(q) as c:
        c.attach_comm(api.comm_id(), 0, 1)
        c.load_particles(api.init_particles(q))
        with pytest.raises(api.EmuError):
            c.adjoint_forward(2, 1)               # the adjoint runs on one GPU


def _local_ranks(p, parts, nranks, nsteps):
    """run the sharded schedule with nranks local ranks; (records in global
    order, the ranks' meshes, the ranks' run infos)"""
    group = api.LocalGroup(nranks)
    ctxs = [api.Context(p) for _ in range(nranks)]
    out = [None] * nranks
    errors = []
    try:
        for r, c in enumerate(ctxs):
            c.attach_local(group, r)

        def rank(r):
            try:
                c = ctxs[r]
                c.load_particles(sharding.shard(parts, r, nranks))
                info = c.evolve(nsteps)
                out[r] = (c.get_particles(), c.get_mesh(), info)
            except Exception as e:     # reported after the join
                errors.append(e)

        threads = [threading.Thread(target=rank, args=(r,)) for r in range(nranks)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    finally:
        for c in ctxs:
            c.close()
        group.close()
    assert not errors, errors
    return sharding.unshard([o[0] for o in out]), [o[1] for o in out], [o[2] for o in out]


@pytest.mark.parametrize("nranks", [2, 3])
@pytest.mark.parametrize("case", ["fp64_1d", "fp64_3d", "mixed_1d", "mixed_3d"])
def test_local_ranks_match_the_unsharded_context(case, nranks):
    if case == "fp64_1d":
        p = W.c2_fast_flavor_1d(ncell_z=16, ndirs=20)
    elif case == "fp64_3d":
        p = W.c5_3d(n=4, ndirs=6, mixed=False)
    elif case == "mixed_1d":
        p = W.c3_three_flavor_1d(ncell_z=16, nphi_equator=4)
    else:
        p = W.c5_3d(n=4, ndirs=6, mixed=True)
    parts = api.init_particles(p)
    nsteps = 6
    ref, mref, iref = _run(p, parts, nsteps, False)
    out, meshes, infos = _local_ranks(p, parts, nranks, nsteps)
    for info in infos:
        assert info.status == 0 and info.steps_done == nsteps
    # every rank holds the same mesh and takes the same steps
    for m, info in zip(meshes[1:], infos[1:]):
        assert np.array_equal(m, meshes[0])
        assert info.time == infos[0].time
    fc = flavor_cols(p.nflavors)
    if p.precision == api.PREC_FP64:
        assert abs(infos[0].time - iref.time) <= 1e-12 * iref.time
        assert colwise_rel(out, ref) < 1e-11
    else:
        assert abs(infos[0].time - iref.time) <= 1e-6 * iref.time
        assert colwise_rel(out[:, fc], ref[:, fc]) < 1e-5
        assert colwise_rel(out[:, :13], ref[:, :13]) < 1e-6
