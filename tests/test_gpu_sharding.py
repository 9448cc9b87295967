"""The sharded device path (NCCL all-reduce of every deposit, captured in
the step graph) with a one-rank communicator: the same results as the
unsharded context -- bit-identical for the mixed path's int64 mesh, within
FP64 deposit-order rounding for the plain path.  Multi-rank schedules are
covered on CPU (tests/test_sharding_cpu.py)."""
import numpy as np
import pytest

from emu_b200 import api
from emu_b200 import workloads as W
from tests.helpers import colwise_rel

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
