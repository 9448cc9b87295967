"""Bounded device-side waits run out without faulting the GPU.

The cooperative whole-step kernel (fused = 2) separates its RK stages with a
grid barrier whose wait gives up after a number of polls and records
EMU_ERR_TIMEOUT instead of spinning forever.  With the limit set to 0 polls
every CTA but the last to arrive gives up at once: the step must finish,
report EMU_ERR_TIMEOUT, and leave the context usable; after the default
limit is restored, a fresh load and run match the oracle."""
import numpy as np
import pytest

from emu_b200 import api
from emu_b200 import workloads as W
from oracle.oracle import Oracle
from tests.helpers import colwise_rel

pytestmark = pytest.mark.gpu


def _params():
    p = W.c2_fast_flavor_1d(ncell_z=16, ndirs=20)    # 320 particles: 3 CTAs
    p.fused = 2
    p.resort_interval = 0
    return p


def test_grid_barrier_wait_runs_out_and_the_context_recovers():
    p = _params()
    parts = api.init_particles(p)
    ref, t_ref, _, _ = Oracle(p).evolve(parts, 3)
    with api.Context(p) as c:
        c.load_particles(parts)
        c.set_wait_limit(0)
        with pytest.raises(api.EmuError) as e:
            c.evolve(3)
        assert e.value.code & api.EMU_ERR_TIMEOUT
        # the default limit again: a fresh load runs clean
        c.set_wait_limit(-1)
        c.load_particles(parts)
        info = c.evolve(3)
        assert info.status == 0 and info.steps_done == 3
        assert abs(info.time - t_ref) <= 1e-12 * t_ref
        out = c.get_particles()
    assert colwise_rel(out, ref) < 1e-11
