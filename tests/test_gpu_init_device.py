"""InitParticles on the device against the host generator: the same
records (bit-identical where no sin/exp is evaluated), the same loaded
state, and the shard of a rank when a communicator is attached."""
import numpy as np
import pytest

from emu_b200 import api, sharding
from emu_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _cases():
    return [("msw", W.ci_msw(), True), ("bipolar", W.ci_bipolar(), True), ("two_beam", W.ci_fast_flavor(), True),
            ("k_test", W.ci_fast_flavor_k(), False), ("c2", W.c2_fast_flavor_1d(ncell_z=16, ndirs=10), True),
            ("c3_mixed", W.c3_three_flavor_1d(ncell_z=8, nphi_equator=4), True),
            ("c5", W.c5_3d(n=4, ndirs=6, mixed=False), True)]


@pytest.mark.parametrize("name,p,exact", _cases(), ids=[c[0] for c in _cases()])
def test_device_initial_conditions_match_host(name, p, exact):
    host = api.init_particles(p)
    with api.Context(p) as c:
        c.init_particles_device()
        dev = c.get_particles()
        dt_dev, _ = c.compute_dt()
    with api.Context(p) as c:
        c.load_particles(host)
        ref = c.get_particles()
        dt_host, _ = c.compute_dt()
    assert dev.shape == host.shape
    if exact:
        assert np.array_equal(dev, ref)
        assert dt_dev == dt_host
    else:
        assert np.abs(dev - ref).max() <= 1e-15 * np.abs(ref).max()
        assert abs(dt_dev - dt_host) <= 1e-14 * dt_host


def test_device_initial_conditions_shard():
    """one-rank communicator: the whole set; the shard selection itself
    (every nranks-th index) is the host function sharding.shard"""
    p = W.c2_fast_flavor_1d(ncell_z=8, ndirs=6)
    host = api.init_particles(p)
    with api.Context(p) as c:
        c.attach_comm(api.comm_id(), 0, 1)
        c.init_particles_device()
        dev = c.get_particles()
    assert np.array_equal(dev, sharding.shard(host, 0, 1))
