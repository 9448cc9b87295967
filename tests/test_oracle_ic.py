"""The host-only benchmark legs build their workloads without the CUDA
library: the parameter defaults set in Python (emu_b200.api.default_params)
and the numpy restatement of the initial particle generator
(oracle/ic.py) must equal the library's emu_params_default and
emu_init_particles bit for bit on the benchmark workloads' shapes."""
import numpy as np
import pytest

from emu_b200 import api
from emu_b200 import workloads as W
from oracle import ic


def test_python_defaults_equal_library_defaults():
    assert bytes(api.default_params()) == bytes(api.library_default_params())


def _cases():
    return [("c2_shape", W.c2_fast_flavor_1d(ncell_z=16)),
            ("c3_shape_ring_directions", W.c3_three_flavor_1d(ncell_z=8)),
            ("c5_shape", W.c5_3d(n=5)),
            ("c5_other_seed", W.c5_3d(n=3, ndirs=17, seed=12345)),
            ("two_flavor_3d_ring", W.c5_3d(n=2, ndirs=1)),
            ]


@pytest.mark.parametrize("name,p", _cases(), ids=[c[0] for c in _cases()])
def test_initial_records_bit_identical(name, p):
    if name == "two_flavor_3d_ring":
        p.nflavors = 2
        p.direction_generator = 0
        p.nphi_equator = 7
        p.nppc[0], p.nppc[2] = 2, 3
    a = ic.init_particles(p)
    b = api.init_particles(p)
    assert a.shape == b.shape
    assert np.array_equal(a, b)


def test_ring_directions_counts():
    # nphi_equator = 1 gives the two poles; 32 gives the 378 directions of C3
    assert ic.uniform_sphere_xyz(1).shape[0] == 2
    assert ic.uniform_sphere_xyz(32).shape[0] == 378
