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


# ---- the library's initial conditions against the reference's own helpers --
from oracle.oracle import RefInit, have_ref_init  # noqa: E402

needs_ref_init = pytest.mark.skipif(not have_ref_init(), reason="oracle/_ref/libemurefinit.so not built")


@needs_ref_init
@pytest.mark.parametrize("nphi", [1, 2, 3, 5, 8, 16, 32])
def test_ring_directions_equal_the_references(nphi):
    """uniform_sphere_xyz (FlavoredNeutrinoContainerInit.cpp:9-37): the
    restatement and the library's records carry the reference's directions
    bit for bit (momentum = direction x pupt)"""
    ref = RefInit().uniform_sphere_xyz(nphi)
    assert np.array_equal(ic.uniform_sphere_xyz(nphi), ref)
    p = W.c3_three_flavor_1d(ncell_z=1, nphi_equator=nphi)
    rec = api.init_particles(p)
    assert rec.shape[0] == ref.shape[0]
    pupt = rec[:, 3 + 7]
    assert np.array_equal(rec[:, 3 + 4:3 + 7], ref * pupt[:, None])


@needs_ref_init
@pytest.mark.parametrize("nf", [2, 3])
def test_minerbo_initial_conditions_equal_the_references(nf):
    """simulation type 5 (FlavoredNeutrinoContainerInit.cpp:574-645): the
    library's N, Nbar and diagonal flavor fractions equal those built from
    the reference's minerbo_Z and minerbo_closure (flux factors above and
    below the closure's 1e-3 small-flux branch)"""
    R = RefInit()
    p = api.default_params(nflavors=nf, simulation_type=5, ncell=(1, 1, 2), Lx=1.0, Ly=1.0, Lz=2.0,
                           nphi_equator=6, st5_nnue=4e32, st5_nnua=3e32, st5_nnux=2e32, st5_fxnue=0.1,
                           st5_fynue=0.2, st5_fznue=0.3, st5_fxnua=0.0, st5_fynua=-0.4, st5_fznua=0.25,
                           st5_fxnux=0.0002, st5_fynux=0.0, st5_fznux=0.0003, st5_amplitude=1e-6)
    rec = api.init_particles(p)
    F = {"e": (p.st5_fxnue, p.st5_fynue, p.st5_fznue), "a": (p.st5_fxnua, p.st5_fynua, p.st5_fznua),
         "x": (p.st5_fxnux, p.st5_fynux, p.st5_fznux)}
    n = {"e": p.st5_nnue, "a": p.st5_nnua, "x": p.st5_nnux}
    dirs = R.uniform_sphere_xyz(p.nphi_equator)
    scale_fac = 1.0 * 1.0 * 1.0 / 1 / dirs.shape[0]
    ff = {k: np.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) for k, v in F.items()}
    Z = {k: R.minerbo_Z(ff[k]) for k in F}
    assert ff["x"] < 1e-3 < ff["e"]
    nh = nf * nf
    for i, r in enumerate(rec):
        u = dirs[i % dirs.shape[0]]
        Ns = {}
        for k in F:
            mu = (F[k][0] * u[0] + F[k][1] * u[1] + F[k][2] * u[2]) / ff[k] if ff[k] > 0 else 0
            Ns[k] = n[k] * scale_fac * R.minerbo_closure(Z[k], mu)
        Ns["x"] = Ns["x"] / 4.0
        N = Ns["e"] + Ns["x"] + (Ns["x"] if nf == 3 else 0.0)
        Nb = Ns["a"] + Ns["x"] + (Ns["x"] if nf == 3 else 0.0)
        assert r[3 + 8] == pytest.approx(N, rel=1e-15)
        assert r[3 + 8 + 2 + nh] == pytest.approx(Nb, rel=1e-15)
        assert r[3 + 10] == pytest.approx(Ns["e"] / N, rel=1e-15)
        assert r[3 + 12 + nh] == pytest.approx(Ns["a"] / Nb, rel=1e-15)
