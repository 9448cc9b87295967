"""Mixed-precision path (FP32 interpolation and commutator, i.e. an FP32
right-hand side, int64 fixed-point deposit, FP64 state accumulation and
renormalisation) against the FP64 oracle.

Stated tolerances:
  one RK4 step      normwise relative error per flavor attribute <= 2e-6
  mesh deposit      per component <= 1e-6 of the largest sum of |contributions|
  12 steps          mean |rho_01| and the domain-integrated |N_01| within
                    1e-5 relative of the FP64 oracle
  reproducibility   bit-identical results across runs (integer mesh sums
                    are independent of atomic / CTA scheduling; per-run FP32
                    partial sums follow the deterministic cell-sorted order);
                    a permuted particle order agrees within FP32 rounding
"""
import numpy as np
import pytest

from emu_b200 import api
from emu_b200 import workloads as W
from oracle.oracle import Oracle
from tests.helpers import colwise_rel, flavor_cols, magnitude_mesh, mesh_rel_mag

pytestmark = pytest.mark.gpu


def _params(nf=3, ncz=32, nphi=4, threed=False):
    if threed:
        p = W.c5_3d(n=4, ndirs=6, mixed=True)
    else:
        p = W.c3_three_flavor_1d(ncell_z=ncz, nphi_equator=nphi, mixed=True) if nf == 3 else \
            W.c2_fast_flavor_1d(ncell_z=ncz, ndirs=10)
    p.precision = api.PREC_MIXED
    p.resort_interval = 4
    return p


@pytest.mark.parametrize("nf,threed", [(2, False), (3, False), (3, True)])
def test_mixed_deposit_and_one_step(nf, threed):
    p = _params(nf, threed=threed)
    parts = api.init_particles(p)
    o = Oracle(p)
    ncomp = 3 + 8 * nf * nf
    with api.Context(p) as c:
        c.load_particles(parts)
        mesh = c.get_mesh()
        ref = o.deposit(parts)
        # FP32 contributions: error relative to the sum of |contributions|
        assert mesh_rel_mag(mesh, ref, magnitude_mesh(o, parts), ncomp) < 1e-6
        dt, _ = c.compute_dt()
        dto, _ = o.compute_dt(ref, o.vvac_max(parts))
        assert abs(dt - dto) <= 1e-6 * dto
        c.step(dto)
        out = c.get_particles()
    q = parts.copy()
    o.rk_step(q, dto)
    fc = flavor_cols(nf)
    assert colwise_rel(out[:, fc], q[:, fc]) < 2e-6
    assert colwise_rel(out[:, :11], q[:, :11]) < 1e-14   # positions, time, momenta exact


def _observables(parts, nf):
    nh = nf * nf
    f01 = 3 + 11
    rho01 = np.hypot(parts[:, f01], parts[:, f01 + 1])
    N01 = np.hypot((parts[:, f01] * parts[:, 3 + 8]).sum(), (parts[:, f01 + 1] * parts[:, 3 + 8]).sum())
    return rho01.mean(), N01


@pytest.mark.parametrize("nf", [2, 3])
def test_mixed_observables_12_steps(nf):
    p = _params(nf)
    parts = api.init_particles(p)
    ref, t_ref, _, _ = Oracle(p).evolve(parts, 12)
    with api.Context(p) as c:
        c.load_particles(parts)
        info = c.evolve(12)
        out = c.get_particles()
    assert info.status == 0 and info.steps_done == 12
    assert abs(info.time - t_ref) <= 1e-6 * t_ref
    a, b = _observables(out, nf), _observables(ref, nf)
    assert abs(a[0] - b[0]) <= 1e-5 * b[0]
    assert abs(a[1] - b[1]) <= 1e-5 * b[1]


def test_mixed_bit_reproducible():
    p = _params(3)
    parts = api.init_particles(p)
    perm = np.random.default_rng(3).permutation(len(parts))
    with api.Context(p) as c:
        c.load_particles(parts)
        c.evolve(6)
        a = c.get_particles()
        ma = c.get_mesh()
        c.load_particles(parts)
        c.evolve(6)
        b = c.get_particles()
        mb = c.get_mesh()
        c.load_particles(parts[perm])
        c.evolve(6)
        d = c.get_particles()
        md = c.get_mesh()
    assert np.array_equal(a, b) and np.array_equal(ma, mb)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    # the mesh (hence dt, hence positions) moves by FP32 rounding
    fc = flavor_cols(3)
    assert colwise_rel(d[inv][:, fc], a[:, fc]) < 1e-5
    assert colwise_rel(d[inv][:, :13], a[:, :13]) < 1e-6


@pytest.mark.parametrize("mixed", [True, False])
def test_large_load_statistics(mixed):
    """A load of more than 65,536 records reduces its statistics (smallest
    pupt for Vvac_max, weight sums for the fixed-point scales) on the
    device: the deposit and compute_dt agree with the oracle as for small
    loads"""
    p = W.c3_three_flavor_1d(ncell_z=256, mixed=mixed)
    p.precision = api.PREC_MIXED if mixed else api.PREC_FP64
    parts = api.init_particles(p)
    assert parts.shape[0] > 65536
    o = Oracle(p)
    ref = o.deposit(parts)
    with api.Context(p) as c:
        c.load_particles(parts)
        mesh = c.get_mesh()
        dt, _ = c.compute_dt()
    dto, _ = o.compute_dt(ref, o.vvac_max(parts))
    if mixed:
        assert mesh_rel_mag(mesh, ref, magnitude_mesh(o, parts), 3 + 72) < 1e-6
        assert abs(dt - dto) <= 1e-6 * dto
    else:
        assert mesh_rel_mag(mesh, ref, magnitude_mesh(o, parts), 3 + 72) < 1e-12
        assert abs(dt - dto) <= 1e-12 * dto
