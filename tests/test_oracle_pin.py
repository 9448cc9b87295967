"""Pin the oracle (oracle/emu_oracle.c) to the reference's own arithmetic.

The golden fixtures were produced by the reference's generated kernel bodies
(tests/golden/make_golden.py); the live comparisons run the same bodies from
oracle/_ref when it has been built.  Tolerance: 1e-13 normwise relative per
attribute / mesh component (the two differ only in FP64 rounding order).
"""
import math

import numpy as np
import pytest

from emu_b200 import api
from oracle.oracle import Oracle, RefHarness, have_ref
from tests.helpers import GOLDEN, colwise_rel, golden_ids, load_golden, mesh_rel

TOL = 1e-13


@pytest.mark.parametrize("path", GOLDEN, ids=golden_ids())
def test_oracle_matches_golden(path):
    p, d = load_golden(path)
    o = Oracle(p)
    parts = d["parts"]
    mesh0 = o.deposit(parts)
    assert mesh_rel(mesh0, d["mesh0"], o.ncomp) < TOL
    rhs = o.interpolate_rhs(d["mesh0"], parts)
    assert colwise_rel(rhs, d["rhs0"]) < TOL
    vmax = o.vvac_max(parts)
    assert abs(vmax - float(d["vvac_max"])) <= 1e-15 * abs(float(d["vvac_max"]))
    dt, st = o.compute_dt(d["mesh0"], vmax)
    assert st == 0 and abs(dt - float(d["dt0"])) <= 1e-13 * float(d["dt0"])
    for k in (0, 2, 3, 4):
        q = parts.copy()
        mesh, s, _ = o.rk_step(q, float(d["dt0"]), rk_type=k)
        assert s == int(d["status_%d" % k])
        assert colwise_rel(q, d["step_%d" % k]) < TOL, k
        assert mesh_rel(mesh, d["mesh_%d" % k], o.ncomp) < TOL, k
    q, s, bad = o.renormalize(d["renorm_in"])
    assert s == int(d["renorm_status"]) and bad == int(d["renorm_bad"])
    assert colwise_rel(q, d["renorm_out"]) < TOL


def _random_case(nf, ncell, order, seed, rho):
    p = api.default_params(nflavors=nf, shape_order=order, ncell=ncell, Lx=2.0, Ly=3.0, Lz=5.0,
                           simulation_type=4, st4_ndens=1e32, st4_ndensbar=2e32, st4_fluxfac=0.2,
                           st4_fluxfacbar=0.3, st4_amplitude=3e-3, direction_generator=1, ndirections=4,
                           seed=seed, rho_in=rho, Ye_in=0.4, max_adaptive_speedup=3.0)
    ev_g = api.EV / api.CLIGHT ** 2
    p.mass1, p.mass2, p.mass3 = 0.01 * ev_g, 0.02 * ev_g, 0.05 * ev_g
    p.theta12, p.theta13, p.theta23, p.deltaCP = 0.5, 0.15, 0.8, 1.2
    parts = api.init_particles(p)
    rng = np.random.default_rng(seed)
    L = np.array([p.Lx, p.Ly, p.Lz])
    parts[:, 0:3] = rng.uniform(0, 1, (len(parts), 3)) * L
    parts[:, 4:7] = parts[:, 0:3]
    return p, parts


@pytest.mark.skipif(not (have_ref(2) and have_ref(3)), reason="reference harness not built")
@pytest.mark.parametrize("nf,ncell,order", [(2, (2, 2, 7), 2), (3, (3, 2, 2), 1), (2, (5, 1, 1), 0),
                                            (3, (1, 6, 1), 2)])
def test_oracle_matches_reference_live(nf, ncell, order):
    p, parts = _random_case(nf, ncell, order, 5 + nf, 2e9)
    o, r = Oracle(p), RefHarness(p)
    mo, mr = o.deposit(parts), r.deposit(parts)
    assert mesh_rel(mo, mr, o.ncomp) < TOL
    assert colwise_rel(o.interpolate_rhs(mr, parts), r.interpolate_rhs(mr, parts)) < TOL
    # adaptive dt branch (max_adaptive_speedup > 1)
    do, so = o.compute_dt(mr, r.vvac_max(parts))
    dr, sr = r.compute_dt(mr, r.vvac_max(parts))
    assert so == sr == 0 and abs(do - dr) <= 1e-13 * dr
    po, pr = parts.copy(), parts.copy()
    o.rk_step(po, dr)
    r.rk_step(pr, dr)
    assert colwise_rel(po, pr) < TOL


@pytest.mark.parametrize("nthreads", [1, 3])
def test_oracle_threads_deterministic(nthreads):
    p, parts = _random_case(3, (2, 3, 4), 2, 3, 0.0)
    o = Oracle(p)
    a = o.deposit(parts, 1)
    b = o.deposit(parts, nthreads)
    assert mesh_rel(b, a, o.ncomp) < 1e-14
    c = o.deposit(parts, nthreads)
    assert np.array_equal(b, c)


def test_shape_factors():
    """ParticleInterpolator.H:34-131 at hand-computed points, including the
    truncation-toward-zero nearest index and the delta == 0 edge."""
    p = api.default_params()
    o = Oracle(p)
    first, w = o.shape(0.0, 2)
    assert first == -2 and np.allclose(w, [0.0, 0.5, 0.5], atol=0)
    first, w = o.shape(0.3, 2)
    assert first == -1 and np.allclose(w, [0.5 * 0.7 ** 2, 0.75 - 0.04, 0.5 * 0.3 ** 2], rtol=1e-15)
    first, w = o.shape(2.7, 2)
    assert first == 1 and np.allclose(w, [0.5 * 0.3 ** 2, 0.75 - 0.04, 0.5 * 0.7 ** 2], rtol=1e-15)
    first, w = o.shape(0.3, 1)
    assert first == -1 and np.allclose(w[:2], [0.2, 0.8], rtol=1e-14)
    first, w = o.shape(1.9, 1)
    assert first == 1 and np.allclose(w[:2], [0.6, 0.4], rtol=1e-14)
    first, w = o.shape(0.3, 0)
    assert first == 0 and w[0] == 1.0
    first, w = o.shape(0.0, 0)
    assert first == -1
    for d in np.linspace(0.01, 5.99, 37):
        for order in (0, 1, 2):
            _, w = o.shape(d, order)
            assert abs(w.sum() - 1.0) < 1e-15


def test_su_length_constants():
    """The Cartan coefficient of the generated 3-flavor length expression."""
    assert math.sqrt(2.0 / 6.0) / 2.0 == 0.28867513459481287
    assert 2 * 0.28867513459481287 == 0.57735026918962573
    p = api.default_params(nflavors=3)
    o = Oracle(p)
    f = np.array([1.0, 0, 0, 0, 0, 0, 0, 0, 0])
    # pure electron flavor: |SU(3) vector| = sqrt(1/4 + 1/12) = 1/sqrt(3)
    assert abs(o.su_length(f) - 1 / math.sqrt(3)) < 4e-16


def test_vacuum_potential_theta23_unused():
    """generate_code.py:202-209 builds U23 from theta13: theta23 never enters."""
    p = api.default_params(nflavors=3)
    ev_g = api.EV / api.CLIGHT ** 2
    p.mass1, p.mass2, p.mass3 = 0.0, 0.01 * ev_g, 0.05 * ev_g
    p.theta12, p.theta13, p.deltaCP = 0.58, 0.15, 3.8
    p.theta23 = 0.1
    a = Oracle(p).vvac(1e-4)
    p.theta23 = 1.3
    b = Oracle(p).vvac(1e-4)
    assert np.array_equal(a, b)
    # Hermitian nubar is the complex conjugate
    nh = 9
    im = [2, 4, 7]
    assert np.allclose(a[nh:][im], -a[:nh][im]) and np.allclose(np.delete(a[nh:], im), np.delete(a[:nh], im))


@pytest.mark.parametrize("name,binding", [("nf2_adaptive", "cap"), ("nf3_adaptive_3d", "adaptive")])
def test_adaptive_fixtures_exercise_the_adaptive_branch(name, binding):
    """The adaptive-dt fixtures' dt0 comes from Evolve.cpp:68-74: at
    speedup 3 the cap (3 dt_stupid) binds, at 10 the adaptive potential;
    either differs from the plain dt_stupid (speedup 0)."""
    path = [g for g in GOLDEN if g.endswith("golden_%s.npz" % name)][0]
    p, d = load_golden(path)
    o = Oracle(p)
    dt0 = float(d["dt0"])
    vmax = float(d["vvac_max"])
    s = p.max_adaptive_speedup
    p.max_adaptive_speedup = 0.0
    plain, _ = Oracle(p).compute_dt(d["mesh0"], vmax)
    p.max_adaptive_speedup = 1e30
    uncapped, _ = Oracle(p).compute_dt(d["mesh0"], vmax)
    assert p.cfl_factor < 0 and abs(dt0 - plain) > 0.5 * plain
    if binding == "cap":
        assert abs(dt0 - s * plain) <= 1e-13 * dt0 and uncapped > dt0
    else:
        assert abs(dt0 - uncapped) <= 1e-13 * dt0 and uncapped < s * plain
    assert o.compute_dt(d["mesh0"], vmax)[0] == pytest.approx(dt0, rel=1e-13)
