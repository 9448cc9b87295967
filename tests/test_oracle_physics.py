"""The reference's physics regression checks (Scripts/tests/*.py, run by
.travis.yml:32-36) applied to the oracle: MSW conversion probability,
fast-flavor growth rates (k = 0 and k != 0), trace and flavor-vector length
conservation.  Tolerances: the reference's own (7e-2, 2e-2, 1e-2) plus
tighter ones that the FP64 RK4 oracle meets."""
import math

import numpy as np

from emu_b200 import api
from emu_b200 import workloads as W
from oracle.oracle import Oracle


def _run(p, parts, nsteps, record_cols, end_time=float("inf")):
    o = Oracle(p)
    vmax = o.vvac_max(parts)
    mesh = o.deposit(parts)
    dt, st = o.compute_dt(mesh, vmax)
    assert st == 0
    t = 0.0
    ts = [0.0]
    rec = [parts[:, record_cols].copy()]
    for _ in range(nsteps):
        last = False
        if end_time - t < dt:
            dt = end_time - t
            last = True
        mesh, s, _ = o.rk_step(parts, dt)
        assert s == 0
        t += dt
        ts.append(t)
        rec.append(parts[:, record_cols].copy())
        if last:
            break
        dt, _ = o.compute_dt(mesh, vmax)
    return np.array(ts), np.array(rec)


def test_msw_ci_case():
    """inputs_msw_test + msw_test.py:26-111"""
    p = W.ci_msw()
    parts = api.init_particles(p)
    assert parts.shape[0] == 2        # nphi_equator = 1 gives +z and -z
    f00, f11, f00b, f11b = 3 + 10, 3 + 13, 3 + 16, 3 + 19
    ts, rec = _run(p, parts, p.nsteps, [f00, f11, f00b, f11b])
    E = parts[0, 3 + 7]
    dm2c4 = (p.mass2 ** 2 - p.mass1 ** 2) * api.CLIGHT ** 4
    V = math.sqrt(2) * api.GF * p.rho_in * p.Ye_in / api.MP
    pee, peeb = W.msw_probabilities(ts, E, dm2c4, p.theta12, V)
    fee, fxx, feeb, fxxb = rec[:, 0, 0], rec[:, 0, 1], rec[:, 0, 2], rec[:, 0, 3]
    for err in (np.abs(fee - pee).max(), np.abs(fxx - (1 - pee)).max(), np.abs(feeb - peeb).max(),
                np.abs(fxxb - (1 - peeb)).max()):
        assert err < 7e-2          # msw_test.py:24
        assert err < 1e-6
    assert np.abs(fee + fxx - 1).max() < 1e-12
    assert np.abs(feeb + fxxb - 1).max() < 1e-12


def test_fast_flavor_ci_growth_rate():
    """inputs_fast_flavor + fast_flavor_test.py:53-90"""
    p = W.ci_fast_flavor()
    parts = api.init_particles(p)
    cols = [3 + 11, 3 + 12, 3 + 17, 3 + 18]
    ts, rec = _run(p, parts, p.nsteps, cols)
    E = 50e6 * api.EV
    dm21c4 = 7.39e-5 * api.EV ** 2
    im_omega = dm21c4 / (2 * E) / api.HBAR
    i0, i1 = 50, 70
    for c in range(4):
        rate = math.log(rec[i1, 0, c] / rec[i0, 0, c]) / (ts[i1] - ts[i0])
        assert abs(im_omega - rate) / im_omega < 2e-2


def test_fast_flavor_k_ci_growth_rate():
    """inputs_fast_flavor_nonzerok + fast_flavor_k_test.py:58-94"""
    p = W.ci_fast_flavor_k()
    parts = api.init_particles(p)
    cols = [3 + 11, 3 + 12, 3 + 17, 3 + 18]
    ts, rec = _run(p, parts, 170, cols)
    k = 2 * math.pi / p.Lx
    im_omega = (0.0 + k * api.HBAR * api.CLIGHT) / api.HBAR
    i0, i1 = 100, 160
    for c in range(4):
        m0 = np.abs(rec[i0, :, c]).max()
        m1 = np.abs(rec[i1, :, c]).max()
        rate = math.log(m1 / m0) / (ts[i1] - ts[i0])
        assert abs(im_omega - rate) / im_omega < 1e-2


def test_c1_msw_analytic_and_conservation():
    """C1: single 50 MeV particle at resonance, 5 oscillation periods."""
    p, recs, t_end = W.c1_msw()
    o = Oracle(p)
    parts, t, dts, status = o.evolve(recs, 100000, end_time=t_end)
    assert status == 0 and abs(t - t_end) <= 1e-12 * t_end
    E = recs[0, 3 + 7]
    dm2c4 = (p.mass2 ** 2 - p.mass1 ** 2) * api.CLIGHT ** 4
    V = math.sqrt(2) * api.GF * p.rho_in * p.Ye_in / api.MP
    pee, peeb = W.msw_probabilities(t, E, dm2c4, p.theta12, V)
    assert abs(parts[0, 3 + 10] - pee) < 1e-6
    assert abs(parts[0, 3 + 16] - peeb) < 1e-6
    assert abs(parts[0, 3 + 10] + parts[0, 3 + 13] - 1) < 1e-12


def test_length_conservation_fast_flavor():
    """plot_constraints.py:71-92: |SU(n) vector| stays at L (renormalised)."""
    p = W.c2_fast_flavor_1d(ncell_z=8, ndirs=12)
    parts = api.init_particles(p)
    o = Oracle(p)
    out, t, dts, status = o.evolve(parts, 20)
    assert status == 0
    nh = 4
    for sp, (fo, lo) in enumerate(((3 + 10, 3 + 9), (3 + 12 + nh, 3 + 11 + nh))):
        L = np.array([o.su_length(r[fo:fo + nh]) for r in out])
        assert np.abs(L - out[:, lo]).max() < 1e-6 * 1.01
