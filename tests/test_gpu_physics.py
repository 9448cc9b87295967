"""The reference's physics checks (Scripts/tests/*.py) on the CUDA path:
MSW conversion probability against the analytic formula (FP64 and the mixed
path), fast-flavor growth rates (k = 0 and k != 0) with the reference's
tolerances, trace conservation.  The step loop is the device-resident one
(emu_evolve_begin / emu_evolve_steps, dt on the device)."""
import math

import numpy as np
import pytest

from emu_b200 import api
from emu_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _run(p, parts, nsteps, cols, end_time=float("inf")):
    """the state after every step: (times, records[:, :, cols])"""
    ts, rec = [0.0], [parts[:, cols].copy()]
    with api.Context(p) as c:
        c.load_particles(parts)
        c.evolve_begin(0.0, end_time, nsteps)
        for _ in range(nsteps):
            c.evolve_steps(1)
            info = c.evolve_end()
            if info.steps_done < len(ts):
                break
            ts.append(info.time)
            rec.append(c.get_particles()[:, cols])
    return np.array(ts), np.array(rec)


@pytest.mark.parametrize("precision", [api.PREC_FP64, api.PREC_MIXED], ids=["fp64", "mixed"])
def test_c1_msw_analytic(precision):
    """C1: single 50 MeV particle at the MSW resonance, 5 oscillation
    periods; P(nu_e -> nu_e) within 1e-6 of Richers et al. 2019 eq. B3"""
    p, recs, t_end = W.c1_msw()
    p.precision = precision
    with api.Context(p) as c:
        c.load_particles(recs)
        info = c.evolve(100000, 0.0, t_end)
        out = c.get_particles()
    assert info.status == 0 and abs(info.time - t_end) <= 1e-12 * t_end
    E = recs[0, 3 + 7]
    dm2c4 = (p.mass2 ** 2 - p.mass1 ** 2) * api.CLIGHT ** 4
    V = math.sqrt(2) * api.GF * p.rho_in * p.Ye_in / api.MP
    pee, peeb = W.msw_probabilities(info.time, E, dm2c4, p.theta12, V)
    assert abs(out[0, 3 + 10] - pee) < 1e-6
    assert abs(out[0, 3 + 16] - peeb) < 1e-6
    assert abs(out[0, 3 + 10] + out[0, 3 + 13] - 1) < 1e-12


def test_msw_ci_case():
    """inputs_msw_test + msw_test.py:26-111 (tolerance 7e-2; met to 1e-6)"""
    p = W.ci_msw()
    parts = api.init_particles(p)
    f00, f11, f00b, f11b = 3 + 10, 3 + 13, 3 + 16, 3 + 19
    ts, rec = _run(p, parts, p.nsteps, [f00, f11, f00b, f11b])
    E = parts[0, 3 + 7]
    dm2c4 = (p.mass2 ** 2 - p.mass1 ** 2) * api.CLIGHT ** 4
    V = math.sqrt(2) * api.GF * p.rho_in * p.Ye_in / api.MP
    pee, peeb = W.msw_probabilities(ts, E, dm2c4, p.theta12, V)
    fee, fxx, feeb, fxxb = rec[:, 0, 0], rec[:, 0, 1], rec[:, 0, 2], rec[:, 0, 3]
    for err in (np.abs(fee - pee).max(), np.abs(fxx - (1 - pee)).max(), np.abs(feeb - peeb).max(),
                np.abs(fxxb - (1 - peeb)).max()):
        assert err < 1e-6
    assert np.abs(fee + fxx - 1).max() < 1e-12


def test_fast_flavor_growth_rate():
    """inputs_fast_flavor + fast_flavor_test.py:53-90 (tolerance 2e-2)"""
    p = W.ci_fast_flavor()
    parts = api.init_particles(p)
    ts, rec = _run(p, parts, p.nsteps, [3 + 11, 3 + 12, 3 + 17, 3 + 18])
    E = 50e6 * api.EV
    im_omega = 7.39e-5 * api.EV ** 2 / (2 * E) / api.HBAR
    i0, i1 = 50, 70
    for c in range(4):
        rate = math.log(rec[i1, 0, c] / rec[i0, 0, c]) / (ts[i1] - ts[i0])
        assert abs(im_omega - rate) / im_omega < 2e-2


def test_fast_flavor_k_growth_rate():
    """inputs_fast_flavor_nonzerok + fast_flavor_k_test.py:58-94 (tolerance 1e-2)"""
    p = W.ci_fast_flavor_k()
    parts = api.init_particles(p)
    ts, rec = _run(p, parts, 170, [3 + 11, 3 + 12, 3 + 17, 3 + 18])
    im_omega = (2 * math.pi / p.Lx) * api.HBAR * api.CLIGHT / api.HBAR
    i0, i1 = 100, 160
    for c in range(4):
        rate = math.log(np.abs(rec[i1, :, c]).max() / np.abs(rec[i0, :, c]).max()) / (ts[i1] - ts[i0])
        assert abs(im_omega - rate) / im_omega < 1e-2
