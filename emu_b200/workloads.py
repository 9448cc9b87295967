"""Named run configurations.

ci_*   the parameter sets of Emu's continuous-integration runs (the
       sample_inputs files exercised by .travis.yml:32-36), restated as
       EmuParams so that no inputs file is needed.
c1..c5 the benchmark configurations: MSW single particle, fast-flavor 1D
       (2 flavors, 128 cells x 80 Fibonacci directions), 3-flavor 1D mixed
       precision (1024 cells x 378 ring directions), the adjoint run, and the
       3D scale run (64^3 cells x 96 directions).  Inputs are synthetic: the
       reference ships no datasets; each builder documents its choices.
"""
import math

import numpy as np

from . import api

DEG = math.pi / 180.
EV_G = api.EV / api.CLIGHT ** 2      # eV -> grams (Parameters.H:81-82)


def _physics(p, m1_ev, m2_ev, m3_ev, th12_deg, th13_deg=48.3, th23_deg=8.61, dcp_deg=222.0):
    p.mass1, p.mass2, p.mass3 = m1_ev * EV_G, m2_ev * EV_G, m3_ev * EV_G
    p.theta12, p.theta13, p.theta23 = th12_deg * DEG, th13_deg * DEG, th23_deg * DEG
    p.alpha1 = p.alpha2 = 0.0
    p.deltaCP = dcp_deg * DEG


def _base(nf=2, **kw):
    p = api.default_params(nflavors=nf, shape_order=2, integration_type=1, rk_type=4, maxError=1e-6,
                           max_adaptive_speedup=0.0, T_in=10.0, Ye_in=1.0)
    for k, v in kw.items():
        api.set_param(p, k, v)
    return p


# ---- the reference's CI cases -------------------------------------------------
def ci_msw(nf=2):
    """inputs_msw_test: vacuum + matter at the MSW resonance, 1 cell."""
    p = _base(nf, simulation_type=0, cfl_factor=0.5, flavor_cfl_factor=0.1, ncell=(1, 1, 1), Lx=1.0, Ly=1.0,
              Lz=1.0, nppc=(1, 1, 1), nphi_equator=1, nsteps=50, end_time=1.0, rho_in=1346160134.709288,
              Ye_in=1.0)
    _physics(p, -0.008596511, 0.0, 0.0, 33.82)
    return p


def ci_bipolar(nf=2):
    p = _base(nf, simulation_type=1, cfl_factor=0.5, flavor_cfl_factor=0.5, ncell=(1, 1, 1), Lx=1e7, Ly=1e7,
              Lz=1e7, nppc=(1, 1, 1), nphi_equator=1, nsteps=200, end_time=1.0, rho_in=0.0)
    _physics(p, -0.008596511, 0.0, 0.0, 33.82)
    return p


def ci_fast_flavor(nf=2):
    """inputs_fast_flavor: two-beam fast-flavor instability, 1 cell."""
    p = _base(nf, simulation_type=2, cfl_factor=0.5, flavor_cfl_factor=0.5, ncell=(1, 1, 1), Lx=1e7, Ly=1e7,
              Lz=1e7, nppc=(1, 1, 1), nphi_equator=1, nsteps=100, end_time=1.0, rho_in=0.0)
    _physics(p, -0.008596511, 0.0, 0.0, 1e-6)
    return p


def ci_fast_flavor_k(nf=2):
    """inputs_fast_flavor_nonzerok: k != 0 instability on 1x1x50 cells."""
    p = _base(nf, simulation_type=3, st3_amplitude=1e-6, st3_wavelength_fraction_of_domain=1, cfl_factor=0.5,
              flavor_cfl_factor=0.5, ncell=(1, 1, 50), Lx=1.0, Ly=1.0, Lz=1.0, nppc=(1, 1, 1), nphi_equator=1,
              nsteps=5000, end_time=1.0e-10, rho_in=0.0)
    _physics(p, 0.0, 0.0, 0.049487372, 1e-6)
    return p


def ci_fiducial_1d(nf=3):
    """inputs_1d_fiducial: randomized k != 0 on 1x1x256 cells, 92 directions."""
    p = _base(nf, simulation_type=4, st4_theta=0.0, st4_thetabar=3.14159265359, st4_phi=0.0, st4_phibar=0.0,
              st4_ndens=4.891290819e+32, st4_ndensbar=4.891290819e+32, st4_fluxfac=.333333333333333,
              st4_fluxfacbar=.333333333333333, st4_amplitude=1e-6, cfl_factor=0.5, flavor_cfl_factor=0.5,
              ncell=(1, 1, 256), Lx=1.0, Ly=1.0, Lz=64.0, nppc=(1, 1, 1), nphi_equator=16, nsteps=5000,
              end_time=5.0e-9, rho_in=0.0)
    _physics(p, 0.0, 0.0, 0.049487372, 1e-6)
    return p


# ---- benchmark configurations ------------------------------------------------
def c1_msw():
    """2 flavors, one 1-cm periodic cell, one particle along +z at 50 MeV,
    theta12 = 0.1 rad, dm^2 = 2.4e-3 eV^2 (m2^2 > m1^2), electron density at
    the nu MSW resonance, self-interaction off (N = 0).  Returns (params,
    records, t_end) with t_end = 5 oscillation periods.  The translation
    limiter is off (cfl_factor = -1, as Scripts/tests/convergence.sh:12 runs
    the MSW case): a 1 cm cell would otherwise cap dt at 17 ps against a
    0.87 ms oscillation period; dt comes from the flavor CFL (0.1)."""
    dm2 = 2.4e-3
    theta = 0.1
    p = _base(2, simulation_type=4, st4_ndens=0.0, st4_ndensbar=0.0, st4_amplitude=0.0, cfl_factor=-1.0,
              flavor_cfl_factor=0.1, ncell=(1, 1, 1), Lx=1.0, Ly=1.0, Lz=1.0, nphi_equator=1, Ye_in=1.0)
    p.mass1, p.mass2, p.mass3 = 0.0, math.sqrt(dm2) * EV_G, 0.0
    p.theta12 = theta
    p.theta13 = p.theta23 = p.deltaCP = 0.0
    E = 50e6 * api.EV
    dm2c4 = dm2 * api.EV ** 2
    ne = dm2c4 * math.cos(2 * theta) / (2 * math.sqrt(2) * api.GF * E)
    p.rho_in = ne * api.MP / p.Ye_in
    recs = api.init_particles(p)
    recs = recs[np.argmax(recs[:, 3 + 6])][None, :].copy()      # the +z particle
    period = 4 * math.pi * E * api.HBAR / (dm2c4 * math.sin(2 * theta))
    p.end_time = 5 * period
    p.nsteps = 100000
    return p, recs, 5 * period


def _fast_flavor_1d(nf, ncell_z, lz, direction_generator, ndirs_or_nphi, seed=0):
    p = _base(nf, simulation_type=4, st4_theta=0.0, st4_thetabar=0.0, st4_phi=0.0, st4_phibar=0.0,
              st4_ndens=4.89e32, st4_ndensbar=4.89e32, st4_fluxfac=0.0, st4_fluxfacbar=1.0 / 3.0,
              st4_amplitude=1e-6, cfl_factor=0.5, flavor_cfl_factor=0.5, ncell=(1, 1, ncell_z), Lx=1.0, Ly=1.0,
              Lz=lz, nppc=(1, 1, 1), rho_in=0.0, seed=seed, direction_generator=direction_generator)
    if direction_generator == 1:
        p.ndirections = ndirs_or_nphi
    else:
        p.nphi_equator = ndirs_or_nphi
    if nf == 2:
        _physics(p, -0.008596511, 0.0, 0.0, 1e-6)
    else:
        _physics(p, 0.0, 0.0, 0.049487372, 1e-6)
    return p


def c2_fast_flavor_1d(ncell_z=128, ndirs=80, nsteps=2000):
    """2 flavors, periodic 1x1x128 cells over 64 cm, 80 Fibonacci directions
    per cell (10,240 particles); nu_e isotropic, nubar_e with flux factor 1/3
    along +z, both n = 4.89e32 cm^-3 at 50 MeV; off-diagonals uniform in
    [-1e-6, 1e-6] (seed 0); FP64; cfl 0.5, flavor cfl 0.5."""
    p = _fast_flavor_1d(2, ncell_z, 64.0 * ncell_z / 128, 1, ndirs)
    p.nsteps = nsteps
    p.end_time = 1.0
    return p


def c3_three_flavor_1d(ncell_z=1024, nphi_equator=32, nsteps=200, mixed=True):
    """3 flavors, 1x1x1024 cells (dz = 0.5 cm), 378 ring directions per cell
    (nphi_equator = 32, 387,072 particles); the C2 angular setup with nu_x
    empty; mixed precision."""
    p = _fast_flavor_1d(3, ncell_z, 0.5 * ncell_z, 0, nphi_equator)
    p.precision = api.PREC_MIXED if mixed else api.PREC_FP64
    p.nsteps = nsteps
    p.end_time = 1.0
    return p


def c4_adjoint():
    """C2 sizes, 500 RK4 steps (checkpoints every 25 steps for the adjoint)."""
    return c2_fast_flavor_1d(nsteps=500)


def c5_3d(n=64, ndirs=96, nsteps=200, mixed=True, seed=1):
    """3 flavors, 64^3 periodic cells (dx = 0.5 cm) x 96 Fibonacci directions
    (25,165,824 particles), the C2 angular setup, seeded perturbations."""
    p = _base(3, simulation_type=4, st4_theta=0.0, st4_thetabar=0.0, st4_phi=0.0, st4_phibar=0.0,
              st4_ndens=4.89e32, st4_ndensbar=4.89e32, st4_fluxfac=0.0, st4_fluxfacbar=1.0 / 3.0,
              st4_amplitude=1e-6, cfl_factor=0.5, flavor_cfl_factor=0.5, ncell=(n, n, n), Lx=0.5 * n,
              Ly=0.5 * n, Lz=0.5 * n, nppc=(1, 1, 1), rho_in=0.0, seed=seed, direction_generator=1,
              ndirections=ndirs)
    _physics(p, 0.0, 0.0, 0.049487372, 1e-6)
    p.precision = api.PREC_MIXED if mixed else api.PREC_FP64
    p.nsteps = nsteps
    p.end_time = 1.0
    return p


WORKLOADS = {
    "c1": c1_msw,
    "c2": c2_fast_flavor_1d,
    "c3": c3_three_flavor_1d,
    "c4": c4_adjoint,
    "c5": c5_3d,
}


# ---- analytic checks (Scripts/tests/*.py) ------------------------------------
def msw_probabilities(t, E, dm2c4, theta, V):
    """Two-flavor matter oscillation (Richers et al. 2019, eq. B3, the formula
    of Scripts/tests/msw_test.py:65-78) for a constant matter potential V
    (erg).  dm2c4 = (m2^2 - m1^2) c^4 (signed).  Returns (Pee, Peebar)."""
    s2 = math.sin(2 * theta) ** 2
    C = math.cos(2 * theta) - 2 * V * E / dm2c4
    Cb = math.cos(2 * theta) + 2 * V * E / dm2c4
    sin2 = s2 / (s2 + C ** 2)
    sin2b = s2 / (s2 + Cb ** 2)
    dme = abs(dm2c4) * math.sqrt(s2 + C ** 2)
    dmeb = abs(dm2c4) * math.sqrt(s2 + Cb ** 2)
    t = np.asarray(t)
    pee = 1. - np.sin(t * dme / (4. * E * api.HBAR)) ** 2 * sin2
    peeb = 1. - np.sin(t * dmeb / (4. * E * api.HBAR)) ** 2 * sin2b
    return pee, peeb
