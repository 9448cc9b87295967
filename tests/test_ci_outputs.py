"""The reference's continuous-integration cases (.travis.yml:32-36: the MSW,
fast-flavor and nonzero-k fast-flavor sample inputs, each followed by its
analysis script) on this library's output.

CPU (needs the reference tree for its scripts): particles from the
library's InitParticles, evolved by the oracle, written every step by the
library's plotfile writer; the reference's own Scripts/tests/msw_test.py,
fast_flavor_test.py and fast_flavor_k_test.py run unchanged on those
plotfiles (their EmuReader and amrex_plot_tools read the particle files) and
must exit 0, i.e. pass their own tolerances.

GPU: emu_main runs the same inputs files on the device, writing plotfiles
every step; the scripts' checks, restated, pass on what the library's
particle reader reads back (the reference tree does not exist where the GPU
runs).  With EMU_KEEP_CI_PLOTFILES=<dir> the plotfiles are copied there, so
that the reference's scripts can be run on them elsewhere.
"""
import math
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

from emu_b200 import api
from oracle.build_oracle import REF_ROOT
from oracle.oracle import Oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MAIN = os.path.join(ROOT, "emu_b200", "emu_main")
SCRIPTS = os.path.join(REF_ROOT, "Scripts", "tests")

_COMMON = {
    "cfl_factor": 0.5, "max_adaptive_speedup": 0, "maxError": 1e-6, "integration.type": 1,
    "integration.rk.type": 4, "nppc": "(1, 1, 1)", "nphi_equator": 1, "max_grid_size": 64, "T_MeV": 10,
    "Ye": 1, "write_plot_every": 1, "write_plot_particles_every": 1, "do_restart": 0, "restart_dir": '""',
    "alpha1_degrees": 0, "alpha2_degrees": 0, "deltaCP_degrees": 222, "theta23_degrees": 8.61,
    "theta13_degrees": 48.3,
}
# the keys of sample_inputs/inputs_msw_test, inputs_fast_flavor and
# inputs_fast_flavor_nonzerok (the values each CI run uses)
CASES = {
    "msw": dict(_COMMON, simulation_type=0, flavor_cfl_factor=0.1, ncell="(1, 1, 1)", Lx=1.0, Ly=1.0, Lz=1.0,
                nsteps=50, end_time=1.0, rho_g_ccm=1346160134.709288, mass1_eV=-0.008596511, mass2_eV=0,
                mass3_eV=0, theta12_degrees=33.82),
    "fast_flavor": dict(_COMMON, simulation_type=2, flavor_cfl_factor=0.5, ncell="(1, 1, 1)", Lx=1e7, Ly=1e7,
                        Lz=1e7, nsteps=100, end_time=1.0, rho_g_ccm=0, mass1_eV=-0.008596511, mass2_eV=0,
                        mass3_eV=0, theta12_degrees=1e-6),
    "fast_flavor_k": dict(_COMMON, simulation_type=3, st3_amplitude=1e-6, st3_wavelength_fraction_of_domain=1,
                          flavor_cfl_factor=0.5, ncell="(1, 1, 50)", Lx=1.0, Ly=1.0, Lz=1.0, nsteps=5000,
                          end_time=1.0e-10, rho_g_ccm=0, mass1_eV=0, mass2_eV=0, mass3_eV=0.049487372,
                          theta12_degrees=1e-6),
}
SCRIPT = {"msw": "msw_test.py", "fast_flavor": "fast_flavor_test.py", "fast_flavor_k": "fast_flavor_k_test.py"}


def inputs_text(case):
    return "".join("%s = %s\n" % (k, v) for k, v in CASES[case].items())


def _write_inputs(tmp_path, case):
    f = tmp_path / ("inputs_" + case)
    f.write_text(inputs_text(case))
    return f


def _oracle_plotfiles(p, out_dir):
    """the evolve_flavor loop on the oracle with a plotfile (particles and
    the last stage's mesh) after initialisation and after every step"""
    parts = api.init_particles(p)
    o = Oracle(p)
    vmax = o.vvac_max(parts)
    mesh = o.deposit(parts)
    api.write_plotfile_host(p, os.path.join(out_dir, "plt00000"), 0.0, 0, mesh, parts)
    dt, st = o.compute_dt(mesh, vmax)
    assert st == 0
    t = 0.0
    for step in range(1, p.nsteps + 1):
        last = p.end_time - t < dt
        if last:
            dt = p.end_time - t
        mesh, st, _ = o.rk_step(parts, dt)
        assert st == 0
        t += dt
        api.write_plotfile_host(p, os.path.join(out_dir, "plt%05d" % step), t, step, mesh, parts)
        if last:
            break
        dt, _ = o.compute_dt(mesh, vmax)


@pytest.mark.skipif(not os.path.isdir(SCRIPTS), reason="reference analysis scripts not present")
@pytest.mark.parametrize("case", sorted(CASES))
def test_reference_scripts_pass_on_this_librarys_plotfiles(case, tmp_path):
    p = api.parse_inputs(str(_write_inputs(tmp_path, case)))
    run = tmp_path / "run"
    run.mkdir()
    # fast_flavor_k_test.py reads Lx from ../sample_inputs/inputs_fast_flavor_nonzerok
    (tmp_path / "sample_inputs").mkdir()
    (tmp_path / "sample_inputs" / "inputs_fast_flavor_nonzerok").write_text(inputs_text("fast_flavor_k"))
    _oracle_plotfiles(p, str(run))
    r = subprocess.run([sys.executable, os.path.join(SCRIPTS, SCRIPT[case])], cwd=run, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


# ---- the same cases through emu_main on the GPU -----------------------------
def _read_series(run_dir, cols):
    ts, rec = [], []
    step = 0
    while os.path.isdir(os.path.join(run_dir, "plt%05d" % step)):
        parts, t, s = api.read_particles(os.path.join(run_dir, "plt%05d" % step), 2)
        assert s == step
        ts.append(t)
        rec.append(parts[:, cols])
        step += 1
    return np.array(ts), np.array(rec)


def _check_msw(p, run_dir):
    """msw_test.py:26-111: f_ee, f_xx (and the antineutrino ones) of particle
    0 against Richers (2019) eq. B3 at the resonance the script sets up,
    tolerance 7e-2; trace conservation"""
    ts, rec = _read_series(run_dir, [3 + 10, 3 + 13, 3 + 16, 3 + 19])
    assert len(ts) == p.nsteps + 1
    clight, hbar, eV, mp = 2.99792458e10, 1.05457266e-27, 1.60218e-12, 1.6726219e-24
    GF = 1.1663787e-5 / (1e9 * eV) ** 2 * (hbar * clight) ** 3
    theta12 = 33.82 * math.pi / 180.
    dm21c4 = 7.39e-5 * eV ** 2
    E = dm21c4 * math.sin(2. * theta12) / (8. * math.pi * hbar * clight)
    rhoYe = 4. * math.pi * hbar * clight * mp / (math.tan(2. * theta12) * math.sqrt(2.) * GF)
    V = math.sqrt(2.) * GF * rhoYe / mp
    s2 = math.sin(2. * theta12) ** 2

    def psurv(sign):
        C = math.cos(2. * theta12) + sign * 2. * V * E / dm21c4
        return 1. - np.sin(ts * dm21c4 * math.sqrt(s2 + C ** 2) / (4. * E * hbar)) ** 2 * s2 / (s2 + C ** 2)
    fee, fxx, feeb, fxxb = (rec[:, 0, k] for k in range(4))
    for f, ana in ((fee, psurv(1)), (fxx, 1 - psurv(1)), (feeb, psurv(-1)), (fxxb, 1 - psurv(-1))):
        assert np.abs(f - ana).max() < 7e-2
    assert np.abs(fee + fxx - 1).max() < 7e-2 and np.abs(feeb + fxxb - 1).max() < 7e-2


def _check_growth(run_dir, i0, i1, im_omega, tol, use_max):
    ts, rec = _read_series(run_dir, [3 + 11, 3 + 12, 3 + 17, 3 + 18])
    assert len(ts) > i1
    for c in range(4):
        a = np.abs(rec[i0, :, c]).max() if use_max else rec[i0, 0, c]
        b = np.abs(rec[i1, :, c]).max() if use_max else rec[i1, 0, c]
        rate = math.log(b / a) / (ts[i1] - ts[i0])
        assert abs(im_omega - rate) / im_omega < tol


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_driver_ci_case_passes_the_scripts_checks(case, tmp_path):
    f = _write_inputs(tmp_path, case)
    run = tmp_path / "run"
    run.mkdir()
    r = subprocess.run([MAIN, str(f)], cwd=run, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    p = api.parse_inputs(str(f))
    if case == "msw":
        _check_msw(p, str(run))
    elif case == "fast_flavor":
        # fast_flavor_test.py:53-90: Im(Omega) = V / hbar, particle 0
        E = 50. * 1e6 * api.EV
        _check_growth(str(run), 50, 70, 7.39e-5 * api.EV ** 2 / (2. * E) / api.HBAR, 2e-2, False)
    else:
        # fast_flavor_k_test.py:58-94: Im(Omega) = (V + k hbar c) / hbar,
        # V = dm21^2 c^4 / 2E, k = 2 pi / Lx
        E = 50. * 1e6 * api.EV
        V = 7.39e-5 * api.EV ** 2 / (2. * E)
        k = 2 * math.pi / p.Lx
        _check_growth(str(run), 100, 160, (V + k * api.HBAR * api.CLIGHT) / api.HBAR, 1e-2, True)
    keep = os.environ.get("EMU_KEEP_CI_PLOTFILES")
    if keep:
        dst = os.path.join(keep, case)
        shutil.rmtree(dst, ignore_errors=True)
        shutil.copytree(str(run), dst)
