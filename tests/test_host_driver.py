"""emu_main, the C++ host driver (the evolve_flavor loop of Source/main.cpp
over the C ABI): command line and inputs errors on CPU, a full run with
plotfiles on the GPU."""
import os
import subprocess

import numpy as np
import pytest

from emu_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MAIN = os.path.join(ROOT, "emu_b200", "emu_main")

FAST_FLAVOR = """
simulation_type = 4
cfl_factor = 0.5
flavor_cfl_factor = 0.5
max_adaptive_speedup = 0
maxError = 1e-6
integration.type = 1
integration.rk.type = 4
ncell = (1, 1, 8)
Lx = 1.0
Ly = 1.0
Lz = 4.0
nppc = (1, 1, 1)
nphi_equator = 4
max_grid_size = 64
nsteps = 7
end_time = 1.0
rho_g_ccm = 0
T_MeV = 10
Ye = 1
write_plot_every = 3
write_plot_particles_every = 3
do_restart = 0
restart_dir = ""
mass1_eV = 0
mass2_eV = 0
mass3_eV = 0
theta12_degrees = 1e-6
theta23_degrees = 0
theta13_degrees = 0
alpha1_degrees = 0
alpha2_degrees = 0
deltaCP_degrees = 0
st4_ndens = 4.89e32
st4_theta = 0
st4_phi = 0
st4_fluxfac = 0
st4_ndensbar = 4.89e32
st4_thetabar = 0
st4_phibar = 0
st4_fluxfacbar = 0.333333333333333
st4_amplitude = 1e-6
emu.seed = 7
"""


def _run(args, cwd):
    return subprocess.run([MAIN] + args, cwd=cwd, capture_output=True, text=True, timeout=300)


def test_driver_usage_and_inputs_errors(tmp_path):
    assert os.path.exists(MAIN)
    assert _run([], tmp_path).returncode == 2
    r = _run([str(tmp_path / "missing")], tmp_path)
    assert r.returncode == 1 and "cannot open" in r.stderr
    f = tmp_path / "inputs"
    f.write_text(FAST_FLAVOR.replace("maxError = 1e-6", ""))
    r = _run([str(f)], tmp_path)
    assert r.returncode == 1 and "maxError" in r.stderr


@pytest.mark.gpu
def test_driver_runs_inputs_and_writes_plotfiles(tmp_path):
    f = tmp_path / "inputs"
    f.write_text(FAST_FLAVOR)
    r = _run([str(f)], tmp_path)
    assert r.returncode == 0, r.stderr
    assert "Average number of particles advanced per microsecond" in r.stdout
    for step in (0, 3, 6, 7):
        assert (tmp_path / ("plt%05d" % step) / "Header").exists() or step == 7
    p = api.parse_inputs(str(f))
    parts = api.init_particles(p)
    out, t, step = api.read_particles(str(tmp_path / "plt00006"), 2)
    assert step == 6
    with api.Context(p) as c:
        c.load_particles(parts)
        info = c.evolve(6)
        ref = c.get_particles()
        assert abs(info.time - t) <= 1e-14 * t
    # order-free comparison: sort by position and momentum direction
    key = lambda a: np.lexsort((a[:, 9], a[:, 8], a[:, 7], a[:, 2], a[:, 1], a[:, 0]))
    a, b = out[key(out)], ref[key(ref)]
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    # override on the command line: 2 steps, no plotfiles after the first
    r = _run([str(f), "nsteps=2", "write_plot_every=100", "write_plot_particles_every=0"], tmp_path / ".")
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_driver_restart_continues_like_the_reference(tmp_path):
    """do_restart = 1 (main.cpp:103-110, RecoverParticles IO.cpp:40-63): the
    run restarted from plt00003 takes the particles, time and step of that
    plotfile, deposits them and takes its first dt from that mesh, as the
    reference's restart does; its plt00006 equals the oracle continuing
    from plt00003 the same way (1e-12), and the uninterrupted run (whose dt
    after step 3 came from the stage-4 mesh) to 1e-6."""
    from oracle.oracle import Oracle
    full, rest = tmp_path / "full", tmp_path / "restart"
    full.mkdir()
    rest.mkdir()
    f = tmp_path / "inputs"
    f.write_text(FAST_FLAVOR)
    r = _run([str(f), "nsteps=6"], full)
    assert r.returncode == 0, r.stderr
    r = _run([str(f), "nsteps=6", "do_restart=1", "restart_dir=%s" % (full / "plt00003")], rest)
    assert r.returncode == 0, r.stderr
    assert "Restarting after time step: 2 t = " in r.stdout
    assert not (rest / "plt00000").exists() and not (rest / "plt00003").exists()
    p = api.parse_inputs(str(f))
    p3, t3, s3 = api.read_particles(str(full / "plt00003"), 2)
    assert s3 == 3
    out, t, step = api.read_particles(str(rest / "plt00006"), 2)
    assert step == 6
    ref, t_ref, _, st = Oracle(p).evolve(p3, 3, start_time=t3)
    assert st == 0 and abs(t - t_ref) <= 1e-13 * t_ref
    key = lambda a: np.lexsort((a[:, 9], a[:, 8], a[:, 7], a[:, 2], a[:, 1], a[:, 0]))
    a, b = out[key(out)], ref[key(ref)]
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    u, tu, _ = api.read_particles(str(full / "plt00006"), 2)
    assert abs(tu - t) <= 1e-6 * t
    uu = u[key(u)]
    assert np.abs(uu[:, 3:] - a[:, 3:]).max() <= 1e-6 * np.abs(a[:, 3:]).max()
