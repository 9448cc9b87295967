"""Parity on the benchmark configurations at full size, through the C ABI.

C3 (3 flavors, 1x1x1024 cells x 378 ring directions = 387,072 particles):
the mixed-precision path against the FP64 oracle (and the FP64 CUDA path)
on the flavor-conversion observables the reference's tests use: the growth
rate of the e-mu off-diagonal density between two times (the log-ratio fit
of Scripts/tests/fast_flavor_test.py:53-90) and mean |rho_emu| of
neutrinos and antineutrinos at the end time.  Both runs end on the same
physical time (the integrator clips the last step onto end_time), so the
comparison is at equal times although the mixed path's timesteps, taken
from its own stage-4 mesh, differ from the FP64 ones by ~1e-7.  Bound: 1e-6
relative (the mixed-precision target); the FP64 CUDA path must match the
oracle to 1e-11.

C2 (2 flavors, 1x1x128 cells x 80 directions = 10,240 particles): the FP64
path against the reference-arithmetic harness over the configuration's
2000 RK4 steps, through the instability's growth and saturation, at 1e-10
normwise relative per particle attribute (measured: 5e-12).

One RK4 step of the FP64 path against the reference-arithmetic harness
(the reference's generated kernel bodies, oracle/_ref) at 1e-12 normwise
relative per particle attribute on the full C3 and on C5's 3D stencils at
32^3 cells x 96 directions (3,145,728 particles).
"""
import os

import numpy as np
import pytest

from emu_b200 import api
from emu_b200 import workloads as W
from oracle.oracle import Oracle, RefHarness, have_ref
from tests.helpers import colwise_rel, magnitude_mesh, mesh_rel_mag

pytestmark = pytest.mark.gpu

NT = os.cpu_count() or 1
MIXED_TOL = 1e-6
T_MID, T_END = 0.885e-10, 1.77e-10     # about 100 and 200 RK4 steps of C3


def _obs(parts, nf):
    nh = nf * nf
    f01 = 3 + 11
    fb01 = 3 + 12 + nh + 1
    return np.array([np.hypot(parts[:, f01], parts[:, f01 + 1]).mean(),
                     np.hypot(parts[:, fb01], parts[:, fb01 + 1]).mean()])


def _gpu_run(p, parts):
    """(observables at T_MID, at T_END, end time) of one context run to
    T_MID, then on to T_END"""
    with api.Context(p) as c:
        c.load_particles(parts)
        info = c.evolve(1000, 0.0, T_MID)
        assert info.status == 0 and abs(info.time - T_MID) <= 1e-15 * T_MID
        a = _obs(c.get_particles(), p.nflavors)
        info = c.evolve(1000, T_MID, T_END)
        assert info.status == 0 and abs(info.time - T_END) <= 1e-15 * T_END
        return a, _obs(c.get_particles(), p.nflavors), info.steps_done


def _growth(a, b):
    return np.log(b / a) / (T_END - T_MID)


@pytest.fixture(scope="module")
def c3_oracle():
    p = W.c3_three_flavor_1d(mixed=False)
    parts = api.init_particles(p)
    o = Oracle(p)
    mid, t, _, st = o.evolve(parts, 1000, T_MID, nthreads=NT)
    assert st == 0 and abs(t - T_MID) <= 1e-15 * T_MID
    end, t, _, st = o.evolve(mid, 1000, T_END, nthreads=NT, start_time=T_MID)
    assert st == 0 and abs(t - T_END) <= 1e-15 * T_END
    return parts, _obs(mid, 3), _obs(end, 3)


def test_c3_fp64_matches_oracle_at_full_size(c3_oracle):
    parts, o_mid, o_end = c3_oracle
    a, b, steps = _gpu_run(W.c3_three_flavor_1d(mixed=False), parts)
    assert steps > 50
    assert np.abs(a - o_mid).max() / o_mid.max() < 1e-11
    assert np.abs(b - o_end).max() / o_end.max() < 1e-11


def test_c3_mixed_observables_within_1e6_of_the_fp64_oracle(c3_oracle):
    parts, o_mid, o_end = c3_oracle
    a, b, _ = _gpu_run(W.c3_three_flavor_1d(mixed=True), parts)
    # mean |rho_emu| (nu, nubar) at the end time
    assert (np.abs(b - o_end) / o_end).max() < MIXED_TOL
    # growth rate of mean |rho_emu| over the second half of the run
    g, go = _growth(a, b), _growth(o_mid, o_end)
    assert (np.abs(g - go) / np.abs(go)).max() < MIXED_TOL
    # the run is in the linear phase of the instability (the observable grows)
    assert (go > 1e10).all()


def _one_step_vs_harness(p):
    parts = api.init_particles(p)
    h = RefHarness(p)
    ref, t_ref, _, st = h.evolve(parts, 1, nthreads=NT)
    mref = h.deposit(ref, NT)
    with api.Context(p) as c:
        c.load_particles(parts)
        info = c.evolve(1)
        out = c.get_particles()
        c.deposit()
        mesh = c.get_mesh()
    assert info.status == st == 0
    assert abs(info.time - t_ref) <= 1e-12 * t_ref
    assert colwise_rel(out[:, 3:], ref[:, 3:]) < 1e-12
    assert mesh_rel_mag(mesh, mref, magnitude_mesh(h, ref), api.ncomp(p.nflavors)) < 1e-12


@pytest.mark.skipif(not have_ref(3), reason="oracle/_ref not built")
def test_c3_one_step_fp64_matches_reference_harness():
    _one_step_vs_harness(W.c3_three_flavor_1d(mixed=False))


@pytest.mark.skipif(not have_ref(3), reason="oracle/_ref not built")
def test_c5_32_cubed_one_step_fp64_matches_reference_harness():
    _one_step_vs_harness(W.c5_3d(n=32, mixed=False))


@pytest.mark.skipif(not have_ref(2), reason="oracle/_ref not built")
def test_c2_full_run_fp64_matches_reference_harness():
    p = W.c2_fast_flavor_1d()
    parts = api.init_particles(p)
    ref, t_ref, _, st = RefHarness(p).evolve(parts, p.nsteps, nthreads=NT)
    with api.Context(p) as c:
        c.load_particles(parts)
        info = c.evolve(p.nsteps)
        out = c.get_particles()
    assert info.status == st == 0 and info.steps_done == p.nsteps == 2000
    assert abs(info.time - t_ref) <= 1e-13 * t_ref
    # saturated: mean |rho_emu| grew from ~1e-6 to O(0.1)
    assert _obs(out, 2)[0] > 0.1
    assert colwise_rel(out[:, 3:], ref[:, 3:]) < 1e-10
    assert (np.abs(_obs(out, 2) - _obs(ref, 2)) / _obs(ref, 2)).max() < 1e-12
