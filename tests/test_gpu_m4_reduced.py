"""The mixed path's stage-4 mesh inside a run.  compute_dt without the
adaptive branch (max_adaptive_speedup <= 1) reads only the diagonal N_ii,
Nbar_ii of the stage-4 mesh M_4; those are deposited apart, and stage 3
deposits M_4 in full only on the last step of an emu_evolve_steps call (or of
the run), the mesh a caller can read.  Every other step keeps M_4 in the
combined layout stage 4 interpolates.

Checked here: a run split over several emu_evolve_steps calls is
bit-identical to one call (particles, meshes, dt), so the layout a step
deposits does not change the trajectory; the dt of the run equals
emu_compute_dt afterwards and the oracle's compute_dt of the full mesh
within FP32 deposit rounding; a step timed by emu_profile_step leaves no
readable mesh (an error, until the next step); with the adaptive branch
every step deposits the full mesh."""
import numpy as np
import pytest

from emu_b200 import api
from emu_b200 import workloads as W
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _params(case):
    if case == "3d":
        p = W.c5_3d(n=4, ndirs=6, mixed=True)
    else:
        p = W.c3_three_flavor_1d(ncell_z=16, nphi_equator=4, mixed=True)
    p.precision = api.PREC_MIXED
    return p


def _run(p, parts, chunks):
    """evolve over the given chunks of steps; (particles, mesh after each
    chunk, final run info)"""
    meshes = []
    with api.Context(p) as c:
        c.load_particles(parts)
        c.evolve_begin(0.0, float("inf"), sum(chunks))
        for n in chunks:
            c.evolve_steps(n)
            meshes.append(c.get_mesh())
        info = c.evolve_end()
        dt_after, _ = c.compute_dt()
        return c.get_particles(), meshes, info, dt_after


@pytest.mark.parametrize("case", ["1d", "3d"])
def test_split_calls_are_bit_identical(case):
    p = _params(case)
    parts = api.init_particles(p)
    a, ma, ia, da = _run(p, parts, [9])
    b, mb, ib, db = _run(p, parts, [4, 1, 4])
    assert ia.status == 0 and ia.steps_done == 9 and ib.steps_done == 9
    assert ia.time == ib.time and ia.dt_next == ib.dt_next
    assert np.array_equal(a, b)
    assert np.array_equal(ma[-1], mb[-1])
    # the mesh read between calls is the full M_4 of that step
    c4, mc4, _, _ = _run(p, parts, [4])
    assert np.array_equal(mb[0], mc4[0])
    # the steps' compute_dt and the one after the run read the same values
    assert ia.dt_next == da


@pytest.mark.parametrize("case", ["1d", "3d"])
def test_run_dt_matches_oracle_dt_of_full_mesh(case):
    p = _params(case)
    parts = api.init_particles(p)
    out, meshes, info, _ = _run(p, parts, [6])
    o = Oracle(p)
    dto, _ = o.compute_dt(meshes[-1], o.vvac_max(parts))
    # the diagonal slots and the full mesh sum the same FP32 run totals in
    # different groupings
    assert abs(info.dt_next - dto) <= 1e-6 * dto


def test_profiled_step_leaves_no_readable_mesh():
    p = _params("3d")
    parts = api.init_particles(p)
    with api.Context(p) as c:
        c.load_particles(parts)
        c.evolve_begin(0.0, float("inf"), 10)
        c.evolve_steps(1)
        m1 = c.get_mesh()
        assert np.isfinite(m1).all()
        c.profile_step()
        with pytest.raises(api.EmuError):
            c.get_mesh()
        dt, _ = c.compute_dt()          # the diagonal slots: still valid
        assert dt > 0
        c.evolve_steps(1)
        assert np.isfinite(c.get_mesh()).all()
        c.evolve_end()


def test_adaptive_branch_deposits_the_full_mesh():
    p = _params("3d")
    p.max_adaptive_speedup = 4.0
    parts = api.init_particles(p)
    ref, t_ref, _, _ = Oracle(p).evolve(parts, 6)
    with api.Context(p) as c:
        c.load_particles(parts)
        c.evolve_begin(0.0, float("inf"), 10)
        c.evolve_steps(1)
        c.profile_step()                # every step full: the mesh stays readable
        assert np.isfinite(c.get_mesh()).all()
        c.evolve_end()
        c.load_particles(parts)
        info = c.evolve(6)
    assert info.status == 0 and info.steps_done == 6
    assert abs(info.time - t_ref) <= 1e-6 * t_ref
