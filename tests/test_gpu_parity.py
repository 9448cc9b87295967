"""CUDA path vs the oracle and the golden fixtures (reference arithmetic),
through the C ABI.

FP64 tolerance: 1e-12 normwise relative per particle attribute / mesh
component after one call (the GPU deposit adds in a different order and the
GPU may fuse multiply-adds; everything else is the same FP64 arithmetic).
"""
import numpy as np
import pytest

from emu_b200 import api
from emu_b200 import workloads as W
from oracle.oracle import Oracle
from tests.helpers import (GOLDEN, colwise_rel, flavor_cols, golden_ids, load_golden, magnitude_mesh, mesh_rel,
                           mesh_rel_mag)

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _ctx(p, **kw):
    q = p.copy()
    for k, v in kw.items():
        api.set_param(q, k, v)
    return api.Context(q)


@pytest.mark.parametrize("path", GOLDEN, ids=golden_ids())
def test_deposit_rhs_dt_vs_golden(path):
    p, d = load_golden(path)
    nc = 3 + 8 * p.nflavors ** 2
    with _ctx(p) as c:
        c.load_particles(d["parts"])
        assert colwise_rel(c.get_particles(), d["parts"]) == 0.0
        assert mesh_rel(c.get_mesh(), d["mesh0"], nc) < TOL
        assert colwise_rel(c.interpolate_rhs(), d["rhs0"]) < TOL
        dt, st = c.compute_dt()
        assert st == 0 and abs(dt - float(d["dt0"])) <= TOL * float(d["dt0"])


@pytest.mark.parametrize("path", GOLDEN, ids=golden_ids())
@pytest.mark.parametrize("integ", ["rk4_coop", "rk4_fused", "rk4_unfused", "fe", "trapezoid", "ssprk3"])
def test_one_step_vs_golden(path, integ):
    p, d = load_golden(path)
    nc = 3 + 8 * p.nflavors ** 2
    kw = {"rk4_coop": dict(integration_type=1, rk_type=4, fused=2),
          "rk4_fused": dict(integration_type=1, rk_type=4, fused=1),
          "rk4_unfused": dict(integration_type=1, rk_type=4, fused=0),
          "fe": dict(integration_type=0, rk_type=4, fused=0),
          "trapezoid": dict(integration_type=1, rk_type=2, fused=0),
          "ssprk3": dict(integration_type=1, rk_type=3, fused=0)}[integ]
    k = {"rk4_coop": 4, "rk4_fused": 4, "rk4_unfused": 4, "fe": 0, "trapezoid": 2, "ssprk3": 3}[integ]
    with _ctx(p, resort_interval=0, **kw) as c:
        c.load_particles(d["parts"])
        # (forward Euler with the 3D adaptive fixture's large dt leaves a
        # flavor-vector length error that Renormalize reports, as the
        # reference's arithmetic does)
        code, bad = c.step(float(d["dt0"]), raise_on_error=False)
        assert code == int(d["status_%d" % k])
        assert colwise_rel(c.get_particles(), d["step_%d" % k]) < TOL
        assert mesh_rel(c.get_mesh(), d["mesh_%d" % k], nc) < TOL


@pytest.mark.parametrize("path", GOLDEN, ids=golden_ids())
def test_renormalize_vs_golden(path):
    p, d = load_golden(path)
    with _ctx(p) as c:
        c.load_particles(d["renorm_in"])
        code, bad = c.renormalize()
        assert code == int(d["renorm_status"])
        assert bad == int(d["renorm_bad"])
        assert colwise_rel(c.get_particles(), d["renorm_out"]) < TOL


def _c2_small(ncz=16, ndirs=20, **kw):
    p = W.c2_fast_flavor_1d(ncell_z=ncz, ndirs=ndirs)
    for k, v in kw.items():
        api.set_param(p, k, v)
    return p


@pytest.mark.parametrize("resort,fused", [(0, 2), (1, 2), (3, 2), (0, 1), (1, 1), (3, 1)])
def test_evolve_matches_oracle(resort, fused):
    """device-resident loop (cooperative step kernel or CUDA graph of stage
    kernels, device dt) vs the oracle's evolve"""
    p = _c2_small(resort_interval=resort, fused=fused)
    parts = api.init_particles(p)
    o = Oracle(p)
    ref, t_ref, dts, st = o.evolve(parts, 12)
    with api.Context(p) as c:
        c.load_particles(parts)
        info = c.evolve(12)
        assert info.status == 0 and info.steps_done == 12
        assert abs(info.time - t_ref) <= 1e-12 * t_ref
        out = c.get_particles()
    assert colwise_rel(out, ref) < 1e-11
    assert colwise_rel(out[:, flavor_cols(2)], ref[:, flavor_cols(2)]) < 1e-11


def test_evolve_3d_matches_oracle():
    """3 flavors, 3D TSC: re-sort every step (automatic), the new state
    deposited by the re-sort gather"""
    p = W.c5_3d(n=4, ndirs=5, mixed=False)
    parts = api.init_particles(p)
    o = Oracle(p)
    ref, t_ref, _, _ = o.evolve(parts, 6)
    with api.Context(p) as c:
        c.load_particles(parts)
        info = c.evolve(6)
        assert info.status == 0 and info.steps_done == 6
        assert abs(info.time - t_ref) <= 1e-12 * t_ref
        out = c.get_particles()
        mesh = c.get_mesh()
    assert colwise_rel(out, ref) < 1e-11
    assert colwise_rel(out[:, flavor_cols(3)], ref[:, flavor_cols(3)]) < 1e-11


@pytest.mark.parametrize("mixed", [False, True])
def test_evolve_3d_wide_tiles_match_oracle(mixed):
    """3D TSC with two particles per cell and no re-sort: the stencil keys of
    a CTA's 128 particles span ~64 cells, so the load deposit and every
    stage-4 deposit of moved particles rank them with the block radix sort
    (the counting sort covers spans of at most 31 cells)"""
    p = W.c5_3d(n=6, ndirs=2, mixed=mixed)
    p.resort_interval = 0
    parts = api.init_particles(p)
    o = Oracle(p)
    ref, t_ref, _, _ = o.evolve(parts, 4)
    with api.Context(p) as c:
        c.load_particles(parts)
        info = c.evolve(4)
        assert info.status == 0 and info.steps_done == 4
        out = c.get_particles()
    fc = flavor_cols(3)
    if mixed:   # (a wrong rank would misplace whole records: O(1) errors)
        assert colwise_rel(out[:, fc], ref[:, fc]) < 1e-4
    else:
        assert colwise_rel(out, ref) < 1e-11


def test_evolve_end_time_clipping():
    p = _c2_small(ncz=8, ndirs=6)
    parts = api.init_particles(p)
    o = Oracle(p)
    _, t1, dts, _ = o.evolve(parts, 3)
    t_end = t1 + 0.5 * dts[-1]
    ref, t_ref, dts2, _ = o.evolve(parts, 100, end_time=t_end)
    with api.Context(p) as c:
        c.load_particles(parts)
        info = c.evolve(100, 0.0, t_end)
        assert info.steps_done == len(dts2)
        assert abs(info.time - t_end) <= 1e-15 * t_end
        out = c.get_particles()
    assert colwise_rel(out, ref) < 1e-11


def test_step_api_sequence_matches_oracle():
    """emu_step + emu_compute_dt driven from the host, 5 steps, 3 flavors 3D"""
    p = W.c5_3d(n=4, ndirs=5, mixed=False)
    parts = api.init_particles(p)
    o = Oracle(p)
    q = parts.copy()
    vmax = o.vvac_max(q)
    mesh = o.deposit(q)
    with api.Context(p) as c:
        c.load_particles(parts)
        for _ in range(5):
            dt_o, _ = o.compute_dt(mesh, vmax)
            dt_c, _ = c.compute_dt()
            assert abs(dt_c - dt_o) <= 1e-12 * dt_o
            mesh, s, _ = o.rk_step(q, dt_o)
            c.step(dt_o)
        assert colwise_rel(c.get_particles(), q) < 1e-11
        # Fz00 of the isotropic nu field cancels to rounding level: compare
        # against the magnitude of the deposited terms
        assert mesh_rel_mag(c.get_mesh(), mesh, magnitude_mesh(o, q), 75) < 1e-13


def test_single_particle_and_edges():
    p = W.ci_msw()
    parts = api.init_particles(p)[:1].copy()
    with api.Context(p) as c:
        c.load_particles(parts)
        dt, _ = c.compute_dt()
        c.step(dt)
        o = Oracle(p)
        q = parts.copy()
        o.rk_step(q, dt)
        assert colwise_rel(c.get_particles(), q) < TOL
    with api.Context(p) as c:
        with pytest.raises(api.EmuError):
            c.load_particles(np.zeros((0, api.nreal(2))))
        with pytest.raises(api.EmuError):
            c.get_particles()


def test_positions_on_faces_and_wrap():
    """particles exactly on cell faces, on the domain origin and moving across
    the periodic boundary"""
    p = _c2_small(ncz=6, ndirs=8)
    parts = api.init_particles(p)
    dz = p.Lz / p.ncell[2]
    parts[:, 2] = (np.arange(len(parts)) % (p.ncell[2] + 1)) * dz % p.Lz
    parts[:3, 2] = [0.0, p.Lz - 1e-12, dz * 3]
    parts[:, 6] = parts[:, 2]
    o = Oracle(p)
    ref, t, _, _ = o.evolve(parts, 4)
    with api.Context(p) as c:
        c.load_particles(parts)
        c.evolve(4)
        out = c.get_particles()
    assert colwise_rel(out, ref) < 1e-11
    assert (out[:, 2] >= 0).all() and (out[:, 2] < p.Lz).all()


def test_renormalize_error_reported_from_step():
    """a particle whose trace is off by 2e-3 (> 100*maxError) after the
    step: status EMU_ERR_TRACE and its load index, no abort"""
    p = _c2_small(ncz=4, ndirs=6)
    parts = api.init_particles(p)
    parts[5, 3 + 10] += 2e-3
    with api.Context(p) as c:
        c.load_particles(parts)
        dt, _ = c.compute_dt()
        code, bad = c.step(dt, raise_on_error=False)
        assert code & api.EMU_ERR_TRACE
        assert bad == 5
        # the context stays usable
        c.load_particles(api.init_particles(p))
        code, bad = c.step(dt, raise_on_error=False)
        assert code == 0 and bad == -1


def test_bad_arguments():
    p = api.default_params(nflavors=4)
    with pytest.raises(api.EmuError):
        api.Context(p)
    p = api.default_params(ncell=(1, 1, 1), Lx=-1.0)
    with pytest.raises(api.EmuError):
        api.Context(p)
