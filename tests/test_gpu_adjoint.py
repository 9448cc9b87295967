"""The hand-written adjoint (FP64 RK4, checkpointed) against torch autograd
through the plain FP64 PyTorch step and against central finite differences
of the CUDA forward with the same (recorded) timesteps.

Tolerances: J and the gradients agree with autograd to 1e-9 normwise (the
two differ only in FP64 summation order); finite differences with h = 1e-7
to 1e-5 of the gradient's largest component."""
import numpy as np
import pytest
import torch

from emu_b200 import api
from emu_b200 import workloads as W
from emu_b200.adjoint import AdjointRun, evolve, flavor_columns, nex_loss, number_columns
from tests.torch_ref import TorchEmu

pytestmark = pytest.mark.gpu


def _cases():
    return [("nf2_1d", W.c2_fast_flavor_1d(ncell_z=8, ndirs=6), 6, 4),
            ("nf3_3d", W.c5_3d(n=3, ndirs=4, mixed=False), 3, 2)]


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def _fixed_dt_J(p, records, dts):
    with api.Context(p) as c:
        c.load_particles(records)
        for dt in dts:
            c.step(float(dt))
        return c.adjoint_objective(gradient=False)[0]


@pytest.mark.parametrize("name,p,nsteps,interval", _cases(), ids=[c[0] for c in _cases()])
def test_adjoint_matches_torch_autograd(name, p, nsteps, interval):
    parts = api.init_particles(p)
    with AdjointRun(p, parts, nsteps, interval) as run:
        f0 = torch.tensor(parts[:, run.fcols], requires_grad=True)
        N = torch.tensor(parts[:, run.ncols], requires_grad=True)
        J = nex_loss(f0, N, run)
        J.backward()
        dts = run.dts
    te = TorchEmu(p, parts)
    f0r = torch.tensor(parts[:, flavor_columns(p.nflavors)], requires_grad=True)
    Nr = torch.tensor(parts[:, number_columns(p.nflavors)], requires_grad=True)
    Jr = te.loss(f0r, Nr, dts)
    Jr.backward()
    assert abs(J.item() - Jr.item()) <= 1e-10 * abs(Jr.item())
    assert _rel(f0.grad.numpy(), f0r.grad.numpy()) < 1e-9
    assert _rel(N.grad.numpy(), Nr.grad.numpy()) < 1e-9


def test_adjoint_matches_finite_differences():
    p = W.c2_fast_flavor_1d(ncell_z=8, ndirs=6)
    parts = api.init_particles(p)
    fc, nc = flavor_columns(2), number_columns(2)
    with AdjointRun(p, parts, 8, 3) as run:
        run.forward(parts[:, fc], parts[:, nc])
        J, lf, lN = run.ctx.adjoint_objective()
        g, gN = run.ctx.adjoint_backward(lf, lN)
        dts = run.dts
    assert abs(_fixed_dt_J(p, parts, dts) - J) <= 1e-12 * J
    scale = np.abs(g).max()
    h = 1e-7
    for pi, ci in [(3, 1), (11, 2), (20, 5), (40, 6)]:
        rp, rm = parts.copy(), parts.copy()
        rp[pi, fc[ci]] += h
        rm[pi, fc[ci]] -= h
        fd = (_fixed_dt_J(p, rp, dts) - _fixed_dt_J(p, rm, dts)) / (2 * h)
        assert abs(fd - g[pi, ci]) <= 1e-5 * scale, (pi, ci, fd, g[pi, ci])
    for pi, k in [(7, 0), (30, 1)]:
        hN = 1e-7 * parts[pi, nc[k]]
        rp, rm = parts.copy(), parts.copy()
        rp[pi, nc[k]] += hN
        rm[pi, nc[k]] -= hN
        fd = (_fixed_dt_J(p, rp, dts) - _fixed_dt_J(p, rm, dts)) / (2 * hN)
        assert abs(fd - gN[pi, k]) <= 1e-5 * np.abs(gN[:, k]).max(), (pi, k, fd, gN[pi, k])


def test_flux_factor_gradient_through_autograd():
    """dJ/d(nubar flux factor): Nbar is linear in the flux factor
    (Init.cpp:567-568), built here as a torch expression of a leaf tensor"""
    p = W.c2_fast_flavor_1d(ncell_z=8, ndirs=6)
    ff0 = p.st4_fluxfacbar
    hf = 1e-7
    recs = {}
    for s in (-1, 0, 1):
        q = p.copy()
        api.set_param(q, "st4_fluxfacbar", ff0 + s * hf)
        recs[s] = api.init_particles(q)
    nc = number_columns(2)
    slope = (recs[1][:, nc[1]] - recs[-1][:, nc[1]]) / (2 * hf)
    parts = recs[0]
    with AdjointRun(p, parts, 6, 4) as run:
        ff = torch.tensor(ff0, dtype=torch.float64, requires_grad=True)
        f0 = torch.tensor(parts[:, run.fcols])
        Nn = torch.tensor(parts[:, nc[0]])
        Nb = torch.tensor(parts[:, nc[1]]) + (ff - ff0) * torch.tensor(slope)
        J = nex_loss(f0, torch.stack([Nn, Nb], 1), run)
        J.backward()
        dts = run.dts
    fd = (_fixed_dt_J(p, recs[1], dts) - _fixed_dt_J(p, recs[-1], dts)) / (2 * hf)
    assert abs(fd - ff.grad.item()) <= 1e-5 * abs(fd)


def test_evolve_function_with_a_torch_loss():
    """evolve() returns the final state; any torch loss of it backpropagates
    through the adjoint"""
    p = W.c2_fast_flavor_1d(ncell_z=8, ndirs=6)
    parts = api.init_particles(p)
    w = torch.tensor(np.random.default_rng(3).standard_normal((parts.shape[0], 8)))
    with AdjointRun(p, parts, 5, 2) as run:
        f0 = torch.tensor(parts[:, run.fcols], requires_grad=True)
        N = torch.tensor(parts[:, run.ncols], requires_grad=True)
        fT = evolve(f0, N, run)
        fin = run.ctx.get_particles()
        assert np.array_equal(fT.detach().numpy(), fin[:, run.fcols])
        (w * fT).sum().backward()
        dts = run.dts
    te = TorchEmu(p, parts)
    f0r = torch.tensor(parts[:, run.fcols], requires_grad=True)
    Nr = torch.tensor(parts[:, run.ncols], requires_grad=True)
    f, pos = f0r, te.pos0
    for dt in dts:
        f, pos = te.step(f, Nr, pos, float(dt))
    (w * f).sum().backward()
    assert _rel(f0.grad.numpy(), f0r.grad.numpy()) < 1e-9
    assert _rel(N.grad.numpy(), Nr.grad.numpy()) < 1e-9


def test_adjoint_errors():
    p = W.c2_fast_flavor_1d(ncell_z=4, ndirs=4)
    parts = api.init_particles(p)
    n, ns = parts.shape[0], 8
    with api.Context(p) as c:
        c.load_particles(parts)
        with pytest.raises(api.EmuError):
            c.adjoint_backward(np.zeros((n, ns)))          # nothing recorded
        c.adjoint_forward(3, 2)
        c.load_particles(parts)                             # invalidates the recording
        with pytest.raises(api.EmuError):
            c.adjoint_backward(np.zeros((n, ns)))
    q = p.copy()
    q.precision = api.PREC_MIXED
    with api.Context(q) as c:
        c.load_particles(parts)
        with pytest.raises(api.EmuError):
            c.adjoint_forward(3, 2)


@pytest.mark.parametrize("store", ["full", "segment", "per_step", "per_step_sub2", "per_step_sub3"])
def test_adjoint_memory_modes_agree(monkeypatch, store):
    """every step stored by the recorded forward (no recompute), stage states
    recomputed and kept for a whole segment, recomputed step by step (budget
    0), or step by step from sub-checkpoints inside a 7-step segment held in
    3 or 4 segment slots (sub-segments of 4 + 3 or 3 + 4 steps; the mode for
    runs whose checkpoints and step states would not fit in memory): same
    gradient to rounding"""
    if store == "segment":
        monkeypatch.setenv("EMU_ADJOINT_FULL_STORE", "0")
    elif store != "full":
        monkeypatch.setenv("EMU_ADJOINT_STORE_MAX_BYTES", "0")
    if store.startswith("per_step_sub"):
        monkeypatch.setenv("EMU_ADJOINT_SUBCHECKPOINT", store[-1])
        monkeypatch.setenv("EMU_ADJOINT_SEG_SLOTS", str(int(store[-1]) + 1))
    p = W.c2_fast_flavor_1d(ncell_z=8, ndirs=6)
    parts = api.init_particles(p)
    fc, nc = flavor_columns(2), number_columns(2)
    with AdjointRun(p, parts, 16, 7) as run:
        run.load(parts[:, fc], parts[:, nc])
        nbytes, stage_store, sub = run.ctx.adjoint_reserve(16, 7)
        assert stage_store == {"full": 2, "segment": 1}.get(store, 0)
        run.forward(parts[:, fc], parts[:, nc])
        J, lf, lN = run.ctx.adjoint_objective()
        g, gN = run.ctx.adjoint_backward(lf, lN)
        dts = run.dts
    te = TorchEmu(p, parts)
    f0r = torch.tensor(parts[:, fc], requires_grad=True)
    Nr = torch.tensor(parts[:, nc], requires_grad=True)
    te.loss(f0r, Nr, dts).backward()
    assert _rel(g, f0r.grad.numpy()) < 1e-9
    assert _rel(gN, Nr.grad.numpy()) < 1e-9


@pytest.mark.parametrize("store", ["segment", "per_step", "per_step_sub2", "per_step_sub2_nomesh"])
def test_adjoint_3d_resorted_every_step(monkeypatch, store):
    """3 flavors, 3D TSC: particles re-sorted after every step (the automatic
    interval).  The recorded forward composes a segment's re-sorts into one
    map; the per-step modes re-sort their recomputes too and undo each step's
    permutation in the sweep, with the stage meshes kept from the state pass
    (or, nomesh, redeposited by the sweep's recompute); sub2: a 6-step
    segment in 2 segment slots (sub-segments of 3, 2 and 1 steps).  Gradient
    against torch autograd."""
    if store != "segment":
        monkeypatch.setenv("EMU_ADJOINT_STORE_MAX_BYTES", "0")
    if store.startswith("per_step_sub2"):
        monkeypatch.setenv("EMU_ADJOINT_SUBCHECKPOINT", "2")
        monkeypatch.setenv("EMU_ADJOINT_SEG_SLOTS", "2")
    if store.endswith("nomesh"):
        monkeypatch.setenv("EMU_ADJOINT_STORE_MESHES", "0")
    p = W.c5_3d(n=3, ndirs=4, mixed=False)
    parts = api.init_particles(p)
    fc, nc = flavor_columns(3), number_columns(3)
    with AdjointRun(p, parts, 7, 6) as run:
        run.forward(parts[:, fc], parts[:, nc])
        J, lf, lN = run.ctx.adjoint_objective()
        g, gN = run.ctx.adjoint_backward(lf, lN)
        dts = run.dts
    te = TorchEmu(p, parts)
    f0r = torch.tensor(parts[:, fc], requires_grad=True)
    Nr = torch.tensor(parts[:, nc], requires_grad=True)
    te.loss(f0r, Nr, dts).backward()
    assert _rel(g, f0r.grad.numpy()) < 1e-9
    assert _rel(gN, Nr.grad.numpy()) < 1e-9
