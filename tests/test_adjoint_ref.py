"""The plain FP64 PyTorch step used as the adjoint's autograd reference:
its forward agrees with the oracle, and its autograd gradient with central
finite differences (CPU only)."""
import numpy as np
import pytest
import torch

from emu_b200 import api
from emu_b200 import workloads as W
from emu_b200.adjoint import flavor_columns, number_columns
from oracle.oracle import Oracle
from tests.torch_ref import TorchEmu


def _cases():
    return [("nf2_1d", W.c2_fast_flavor_1d(ncell_z=8, ndirs=6)),
            ("nf3_3d", W.c5_3d(n=3, ndirs=4, mixed=False))]


def _oracle_run(p, parts, nsteps):
    o = Oracle(p)
    q = parts.copy()
    mesh, vmax, dts = o.deposit(q), o.vvac_max(q), []
    for _ in range(nsteps):
        dt, _ = o.compute_dt(mesh, vmax)
        dts.append(dt)
        mesh, _, _ = o.rk_step(q, dt)
    return q, dts


@pytest.mark.parametrize("name,p", _cases(), ids=[c[0] for c in _cases()])
def test_torch_step_matches_oracle(name, p):
    parts = api.init_particles(p)
    fc, nc = flavor_columns(p.nflavors), number_columns(p.nflavors)
    q, dts = _oracle_run(p, parts, 4)
    te = TorchEmu(p, parts)
    f, pos = torch.tensor(parts[:, fc]), te.pos0
    for dt in dts:
        f, pos = te.step(f, torch.tensor(parts[:, nc]), pos, dt)
    assert np.abs(f.numpy() - q[:, fc]).max() <= 1e-13 * np.abs(q[:, fc]).max()
    assert np.array_equal(pos, q[:, :3])


@pytest.mark.parametrize("name,p", _cases(), ids=[c[0] for c in _cases()])
def test_torch_gradient_matches_fd(name, p):
    parts = api.init_particles(p)
    fc, nc = flavor_columns(p.nflavors), number_columns(p.nflavors)
    _, dts = _oracle_run(p, parts, 3)
    te = TorchEmu(p, parts)
    f0 = torch.tensor(parts[:, fc], requires_grad=True)
    N0 = torch.tensor(parts[:, nc], requires_grad=True)
    te.loss(f0, N0, dts).backward()
    g, gN = f0.grad.numpy(), N0.grad.numpy()
    scale = np.abs(g).max()
    h = 1e-7
    nh = p.nflavors ** 2
    for pi, ci in [(3, 1), (5, 2), (2, nh + 1), (7, nh + 2)]:
        fp, fm = parts[:, fc].copy(), parts[:, fc].copy()
        fp[pi, ci] += h
        fm[pi, ci] -= h
        N = torch.tensor(parts[:, nc])
        fd = (te.loss(torch.tensor(fp), N, dts).item() - te.loss(torch.tensor(fm), N, dts).item()) / (2 * h)
        assert abs(fd - g[pi, ci]) <= 1e-6 * scale
    # N weight: relative step
    Nv = parts[:, nc].copy()
    hN = 1e-7 * Nv[4, 0]
    Np, Nm = Nv.copy(), Nv.copy()
    Np[4, 0] += hN
    Nm[4, 0] -= hN
    f = torch.tensor(parts[:, fc])
    fd = (te.loss(f, torch.tensor(Np), dts).item() - te.loss(f, torch.tensor(Nm), dts).item()) / (2 * hN)
    assert abs(fd - gN[4, 0]) <= 1e-6 * abs(gN[4, 0])
