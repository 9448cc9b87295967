"""PyTorch front end of the library's discrete adjoint (FP64 RK4).

The forward run and its gradient are the library's CUDA kernels behind the
C ABI (emu_adjoint_forward / emu_adjoint_objective / emu_adjoint_backward);
this module only adapts them to torch.autograd so that initial conditions
built from torch tensors (for instance an antineutrino number that depends
on a flux factor) receive gradients by the chain rule.

    run = AdjointRun(params, records, nsteps=500, checkpoint_interval=25)
    f0 = torch.tensor(records[:, run.fcols], requires_grad=True)
    N = torch.tensor(records[:, run.ncols], requires_grad=True)
    J = nex_loss(f0, N, run)          # sum_cells |N_emu|^2 / V_cell at the end
    J.backward()                      # f0.grad, N.grad

The timestep of every step is the one the recorded forward run chose; it is
held fixed in the derivative.  Particle positions and momenta come from the
template records and are not differentiated.
"""
import numpy as np
import torch

from . import api

# record columns: x y z | time x y z pupx pupy pupz pupt N L f.. Nbar Lbar fbar..
_ATTR = 3


def flavor_columns(nf):
    """record columns of the 2 nf^2 flavor reals (nu then nubar)"""
    nh = nf * nf
    return list(range(_ATTR + 10, _ATTR + 10 + nh)) + list(range(_ATTR + 12 + nh, _ATTR + 12 + 2 * nh))


def number_columns(nf):
    """record columns of N and Nbar"""
    nh = nf * nf
    return [_ATTR + 8, _ATTR + 10 + nh]


class AdjointRun:
    """A device context plus the template particles of one differentiable run."""

    def __init__(self, params, records, nsteps, checkpoint_interval=25):
        if params.precision != api.PREC_FP64:
            raise ValueError("the adjoint is FP64 only")
        self.params = params.copy() if hasattr(params, "copy") else params
        self.records = np.ascontiguousarray(records, dtype=np.float64).copy()
        self.nf = params.nflavors
        self.fcols = flavor_columns(self.nf)
        self.ncols = number_columns(self.nf)
        self.nsteps = int(nsteps)
        self.interval = int(checkpoint_interval)
        self.ctx = api.Context(params)
        self.dts = None
        self.info = None

    def load(self, f0, N):
        r = self.records.copy()
        r[:, self.fcols] = f0
        r[:, self.ncols] = N
        self.ctx.load_particles(r)

    def forward(self, f0, N):
        """recorded forward run from (f0, N); returns the final records"""
        self.load(f0, N)
        self.dts, self.info = self.ctx.adjoint_forward(self.nsteps, self.interval)
        return self.ctx.get_particles()

    def close(self):
        self.ctx.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _np(t):
    return t.detach().to("cpu", torch.float64).numpy()


class _Evolve(torch.autograd.Function):
    @staticmethod
    def forward(fctx, f0, N, run):
        out = run.forward(_np(f0), _np(N))
        fctx.run = run
        return torch.from_numpy(np.ascontiguousarray(out[:, run.fcols])).to(f0.device)

    @staticmethod
    def backward(fctx, g):
        lf, lN = fctx.run.ctx.adjoint_backward(_np(g))
        return torch.from_numpy(lf).to(g.device), torch.from_numpy(lN).to(g.device), None


class _NexLoss(torch.autograd.Function):
    @staticmethod
    def forward(fctx, f0, N, run):
        run.forward(_np(f0), _np(N))
        J, lf, lN = run.ctx.adjoint_objective()
        fctx.run = run
        fctx.lam = (lf, lN)
        return torch.tensor(J, dtype=torch.float64, device=f0.device)

    @staticmethod
    def backward(fctx, gJ):
        lf, lN = fctx.lam
        # J depends on N directly (final deposit) and through the evolution
        lf0, lN0 = fctx.run.ctx.adjoint_backward(lf, lN)
        s = gJ.detach().to("cpu", torch.float64)
        dev = gJ.device
        return (torch.from_numpy(lf0).to(dev) * s).to(dev), (torch.from_numpy(lN0).to(dev) * s).to(dev), None


def evolve(f0, N, run):
    """final flavor state [n, 2nf^2] of the recorded run; differentiable in
    f0 through the adjoint (N enters the evolution only through the
    deposits, and its gradient is returned for N as well)"""
    return _Evolve.apply(f0, N, run)


def nex_loss(f0, N, run):
    """J = sum over cells of |N_emu|^2 / V_cell of the final state"""
    return _NexLoss.apply(f0, N, run)
