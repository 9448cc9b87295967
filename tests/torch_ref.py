"""Plain FP64 PyTorch version of one RK4 step of the evolution path (test
infrastructure): the gradient of its objective by torch autograd is the
reference for the library's hand-written adjoint.

Same semantics as the oracle (deposit_to_mesh Evolve.cpp:91-126,
interpolate_rhs_from_mesh Evolve.cpp:128-176 with the generated fills,
Renormalize generate_code.py:391-445, RK4 main.cpp:129-203), written with
differentiable torch operations on the flavor state and the N weights.
Stencils, vacuum potentials and positions are not differentiated; the
vacuum potential per particle comes from the oracle.
"""
import numpy as np
import torch

from emu_b200 import api
from oracle.oracle import Oracle

RK4_A = (0.5, 0.5, 1.0)
RK4_B = (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0)


def herm_re(nf, i, j):
    return i * (2 * nf - i) + (0 if j == i else 2 * (j - i) - 1)


def herm_im(nf, i, j):
    return herm_re(nf, i, j) + 1


class TorchEmu:
    def __init__(self, p, records):
        nf = p.nflavors
        self.nf, self.nh = nf, nf * nf
        self.o = Oracle(p)
        self.n = records.shape[0]
        self.ncell = np.array(p.ncell, dtype=np.int64)
        self.Ldom = np.array([p.Lx, p.Ly, p.Lz])
        dx = self.Ldom / self.ncell
        self.dxi = 1.0 / dx
        self.ord = [p.shape_order if self.ncell[d] > 1 else 0 for d in range(3)]
        self.inv_vol = float(np.prod(self.dxi))
        self.coef = np.sqrt(2.0) * api.GF * self.inv_vol
        self.matter = p.rho_in * p.Ye_in / api.MP / self.inv_vol
        self.inv_hbar = 1.0 / api.HBAR
        self.maxError = p.maxError
        pup = records[:, 3 + 4:3 + 8]
        self.v = pup[:, :3] / pup[:, 3:4]
        self.kxv = self.v * api.CLIGHT
        self.pos0 = records[:, 0:3].copy()
        self.vvac = torch.tensor(np.stack([self.o.vvac(float(t)) for t in pup[:, 3]]))
        nh = self.nh
        self.Lattr = torch.tensor(records[:, [3 + 9, 3 + 11 + nh]])
        self.vt = torch.tensor(self.v)
        im = torch.zeros(nh, dtype=torch.bool)
        for i in range(nf):
            for j in range(i + 1, nf):
                im[herm_im(nf, i, j)] = True
        self.is_im = im
        # Hermitian expansion: column gathers of [h, 0]
        ridx = np.zeros((nf, nf), dtype=np.int64)
        iidx = np.full((nf, nf), nh, dtype=np.int64)
        isgn = np.zeros((nf, nf))
        for i in range(nf):
            for j in range(nf):
                a, b = min(i, j), max(i, j)
                ridx[i, j] = herm_re(nf, a, b)
                if a != b:
                    iidx[i, j] = herm_im(nf, a, b)
                    isgn[i, j] = 1.0 if i < j else -1.0
        self.ridx = torch.tensor(ridx.reshape(-1))
        self.iidx = torch.tensor(iidx.reshape(-1))
        self.isgn = torch.tensor(isgn.reshape(-1))

    # ---- stencil (ParticleInterpolator.H) ----
    def stencil(self, pos):
        wid = [3 if o >= 2 else (2 if o == 1 else 1) for o in self.ord]
        first = np.zeros((self.n, 3), dtype=np.int64)
        w = np.zeros((self.n, 3, 3))
        for p in range(self.n):
            for d in range(3):
                f, wd = self.o.shape(pos[p, d] * self.dxi[d], self.ord[d])
                first[p, d] = f
                w[p, d, :] = wd
        idx, ww = [], []
        nx, ny, nz = self.ncell
        for kk in range(wid[2]):
            for jj in range(wid[1]):
                for ii in range(wid[0]):
                    i = np.mod(first[:, 0] + ii, nx)
                    j = np.mod(first[:, 1] + jj, ny)
                    k = np.mod(first[:, 2] + kk, nz)
                    idx.append((k * ny + j) * nx + i)
                    ww.append(w[:, 0, ii] * w[:, 1, jj] * w[:, 2, kk])
        return torch.tensor(np.stack(idx, 1)), torch.tensor(np.stack(ww, 1))

    # ---- deposit_to_mesh ----
    def deposit(self, f, N, st):
        idx, w = st
        nh = self.nh
        fN = torch.cat([f[:, :nh] * N[:, 0:1], f[:, nh:] * N[:, 1:2]], 1)
        vals = torch.cat([fN, fN * self.vt[:, 0:1], fN * self.vt[:, 1:2], fN * self.vt[:, 2:3]], 1)
        M = torch.zeros(int(np.prod(self.ncell)), 8 * nh, dtype=torch.float64)
        for s in range(idx.shape[1]):
            M = M.index_add(0, idx[:, s], w[:, s:s + 1] * vals)
        return M

    # ---- interpolated potential ----
    def potential(self, M, st):
        idx, w = st
        nh = self.nh
        vx, vy, vz = self.vt[:, 0:1], self.vt[:, 1:2], self.vt[:, 2:3]
        Vn, Vb = self.vvac[:, :nh], self.vvac[:, nh:]
        for s in range(idx.shape[1]):
            m = M[idx[:, s]]
            SI = m[:, 0:nh] - m[:, 2 * nh:3 * nh] * vx - m[:, 4 * nh:5 * nh] * vy - m[:, 6 * nh:7 * nh] * vz
            Sb = m[:, nh:2 * nh] - m[:, 3 * nh:4 * nh] * vx - m[:, 5 * nh:6 * nh] * vy - m[:, 7 * nh:8 * nh] * vz
            inside = torch.where(self.is_im, SI + Sb, SI - Sb)
            inside = torch.cat([inside[:, :1] + self.matter, inside[:, 1:]], 1)
            t = (self.coef * w[:, s:s + 1]) * inside
            Vn = Vn + t
            Vb = Vb + torch.where(self.is_im, t, -t)
        return torch.cat([Vn, Vb], 1)

    # ---- -i/hbar [H, F] in real components ----
    def _expand(self, h):
        nf = self.nf
        hz = torch.cat([h, torch.zeros(h.shape[0], 1, dtype=h.dtype)], 1)
        re = hz[:, self.ridx].reshape(-1, nf, nf)
        im = (hz[:, self.iidx] * self.isgn).reshape(-1, nf, nf)
        return torch.complex(re, im)

    def commutator(self, h, f):
        H, F = self._expand(h), self._expand(f)
        K = -1j * (H @ F - F @ H) * self.inv_hbar
        nf = self.nf
        cols = [None] * self.nh
        for i in range(nf):
            for j in range(i, nf):
                cols[herm_re(nf, i, j)] = K[:, i, j].real
                if j > i:
                    cols[herm_im(nf, i, j)] = K[:, i, j].imag
        return torch.stack(cols, 1)

    def rhs(self, f, M, st):
        V = self.potential(M, st)
        nh = self.nh
        return torch.cat([self.commutator(V[:, :nh], f[:, :nh]), self.commutator(V[:, nh:], f[:, nh:])], 1)

    # ---- Renormalize (branches as in the generated fill) ----
    def _su_length(self, f):
        nf = self.nf
        s = torch.zeros(f.shape[0], dtype=f.dtype)
        for i in range(nf):
            for j in range(i + 1, nf):
                s = s + f[:, herm_im(nf, i, j)] ** 2 + f[:, herm_re(nf, i, j)] ** 2
        for l in range(1, nf):
            cl = np.sqrt(2.0 / (l * (l + 1.0))) / 2.0
            t = torch.zeros_like(s)
            for i in range(l):
                t = t + cl * f[:, herm_re(nf, i, i)]
            t = t - (cl * l) * f[:, herm_re(nf, l, l)]
            s = s + t * t
        return torch.sqrt(s)

    def _renorm_species(self, f, L):
        nf, nh, me = self.nf, self.nh, self.maxError
        diag = [herm_re(nf, i, i) for i in range(nf)]
        cols = [f[:, e] for e in range(nh)]
        err = sum(cols[d] for d in diag) - 1.0
        tr = err.detach().abs() > me
        for d in diag:
            cols[d] = torch.where(tr, cols[d] - err / nf, cols[d])
        for d in diag:
            cols[d] = torch.where(cols[d].detach() < -me, torch.zeros_like(cols[d]), cols[d])
        f2 = torch.stack(cols, 1)
        length = self._su_length(f2)
        sc = ((length - L).detach().abs() > me).unsqueeze(1)
        return torch.where(sc, f2 / (length / L).unsqueeze(1), f2)

    def renormalize(self, f):
        nh = self.nh
        return torch.cat([self._renorm_species(f[:, :nh], self.Lattr[:, 0]),
                          self._renorm_species(f[:, nh:], self.Lattr[:, 1])], 1)

    # ---- one RK4 step, positions frozen during the stages ----
    def step(self, f, N, pos, dt):
        st = self.stencil(pos)
        Y0 = f
        K1 = self.rhs(Y0, self.deposit(Y0, N, st), st)
        Y2 = Y0 + (RK4_A[0] * dt) * K1
        K2 = self.rhs(Y2, self.deposit(Y2, N, st), st)
        Y3 = Y0 + (RK4_A[1] * dt) * K2
        K3 = self.rhs(Y3, self.deposit(Y3, N, st), st)
        Y4 = Y0 + (RK4_A[2] * dt) * K3
        K4 = self.rhs(Y4, self.deposit(Y4, N, st), st)
        Yn = Y0 + dt * (RK4_B[0] * K1 + RK4_B[1] * K2 + RK4_B[2] * K3 + RK4_B[3] * K4)
        x = pos.copy()
        for b in RK4_B:
            x = (dt * b) * self.kxv + x
        for d in range(3):
            L = self.Ldom[d]
            out = (x[:, d] >= L) | (x[:, d] < 0)
            xd = np.where(out, np.fmod(x[:, d], L), x[:, d])
            xd = np.where(xd < 0, xd + L, xd)
            x[:, d] = xd
        return self.renormalize(Yn), x

    def objective(self, f, N, pos):
        M = self.deposit(f, N, self.stencil(pos))
        k1, k2 = herm_re(self.nf, 0, 1), herm_im(self.nf, 0, 1)
        return self.inv_vol * (M[:, k1] ** 2 + M[:, k2] ** 2).sum()

    def loss(self, f0, N, dts):
        f, pos = f0, self.pos0
        for dt in dts:
            f, pos = self.step(f, N, pos, float(dt))
        return self.objective(f, N, pos)
