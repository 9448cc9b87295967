"""Initial particle records, restated in numpy -- TEST INFRASTRUCTURE ONLY.

The CPU legs of bench.py (the reference arm and the cpu_baseline sample) need
the same initial particles as the CUDA path without loading the CUDA
library, and the tests pin this restatement to the library's generator
(emu_init_particles) bit for bit.  It covers what the benchmark workloads
use: simulation type 4, "randomized k != 0" (Source/
FlavoredNeutrinoContainerInit.cpp:506-569), with the latitude-ring direction
set uniform_sphere_xyz (:9-37) or a Fibonacci sphere, particle positions of
get_position_unit_cell (:84-97) and the SU(n) lengths of the
set_trace_length fill (:651).

Randomness: the reference seeds amrex::Random() from the clock
(Source/main.cpp:240), so its initial states are not reproducible; the
library draws every uniform number as a counter-based hash of (seed,
particle index, draw index) (splitmix64 finaliser), restated here with
numpy's wrapping uint64 arithmetic.

`params` is any object with the emu_params field names (an
emu_b200.api.EmuParams, or a types.SimpleNamespace).
"""
import math

import numpy as np

EV = 1.60218e-12          # Source/Constants.H


def uniform_sphere_xyz(nphi_at_equator):
    """Latitude rings (FlavoredNeutrinoContainerInit.cpp:9-37)."""
    xyz = []
    if nphi_at_equator <= 0:
        return np.zeros((0, 3))
    dtheta = math.pi * math.sqrt(3) / nphi_at_equator
    theta = 0.0
    phi0 = 0.0
    while theta < math.pi / 2.:
        nphi = nphi_at_equator if theta == 0 else int(_lround(nphi_at_equator * math.cos(theta)))
        dphi = 2. * math.pi / nphi if nphi else math.inf   # (a ring of 0: IEEE division, no directions)
        if nphi == 1:
            theta = math.pi / 2.
        for iphi in range(nphi):
            phi = phi0 + iphi * dphi
            x = math.cos(theta) * math.cos(phi)
            y = math.cos(theta) * math.sin(phi)
            z = math.sin(theta)
            xyz.append((x, y, z))
            if theta > 0:
                xyz.append((-x, -y, -z))
        theta += dtheta
        phi0 = phi0 + 0.5 * dphi
    return np.array(xyz, dtype=np.float64)


def _lround(v):
    """C lround: halfway cases away from zero."""
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)


def fibonacci_sphere(n):
    """Golden-angle spiral of n directions of equal solid angle."""
    ga = math.pi * (3.0 - math.sqrt(5.0))
    out = np.zeros((n, 3))
    for i in range(n):
        z = 1.0 - (2.0 * i + 1.0) / n
        r = math.sqrt(max(0.0, 1.0 - z * z))
        phi = ga * i
        out[i] = (r * math.cos(phi), r * math.sin(phi), z)
    return out


_M1 = np.uint64(0x9e3779b97f4a7c15)
_M2 = np.uint64(0xbf58476d1ce4e5b9)
_M3 = np.uint64(0x94d049bb133111eb)
_FNV = np.uint64(0x100000001b3)


def _mix64(z):
    z = z + _M1
    z = (z ^ (z >> np.uint64(30))) * _M2
    z = (z ^ (z >> np.uint64(27))) * _M3
    return z ^ (z >> np.uint64(31))


def _uniform(seed, pidx, k):
    """The k-th uniform draw in [0, 1) of every particle in pidx."""
    with np.errstate(over="ignore"):
        h = _mix64(np.uint64(seed) ^ _mix64(pidx * _FNV + np.uint64(k)))
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _symmetric(seed, pidx, k):
    return 2. * (_uniform(seed, pidx, k) - 0.5)


def _herm_re(nf, i, j):
    return i * (2 * nf - i) + (0 if j == i else 2 * (j - i) - 1)


def su_length(nf, f):
    """SU(n) vector length per row of f (HermitianUtils.py:102-123), in the
    generated expression's summation order."""
    s = np.zeros(f.shape[0])
    for i in range(nf):
        for j in range(i + 1, nf):
            a = f[:, _herm_re(nf, i, j) + 1]
            b = f[:, _herm_re(nf, i, j)]
            s = s + a * a
            s = s + b * b
    for l in range(1, nf):
        cl = 0.5 if l == 1 else 0.28867513459481287
        t = np.zeros(f.shape[0])
        for i in range(l):
            t = t + cl * f[:, _herm_re(nf, i, i)]
        t = t - (cl * l) * f[:, _herm_re(nf, l, l)]
        s = s + t * t
    return np.sqrt(s)


def directions(p):
    if p.direction_generator == 1:
        return fibonacci_sphere(p.ndirections)
    return uniform_sphere_xyz(p.nphi_equator)


def init_particles(p):
    """(n, 3 + nattribs) FP64 records in the library's order (cell (i, j, k)
    with cellid = (i ny + j) nz + k, then position in the cell, then
    direction), simulation type 4 only."""
    if p.simulation_type != 4:
        raise NotImplementedError("oracle.ic restates simulation type 4 only")
    nf = p.nflavors
    nh = nf * nf
    nr = 3 + 8 + 2 * (2 + nh)
    ncell = [int(p.ncell[d]) for d in range(3)]
    nppc = [int(p.nppc[d]) for d in range(3)]
    L = [p.Lx, p.Ly, p.Lz]
    dx = [L[d] / float(ncell[d]) for d in range(3)]
    nlocs = nppc[0] * nppc[1] * nppc[2]
    dirs = directions(p)
    ndirs = dirs.shape[0]
    scale_fac = dx[0] * dx[1] * dx[2] / nlocs / ndirs
    total = ncell[0] * ncell[1] * ncell[2] * nlocs * ndirs
    pidx = np.arange(total, dtype=np.int64)
    per_cell = nlocs * ndirs
    cellid = pidx // per_cell
    iloc = (pidx // ndirs) % nlocs
    idir = pidx % ndirs
    k = cellid % ncell[2]
    j = (cellid // ncell[2]) % ncell[1]
    i = cellid // (ncell[2] * ncell[1])
    nx, ny, nz = nppc
    ix = iloc // (ny * nz)
    iy = (iloc % (ny * nz)) % ny
    iz = (iloc % (ny * nz)) // ny
    x = 0.0 + (i + (0.5 + ix) / nx) * dx[0]
    y = 0.0 + (j + (0.5 + iy) / ny) * dx[1]
    z = 0.0 + (k + (0.5 + iz) / nz) * dx[2]
    rec = np.zeros((total, nr))
    rec[:, 0], rec[:, 1], rec[:, 2] = x, y, z
    rd = 3
    rec[:, rd + 1], rec[:, rd + 2], rec[:, rd + 3] = x, y, z
    ux, uy, uz = dirs[idir, 0], dirs[idir, 1], dirs[idir, 2]
    f = rd + 10                  # first nu flavor real
    fb = rd + 10 + nh + 2        # first nubar flavor real
    upid = pidx.astype(np.uint64)
    a = p.st4_amplitude
    draws = [_symmetric(p.seed, upid, kk) for kk in range(8 if nf == 3 else 4)]
    rec[:, f] = 1.0
    rec[:, fb] = 1.0
    o01 = _herm_re(nf, 0, 1)
    rec[:, f + o01] = a * draws[0]
    rec[:, f + o01 + 1] = a * draws[1]
    rec[:, fb + o01] = a * draws[2]
    rec[:, fb + o01 + 1] = a * draws[3]
    if nf == 3:
        o02 = _herm_re(nf, 0, 2)
        rec[:, f + o02] = a * draws[4]
        rec[:, f + o02 + 1] = a * draws[5]
        rec[:, fb + o02] = a * draws[6]
        rec[:, fb + o02 + 1] = a * draws[7]
    fh = (math.cos(p.st4_phi) * math.sin(p.st4_theta), math.sin(p.st4_phi) * math.sin(p.st4_theta),
          math.cos(p.st4_theta))
    fhb = (math.cos(p.st4_phibar) * math.sin(p.st4_thetabar), math.sin(p.st4_phibar) * math.sin(p.st4_thetabar),
           math.cos(p.st4_thetabar))
    ct = fh[0] * ux + fh[1] * uy + fh[2] * uz
    ctb = fhb[0] * ux + fhb[1] * uy + fhb[2] * uz
    rec[:, rd + 8] = p.st4_ndens * scale_fac * (1. + 3. * p.st4_fluxfac * ct)
    rec[:, rd + 8 + 2 + nh] = p.st4_ndensbar * scale_fac * (1. + 3. * p.st4_fluxfacbar * ctb)
    pupt = 50. * 1e6 * EV
    rec[:, rd + 7] = pupt
    rec[:, rd + 4] = ux * pupt
    rec[:, rd + 5] = uy * pupt
    rec[:, rd + 6] = uz * pupt
    rec[:, rd + 9] = su_length(nf, rec[:, f:f + nh])
    rec[:, rd + 9 + 2 + nh] = su_length(nf, rec[:, fb:fb + nh])
    return rec
