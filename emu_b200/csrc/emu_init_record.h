// emu_init_record.h -- one initial particle record of
// FlavoredNeutrinoContainer::InitParticles
// (Source/FlavoredNeutrinoContainerInit.cpp:136-661), shared by the host
// generator (emu_init.cpp) and the device generator (emu_capi.cu): the record
// of global particle index pidx is a pure function of (InitSpec, pidx).
//
// Particle order of the reference's tile loop: cell (i, j, k) with
// cellid = (i*ny + j)*nz + k, then position in the cell, then direction.
// Randomness: every uniform draw is a counter-based hash of (seed, particle
// index, draw index) (the reference seeds from the clock, main.cpp:240).
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define EMU_HD __host__ __device__
#else
#define EMU_HD
#endif

namespace emu_init {

struct InitSpec {
    int nf, nr;
    int ncell[3], nppc[3];
    int nlocs, ndirs;
    int simulation_type;
    uint64_t seed;
    double dx[3];
    double scale_fac;
    double pupt;                    // 50 MeV (sim types 1-5), or the sim type 0 energy
    double dm2, c4;                 // (m2 - m1)^2, c^4
    double GF, hbarc;
    // sim type 3
    double st3_k, st3_amplitude;
    // sim type 4 (flux directions precomputed)
    double st4_fh[3], st4_fhb[3];
    double st4_ndens, st4_ndensbar, st4_fluxfac, st4_fluxfacbar, st4_amplitude;
    // sim type 5 (Minerbo: Z, Z/sinh(Z) factor, flux factor, flux vector per species e, a, x)
    double st5_n[3], st5_Z[3], st5_norm[3], st5_ff[3], st5_f[3][3], st5_amplitude;
};

EMU_HD inline int herm_re(int nf, int i, int j)
{
    return i * (2 * nf - i) + (j == i ? 0 : 2 * (j - i) - 1);
}

// SU(n) vector length (HermitianUtils.py:102-123), generated expression order
EMU_HD inline double su_length(int nf, const double* f)
{
    double s = 0.0;
    for (int i = 0; i < nf; i++)
        for (int j = i + 1; j < nf; j++) {
            double a = f[herm_re(nf, i, j) + 1], b = f[herm_re(nf, i, j)];
            s = s + a * a;
            s = s + b * b;
        }
    for (int l = 1; l < nf; l++) {
        double cl = (l == 1) ? 0.5 : 0.28867513459481287;   // sqrt(2/(l(l+1)))/2
        double t = 0.0;
        for (int i = 0; i < l; i++) t = t + cl * f[herm_re(nf, i, i)];
        t = t - (cl * l) * f[herm_re(nf, l, l)];
        s = s + t * t;
    }
    return sqrt(s);
}

// splitmix64 finaliser as a counter-based generator
EMU_HD inline uint64_t mix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t seed, particle, k;
    EMU_HD double uniform()   // [0, 1)
    {
        uint64_t h = mix64(seed ^ mix64(particle * 0x100000001b3ull + (k++)));
        return (double)(h >> 11) * (1.0 / 9007199254740992.0);
    }
    EMU_HD double symmetric() { return 2. * (uniform() - 0.5); }   // Init.cpp:111-113
};

// rec: 3 + nattribs doubles (zeroed here); dirs: 3 * ndirs unit vectors.
// Returns false for an unknown simulation type.
EMU_HD inline bool init_record(const InitSpec& s, const double* dirs, long long pidx, double* rec)
{
    const int nf = s.nf, nh = nf * nf;
    const long long per_cell = (long long)s.nlocs * s.ndirs;
    const long long cellid = pidx / per_cell;
    const int iloc = (int)((pidx / s.ndirs) % s.nlocs);
    const int idir = (int)(pidx % s.ndirs);
    const int k = (int)(cellid % s.ncell[2]);
    const int j = (int)((cellid / s.ncell[2]) % s.ncell[1]);
    const int i = (int)(cellid / ((long long)s.ncell[2] * s.ncell[1]));
    // get_position_unit_cell (Init.cpp:84-97)
    const int nx = s.nppc[0], ny = s.nppc[1], nz = s.nppc[2];
    const int ix = iloc / (ny * nz), iy = (iloc % (ny * nz)) % ny, iz = (iloc % (ny * nz)) / ny;
    const double x = 0.0 + (i + (0.5 + ix) / nx) * s.dx[0];
    const double y = 0.0 + (j + (0.5 + iy) / ny) * s.dx[1];
    const double z = 0.0 + (k + (0.5 + iz) / nz) * s.dx[2];
    for (int c = 0; c < s.nr; c++) rec[c] = 0.0;
    double* rd = rec + 3;
    double* f = rd + 10;
    double* fb = rd + 10 + nh + 2;
    double& N = rd[8];
    double& Nbar = rd[8 + 2 + nh];
    rec[0] = x; rec[1] = y; rec[2] = z;
    rd[1] = x; rd[2] = y; rd[3] = z;
    const double ux = dirs[3 * idir], uy = dirs[3 * idir + 1], uz = dirs[3 * idir + 2];
    Rng rng{s.seed, (uint64_t)pidx, 0};
    switch (s.simulation_type) {
    case 0:   // vacuum oscillation test (Init.cpp:321-359)
        N = 1.0; Nbar = 1.0;
        f[herm_re(nf, 0, 0)] = 1.0;
        fb[herm_re(nf, 0, 0)] = 1.0;
        break;
    case 1: {   // bipolar (Init.cpp:364-404)
        f[0] = 1.0; fb[0] = 1.0;
        const double ndens = 10. * s.dm2 * s.c4 / (2. * sqrt(2.) * s.GF * s.pupt);
        N = ndens * s.scale_fac;
        Nbar = ndens * s.scale_fac;
        break;
    }
    case 2: {   // 2-beam fast flavor (Init.cpp:409-450)
        f[0] = 1.0; fb[0] = 1.0;
        const double omega = s.dm2 * s.c4 / (2. * s.pupt);
        const double mu_ndens = sqrt(2.) * s.GF;
        const double ndens = omega / (2. * mu_ndens);
        N = ndens * s.scale_fac * (1. + uz);
        Nbar = ndens * s.scale_fac * (1. - uz);
        break;
    }
    case 3: {   // k != 0 fast flavor (Init.cpp:455-501)
        f[0] = 1.0; fb[0] = 1.0;
        f[herm_re(nf, 0, 1)] = s.st3_amplitude * sin(s.st3_k * z);
        fb[herm_re(nf, 0, 1)] = s.st3_amplitude * sin(s.st3_k * z);
        const double omega = s.dm2 * s.c4 / (2. * s.pupt);
        const double mu_ndens = sqrt(2.) * s.GF;
        const double ndens = (omega + s.st3_k * s.hbarc) / (2. * mu_ndens);
        N = ndens * s.scale_fac * (1. + uz);
        Nbar = ndens * s.scale_fac * (1. - uz);
        break;
    }
    case 4: {   // randomized k != 0 (Init.cpp:506-569)
        const double a = s.st4_amplitude;
        const double r1 = rng.symmetric(), r2 = rng.symmetric(), r3 = rng.symmetric(), r4 = rng.symmetric();
        f[0] = 1.0; fb[0] = 1.0;
        f[herm_re(nf, 0, 1)] = a * r1;
        f[herm_re(nf, 0, 1) + 1] = a * r2;
        fb[herm_re(nf, 0, 1)] = a * r3;
        fb[herm_re(nf, 0, 1) + 1] = a * r4;
        if (nf == 3) {
            const double s1 = rng.symmetric(), s2 = rng.symmetric(), s3 = rng.symmetric(), s4 = rng.symmetric();
            f[herm_re(nf, 0, 2)] = a * s1;
            f[herm_re(nf, 0, 2) + 1] = a * s2;
            fb[herm_re(nf, 0, 2)] = a * s3;
            fb[herm_re(nf, 0, 2) + 1] = a * s4;
        }
        const double ct = s.st4_fh[0] * ux + s.st4_fh[1] * uy + s.st4_fh[2] * uz;
        const double ctb = s.st4_fhb[0] * ux + s.st4_fhb[1] * uy + s.st4_fhb[2] * uz;
        N = s.st4_ndens * s.scale_fac * (1. + 3. * s.st4_fluxfac * ct);
        Nbar = s.st4_ndensbar * s.scale_fac * (1. + 3. * s.st4_fluxfacbar * ctb);
        break;
    }
    case 5: {   // Minerbo closure (Init.cpp:574-645)
        double nsp[3];
        for (int q = 0; q < 3; q++) {
            const double mu = s.st5_ff[q] > 0
                                  ? (s.st5_f[q][0] * ux + s.st5_f[q][1] * uy + s.st5_f[q][2] * uz) / s.st5_ff[q]
                                  : 0;
            double r = exp(s.st5_Z[q] * mu);
            if (s.st5_Z[q] / 3.0 > 1e-3) r *= s.st5_norm[q];
            nsp[q] = s.st5_n[q] * s.scale_fac * r;
        }
        const double Ne = nsp[0], Na = nsp[1], Nx = nsp[2] / 4.0;
        N = Ne + Nx;
        Nbar = Na + Nx;
        if (nf == 3) { N += Nx; Nbar += Nx; }
        const int d0 = herm_re(nf, 0, 0), d1 = herm_re(nf, 1, 1);
        f[d0] = Ne / N; f[d1] = Nx / N;
        fb[d0] = Na / Nbar; fb[d1] = Nx / Nbar;
        int d2 = -1;
        if (nf == 3) {
            d2 = herm_re(nf, 2, 2);
            f[d2] = Nx / N;
            fb[d2] = Nx / Nbar;
        }
        const double a = s.st5_amplitude;
        const int o01 = herm_re(nf, 0, 1);
        f[o01] = a * rng.symmetric() * (f[d0] - f[d1]);
        f[o01 + 1] = a * rng.symmetric() * (f[d0] - f[d1]);
        fb[o01] = a * rng.symmetric() * (fb[d0] - fb[d1]);
        fb[o01 + 1] = a * rng.symmetric() * (fb[d0] - fb[d1]);
        if (nf == 3) {
            const int o02 = herm_re(nf, 0, 2), o12 = herm_re(nf, 1, 2);
            f[o02] = a * rng.symmetric() * (f[d0] - f[d2]);
            f[o02 + 1] = a * rng.symmetric() * (f[d0] - f[d2]);
            f[o12] = a * rng.symmetric() * (f[d1] - f[d2]);
            f[o12 + 1] = a * rng.symmetric() * (f[d1] - f[d2]);
            fb[o02] = a * rng.symmetric() * (fb[d0] - fb[d2]);
            fb[o02 + 1] = a * rng.symmetric() * (fb[d0] - fb[d2]);
            fb[o12] = a * rng.symmetric() * (fb[d1] - fb[d2]);
            fb[o12 + 1] = a * rng.symmetric() * (fb[d1] - fb[d2]);
        }
        break;
    }
    default:
        return false;
    }
    rd[7] = s.pupt;
    rd[4] = ux * s.pupt;
    rd[5] = uy * s.pupt;
    rd[6] = uz * s.pupt;
    // set_trace_length fill (Init.cpp:651)
    rd[9] = su_length(nf, f);
    rd[9 + 2 + nh] = su_length(nf, fb);
    return true;
}

}  // namespace emu_init
