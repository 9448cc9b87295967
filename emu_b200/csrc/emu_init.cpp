// emu_init.cpp -- initial particle set on the host, restating
// FlavoredNeutrinoContainer::InitParticles
// (Source/FlavoredNeutrinoContainerInit.cpp:136-661) for simulation types
// 0-5, the latitude-ring direction generator uniform_sphere_xyz (:9-37), the
// Minerbo closure (:39-124), plus a Fibonacci-sphere generator.
//
// Randomness: the reference draws amrex::Random() from a clock-seeded
// generator (Source/main.cpp:240), so its runs are not reproducible.  Here
// every uniform draw is a counter-based hash of (seed, particle index, draw
// index), so an initial state is a pure function of the inputs.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "emu_b200.h"
#include "emu_host.h"

namespace {

const double kEV = 1.60218e-12;
const double kPi = 3.14159265358979323846;   // MathConst::pi

int herm_re(int nf, int i, int j)
{
    int base = 0;
    for (int r = 0; r < i; r++) base += 1 + 2 * (nf - 1 - r);
    return base + (j == i ? 0 : 1 + 2 * (j - i - 1));
}

double su_length(int nf, const double* f)
{
    double s = 0.0;
    for (int i = 0; i < nf; i++)
        for (int j = i + 1; j < nf; j++) {
            double a = f[herm_re(nf, i, j) + 1], b = f[herm_re(nf, i, j)];
            s = s + a * a;
            s = s + b * b;
        }
    for (int l = 1; l < nf; l++) {
        double cl = std::sqrt(2.0 / (l * (l + 1.0))) / 2.0;
        double t = 0.0;
        for (int i = 0; i < l; i++) t = t + cl * f[herm_re(nf, i, i)];
        t = t - (cl * l) * f[herm_re(nf, l, l)];
        s = s + t * t;
    }
    return std::sqrt(s);
}

// splitmix64 finaliser as a counter-based generator
uint64_t mix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t seed, particle, k = 0;
    double uniform()   // [0, 1)
    {
        uint64_t h = mix64(seed ^ mix64(particle * 0x100000001b3ull + (k++)));
        return (double)(h >> 11) * (1.0 / 9007199254740992.0);
    }
    double symmetric() { return 2. * (uniform() - 0.5); }   // Init.cpp:111-113
};

struct Dir { double x, y, z; };

// Init.cpp:9-37
std::vector<Dir> uniform_sphere_xyz(int nphi_at_equator)
{
    std::vector<Dir> xyz;
    if (nphi_at_equator <= 0) return xyz;
    double dtheta = M_PI * std::sqrt(3) / nphi_at_equator;
    double theta = 0;
    double phi0 = 0;
    while (theta < M_PI / 2.) {
        int nphi = theta == 0 ? nphi_at_equator : (int)std::lround(nphi_at_equator * std::cos(theta));
        double dphi = 2. * M_PI / nphi;
        if (nphi == 1) theta = M_PI / 2.;
        for (int iphi = 0; iphi < nphi; iphi++) {
            double phi = phi0 + iphi * dphi;
            double x = std::cos(theta) * std::cos(phi);
            double y = std::cos(theta) * std::sin(phi);
            double z = std::sin(theta);
            xyz.push_back({x, y, z});
            if (theta > 0) xyz.push_back({-x, -y, -z});
        }
        theta += dtheta;
        phi0 = phi0 + 0.5 * dphi;
    }
    return xyz;
}

// golden-angle spiral with n points of equal solid angle
std::vector<Dir> fibonacci_sphere(int n)
{
    std::vector<Dir> xyz;
    const double ga = M_PI * (3.0 - std::sqrt(5.0));
    for (int i = 0; i < n; i++) {
        double z = 1.0 - (2.0 * i + 1.0) / n;
        double r = std::sqrt(std::max(0.0, 1.0 - z * z));
        double phi = ga * i;
        xyz.push_back({r * std::cos(phi), r * std::sin(phi), z});
    }
    return xyz;
}

// Minerbo closure, Init.cpp:39-80 and 115-124
double minerbo_residual(double ff, double Z) { return ff - 1.0 / std::tanh(Z) + 1.0 / Z; }
double minerbo_residual_derivative(double, double Z) { return 1.0 / (std::sinh(Z) * std::sinh(Z)) - 1.0 / (Z * Z); }
bool minerbo_Z(double ff, double& Z)
{
    const double maxresidual = 1e-6, minfluxfac = 1e-3;
    const int maxcount = 20;
    Z = 1.0;
    if (ff < minfluxfac) {
        Z = 3. * ff;
        return true;
    }
    double residual = 1.0;
    int count = 0;
    while (std::abs(residual) > maxresidual && count < maxcount) {
        residual = minerbo_residual(ff, Z);
        double slope = minerbo_residual_derivative(ff, Z);
        Z -= residual / slope;
        count++;
    }
    return !(residual > maxresidual);
}
double minerbo_closure(double Z, double mu)
{
    double r = std::exp(Z * mu);
    if (Z / 3.0 > 1e-3) r *= Z / std::sinh(Z);
    return r;
}

}  // namespace

extern "C" int emu_init_particles(const emu_params* p, double* out, int64_t capacity, int64_t* n_out)
{
    if (!p || !n_out) return EMU_ERR_ARG;
    std::string why;
    if (!emu_host::validate(*p, why)) return EMU_ERR_ARG;
    const int nf = p->nflavors, nh = nf * nf;
    const int na = 8 + 2 * (2 + nh), nr = 3 + na;
    const double L[3] = {p->Lx, p->Ly, p->Lz};
    double dx[3];
    for (int d = 0; d < 3; d++) dx[d] = L[d] / (double)p->ncell[d];
    const int nlocs = p->nppc[0] * p->nppc[1] * p->nppc[2];
    std::vector<Dir> dirs = p->direction_generator == 1 ? fibonacci_sphere(p->ndirections)
                                                        : uniform_sphere_xyz(p->nphi_equator);
    const int ndirs = (int)dirs.size();
    if (ndirs == 0 || nlocs <= 0) return EMU_ERR_ARG;
    const double scale_fac = dx[0] * dx[1] * dx[2] / nlocs / ndirs;
    const long long ncells = (long long)p->ncell[0] * p->ncell[1] * p->ncell[2];
    const long long total = ncells * nlocs * ndirs;
    *n_out = total;
    if (!out) return EMU_OK;
    if (capacity < total) return EMU_ERR_ARG;

    double Ze = 0, Za = 0, Zx = 0, ffe = 0, ffa = 0, ffx = 0;
    if (p->simulation_type == 5) {
        ffe = std::sqrt(p->st5_fxnue * p->st5_fxnue + p->st5_fynue * p->st5_fynue + p->st5_fznue * p->st5_fznue);
        ffa = std::sqrt(p->st5_fxnua * p->st5_fxnua + p->st5_fynua * p->st5_fynua + p->st5_fznua * p->st5_fznua);
        ffx = std::sqrt(p->st5_fxnux * p->st5_fxnux + p->st5_fynux * p->st5_fynux + p->st5_fznux * p->st5_fznux);
        if (!minerbo_Z(ffe, Ze) || !minerbo_Z(ffa, Za) || !minerbo_Z(ffx, Zx)) return EMU_ERR_ARG;
    }
    const double c4 = emu_host::c4();
    const double hbarc = emu_host::hbarc();
    const double GF = emu_host::gf();

    long long pidx = 0;
    // cell order of the reference's tile loop: cellid = (i*ny + j)*nz + k
    for (int i = 0; i < p->ncell[0]; i++)
        for (int j = 0; j < p->ncell[1]; j++)
            for (int k = 0; k < p->ncell[2]; k++)
                for (int iloc = 0; iloc < nlocs; iloc++) {
                    // get_position_unit_cell (Init.cpp:84-97)
                    const int nx = p->nppc[0], ny = p->nppc[1], nz = p->nppc[2];
                    const int ix = iloc / (ny * nz), iy = (iloc % (ny * nz)) % ny, iz = (iloc % (ny * nz)) / ny;
                    const double r[3] = {(0.5 + ix) / nx, (0.5 + iy) / ny, (0.5 + iz) / nz};
                    const double x = 0.0 + (i + r[0]) * dx[0];
                    const double y = 0.0 + (j + r[1]) * dx[1];
                    const double z = 0.0 + (k + r[2]) * dx[2];
                    for (int idir = 0; idir < ndirs; idir++, pidx++) {
                        double* rec = out + pidx * nr;
                        std::memset(rec, 0, sizeof(double) * nr);
                        double* rd = rec + 3;
                        double* f = rd + 10;
                        double* fb = rd + 10 + nh + 2;
                        double& N = rd[8];
                        double& Nbar = rd[8 + 2 + nh];
                        rec[0] = x; rec[1] = y; rec[2] = z;
                        rd[1] = x; rd[2] = y; rd[3] = z;
                        rd[0] = 0;
                        const Dir u = dirs[idir];
                        Rng rng{p->seed, (uint64_t)pidx, 0};
                        const double dm2 = (p->mass2 - p->mass1) * (p->mass2 - p->mass1);
                        double pupt = 50. * 1e6 * kEV;
                        switch (p->simulation_type) {
                        case 0: {   // vacuum oscillation test (Init.cpp:321-359)
                            N = 1.0; Nbar = 1.0;
                            f[herm_re(nf, 0, 0)] = 1.0;
                            fb[herm_re(nf, 0, 0)] = 1.0;
                            pupt = dm2 * c4 * std::sin(2. * p->theta12) / (8. * M_PI * hbarc);
                            break;
                        }
                        case 1: {   // bipolar (Init.cpp:364-404)
                            f[0] = 1.0; fb[0] = 1.0;
                            const double ndens = 10. * dm2 * c4 / (2. * std::sqrt(2.) * GF * pupt);
                            N = ndens * scale_fac;
                            Nbar = ndens * scale_fac;
                            break;
                        }
                        case 2: {   // 2-beam fast flavor (Init.cpp:409-450)
                            f[0] = 1.0; fb[0] = 1.0;
                            const double omega = dm2 * c4 / (2. * pupt);
                            const double mu_ndens = std::sqrt(2.) * GF;
                            const double ndens = omega / (2. * mu_ndens);
                            N = ndens * scale_fac * (1. + u.z);
                            Nbar = ndens * scale_fac * (1. - u.z);
                            break;
                        }
                        case 3: {   // k != 0 fast flavor (Init.cpp:455-501)
                            const double lambda = L[2] / (double)p->st3_wavelength_fraction_of_domain;
                            const double kk = (2. * M_PI) / lambda;
                            f[0] = 1.0; fb[0] = 1.0;
                            f[herm_re(nf, 0, 1)] = p->st3_amplitude * std::sin(kk * z);
                            fb[herm_re(nf, 0, 1)] = p->st3_amplitude * std::sin(kk * z);
                            const double omega = dm2 * c4 / (2. * pupt);
                            const double mu_ndens = std::sqrt(2.) * GF;
                            const double ndens = (omega + kk * hbarc) / (2. * mu_ndens);
                            N = ndens * scale_fac * (1. + u.z);
                            Nbar = ndens * scale_fac * (1. - u.z);
                            break;
                        }
                        case 4: {   // randomized k != 0 (Init.cpp:506-569)
                            const double a = p->st4_amplitude;
                            const double r1 = rng.symmetric(), r2 = rng.symmetric(), r3 = rng.symmetric(),
                                         r4 = rng.symmetric();
                            f[0] = 1.0; fb[0] = 1.0;
                            f[herm_re(nf, 0, 1)] = a * r1;
                            f[herm_re(nf, 0, 1) + 1] = a * r2;
                            fb[herm_re(nf, 0, 1)] = a * r3;
                            fb[herm_re(nf, 0, 1) + 1] = a * r4;
                            if (nf == 3) {
                                const double s1 = rng.symmetric(), s2 = rng.symmetric(), s3 = rng.symmetric(),
                                             s4 = rng.symmetric();
                                f[herm_re(nf, 0, 2)] = a * s1;
                                f[herm_re(nf, 0, 2) + 1] = a * s2;
                                fb[herm_re(nf, 0, 2)] = a * s3;
                                fb[herm_re(nf, 0, 2) + 1] = a * s4;
                            }
                            const double fh[3] = {std::cos(p->st4_phi) * std::sin(p->st4_theta),
                                                  std::sin(p->st4_phi) * std::sin(p->st4_theta), std::cos(p->st4_theta)};
                            const double fhb[3] = {std::cos(p->st4_phibar) * std::sin(p->st4_thetabar),
                                                   std::sin(p->st4_phibar) * std::sin(p->st4_thetabar),
                                                   std::cos(p->st4_thetabar)};
                            const double ct = fh[0] * u.x + fh[1] * u.y + fh[2] * u.z;
                            const double ctb = fhb[0] * u.x + fhb[1] * u.y + fhb[2] * u.z;
                            N = p->st4_ndens * scale_fac * (1. + 3. * p->st4_fluxfac * ct);
                            Nbar = p->st4_ndensbar * scale_fac * (1. + 3. * p->st4_fluxfacbar * ctb);
                            break;
                        }
                        case 5: {   // Minerbo closure (Init.cpp:574-645)
                            const double mue = ffe > 0 ? (p->st5_fxnue * u.x + p->st5_fynue * u.y + p->st5_fznue * u.z) / ffe : 0;
                            const double mua = ffa > 0 ? (p->st5_fxnua * u.x + p->st5_fynua * u.y + p->st5_fznua * u.z) / ffa : 0;
                            const double mux = ffx > 0 ? (p->st5_fxnux * u.x + p->st5_fynux * u.y + p->st5_fznux * u.z) / ffx : 0;
                            const double Ne = p->st5_nnue * scale_fac * minerbo_closure(Ze, mue);
                            const double Na = p->st5_nnua * scale_fac * minerbo_closure(Za, mua);
                            const double Nx = p->st5_nnux * scale_fac * minerbo_closure(Zx, mux) / 4.0;
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
                            const double a = p->st5_amplitude;
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
                            return EMU_ERR_ARG;
                        }
                        if (p->simulation_type != 0) {
                            // sim types 1-5 use 50 MeV (sim type 0 set pupt above)
                        }
                        rd[7] = pupt;
                        rd[4] = u.x * pupt;
                        rd[5] = u.y * pupt;
                        rd[6] = u.z * pupt;
                        // set_trace_length fill (Init.cpp:651)
                        rd[9] = su_length(nf, f);
                        rd[9 + 2 + nh] = su_length(nf, fb);
                    }
                }
    (void)kPi;
    return EMU_OK;
}
