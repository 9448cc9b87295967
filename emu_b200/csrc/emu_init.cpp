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
#include "emu_init_record.h"

namespace {

const double kEV = 1.60218e-12;

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

}  // namespace

// The generator's inputs: everything the record of one particle depends on,
// with the per-run transcendental factors evaluated once here.
bool emu_host::make_init_spec(const emu_params& p, emu_init::InitSpec& s, std::vector<double>& dirs,
                              long long& total, std::string& why)
{
    if (!validate(p, why)) return false;
    std::memset(&s, 0, sizeof(s));
    const int nf = p.nflavors, nh = nf * nf;
    s.nf = nf;
    s.nr = 3 + 8 + 2 * (2 + nh);
    const double L[3] = {p.Lx, p.Ly, p.Lz};
    for (int d = 0; d < 3; d++) {
        s.ncell[d] = p.ncell[d];
        s.nppc[d] = p.nppc[d];
        s.dx[d] = L[d] / (double)p.ncell[d];
    }
    s.nlocs = p.nppc[0] * p.nppc[1] * p.nppc[2];
    std::vector<Dir> dv = p.direction_generator == 1 ? fibonacci_sphere(p.ndirections)
                                                     : uniform_sphere_xyz(p.nphi_equator);
    s.ndirs = (int)dv.size();
    if (s.ndirs == 0 || s.nlocs <= 0) {
        why = "no directions or no particles per cell";
        return false;
    }
    dirs.resize(3 * dv.size());
    for (size_t q = 0; q < dv.size(); q++) {
        dirs[3 * q] = dv[q].x;
        dirs[3 * q + 1] = dv[q].y;
        dirs[3 * q + 2] = dv[q].z;
    }
    s.scale_fac = s.dx[0] * s.dx[1] * s.dx[2] / s.nlocs / s.ndirs;
    total = (long long)p.ncell[0] * p.ncell[1] * p.ncell[2] * s.nlocs * s.ndirs;
    s.simulation_type = p.simulation_type;
    if (s.simulation_type < 0 || s.simulation_type > 5) {
        why = "simulation_type must be 0-5";
        return false;
    }
    s.seed = p.seed;
    s.c4 = c4();
    s.hbarc = hbarc();
    s.GF = gf();
    s.dm2 = (p.mass2 - p.mass1) * (p.mass2 - p.mass1);
    s.pupt = 50. * 1e6 * kEV;
    if (s.simulation_type == 0) s.pupt = s.dm2 * s.c4 * std::sin(2. * p.theta12) / (8. * M_PI * s.hbarc);
    s.st3_amplitude = p.st3_amplitude;
    if (p.st3_wavelength_fraction_of_domain != 0) {
        const double lambda = L[2] / (double)p.st3_wavelength_fraction_of_domain;
        s.st3_k = (2. * M_PI) / lambda;
    }
    s.st4_fh[0] = std::cos(p.st4_phi) * std::sin(p.st4_theta);
    s.st4_fh[1] = std::sin(p.st4_phi) * std::sin(p.st4_theta);
    s.st4_fh[2] = std::cos(p.st4_theta);
    s.st4_fhb[0] = std::cos(p.st4_phibar) * std::sin(p.st4_thetabar);
    s.st4_fhb[1] = std::sin(p.st4_phibar) * std::sin(p.st4_thetabar);
    s.st4_fhb[2] = std::cos(p.st4_thetabar);
    s.st4_ndens = p.st4_ndens;
    s.st4_ndensbar = p.st4_ndensbar;
    s.st4_fluxfac = p.st4_fluxfac;
    s.st4_fluxfacbar = p.st4_fluxfacbar;
    s.st4_amplitude = p.st4_amplitude;
    if (s.simulation_type == 5) {
        const double F[3][3] = {{p.st5_fxnue, p.st5_fynue, p.st5_fznue},
                                {p.st5_fxnua, p.st5_fynua, p.st5_fznua},
                                {p.st5_fxnux, p.st5_fynux, p.st5_fznux}};
        const double n[3] = {p.st5_nnue, p.st5_nnua, p.st5_nnux};
        for (int q = 0; q < 3; q++) {
            for (int d = 0; d < 3; d++) s.st5_f[q][d] = F[q][d];
            s.st5_ff[q] = std::sqrt(F[q][0] * F[q][0] + F[q][1] * F[q][1] + F[q][2] * F[q][2]);
            s.st5_n[q] = n[q];
            if (!minerbo_Z(s.st5_ff[q], s.st5_Z[q])) {
                why = "Minerbo closure: no solution for the flux factor";
                return false;
            }
            s.st5_norm[q] = s.st5_Z[q] / std::sinh(s.st5_Z[q]);
        }
        s.st5_amplitude = p.st5_amplitude;
    }
    return true;
}

extern "C" int emu_init_particles(const emu_params* p, double* out, int64_t capacity, int64_t* n_out)
{
    if (!p || !n_out) return EMU_ERR_ARG;
    emu_init::InitSpec s;
    std::vector<double> dirs;
    long long total = 0;
    std::string why;
    if (!emu_host::make_init_spec(*p, s, dirs, total, why)) {
        emu_host::set_error("emu_init_particles: " + why);
        return EMU_ERR_ARG;
    }
    *n_out = total;
    if (!out) return EMU_OK;
    if (capacity < total) return EMU_ERR_ARG;
    for (long long q = 0; q < total; q++)
        if (!emu_init::init_record(s, dirs.data(), q, out + q * s.nr)) return EMU_ERR_ARG;
    return EMU_OK;
}
