/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Runs the reference's own per-particle arithmetic on the CPU: the kernel
 * bodies that Emu's generator (Scripts/symbolic_hermitians/generate_code.py N)
 * writes into Source/generated_files/, plus Source/ParticleInterpolator.H and
 * Source/Constants.H, all #included unmodified from where they lie.  The
 * AMReX machinery around those bodies (ParticleToMesh with ghost cells and
 * SumBoundary, FillBoundary, MeshToParticle, the Runge-Kutta TimeIntegrator,
 * periodic Redistribute, ReduceOps) is absent from the reference tree (empty
 * amrex submodule) and is restated here in plain loops.
 *
 * Built by oracle/build_oracle.py into oracle/_ref/libemuref<N>.so, once per
 * NUM_FLAVORS, since the generated bodies are flavor-specific.  The exported
 * functions mirror oracle/emu_oracle.h with the prefix ref_.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <sstream>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "emu_oracle.h"

#include "Constants.H"            /* reference Source/Constants.H */
#include "ParticleInterpolator.H" /* reference Source/ParticleInterpolator.H */

using amrex::Real;
using std::max;

/* error recording for the generated Renormalize body (amrex::Error aborts in
 * the reference; here it records which check fired) */
static thread_local int g_err = 0;
namespace amrex {
inline void Error(const std::string& msg)
{
    if (msg.rfind("Matrix trace", 0) == 0) g_err |= ORACLE_ERR_TRACE;
    else if (msg.rfind("Diagonal element", 0) == 0) g_err |= ORACLE_ERR_NEGDIAG;
    else if (msg.rfind("flavor vector length", 0) == 0) g_err |= ORACLE_ERR_LENGTH;
    else g_err |= 64;
}
namespace Gpu { namespace Atomic {
inline void AddNoRet(double* p, double v) { *p += v; }
}}  // namespace Gpu::Atomic
}  // namespace amrex

struct PIdx {
    enum {
        time = 0, x, y, z, pupx, pupy, pupz, pupt,
#include "generated_files/FlavoredNeutrinoContainer.H_fill"
        nattribs
    };
};

namespace GIdx {
enum {
    rho, T, Ye,
#include "generated_files/Evolve.H_fill"
    ncomp
};
}

/* the fields of TestParams (Source/Parameters.H:11-50) that the bodies read */
struct HParams {
    Real mass1, mass2, mass3, theta12, theta13, theta23, alpha1, alpha2, deltaCP, maxError;
};

static HParams to_hparams(const oracle_params* P)
{
    HParams h;
    h.mass1 = P->mass1; h.mass2 = P->mass2; h.mass3 = P->mass3;
    h.theta12 = P->theta12; h.theta13 = P->theta13; h.theta23 = P->theta23;
    h.alpha1 = P->alpha1; h.alpha2 = P->alpha2; h.deltaCP = P->deltaCP;
    h.maxError = P->maxError;
    return h;
}

/* particle record view: [pos_x,pos_y,pos_z, rdata...] */
struct PView {
    double* d;
    double& pos(int i) const { return d[i]; }
    double& rdata(int i) const { return d[3 + i]; }
};

static const int NREAL = 3 + PIdx::nattribs;

/* grown single-box fab, (i,j,k,n) with i fastest, n slowest (Array4 order) */
struct Fab {
    int ng[3], n[3], len[3];
    int ncomp;
    std::vector<double> v;
    void define(const int ncell[3], const int ngrow[3], int nc)
    {
        for (int d = 0; d < 3; d++) { ng[d] = ngrow[d]; n[d] = ncell[d]; len[d] = n[d] + 2 * ng[d]; }
        ncomp = nc;
        v.assign((size_t)len[0] * len[1] * len[2] * nc, 0.0);
    }
    size_t at(int i, int j, int k, int c) const
    {
        return (((size_t)c * len[2] + (k + ng[2])) * len[1] + (j + ng[1])) * len[0] + (i + ng[0]);
    }
};

struct FabArr {   /* Array4-like accessor with a component offset (make_alias) */
    Fab* f;
    int c0;
    double& operator()(int i, int j, int k, int c) const { return f->v[f->at(i, j, k, c0 + c)]; }
};

static int wrapi(int a, int n) { int r = a % n; return r < 0 ? r + n : r; }

struct Geo {
    int ord[3], ngrow[3];
    Real dx[3], dxi[3], plo[3];
};

static Geo make_geo(const oracle_params* P)
{
    Geo g;
    Real L[3] = {P->Lx, P->Ly, P->Lz};
    for (int d = 0; d < 3; d++) {
        g.ord[d] = P->ncell[d] > 1 ? P->shape_order : 0;         /* Evolve.cpp:102-104, 134-136 */
        g.ngrow[d] = 1 + (1 + (P->ncell[d] == 1 ? 0 : P->shape_order)) / 2;  /* main.cpp:68-71 */
        g.dx[d] = L[d] / (Real)P->ncell[d];
        g.dxi[d] = 1.0 / g.dx[d];
        g.plo[d] = 0.0;
    }
    return g;
}

/* SumBoundary with periodicity: add every ghost cell into its periodic image */
static void sum_boundary(Fab& F, int c_lo, int c_hi)
{
    for (int c = c_lo; c < c_hi; c++)
        for (int k = -F.ng[2]; k < F.n[2] + F.ng[2]; k++)
            for (int j = -F.ng[1]; j < F.n[1] + F.ng[1]; j++)
                for (int i = -F.ng[0]; i < F.n[0] + F.ng[0]; i++) {
                    bool valid = i >= 0 && i < F.n[0] && j >= 0 && j < F.n[1] && k >= 0 && k < F.n[2];
                    if (valid) continue;
                    F.v[F.at(wrapi(i, F.n[0]), wrapi(j, F.n[1]), wrapi(k, F.n[2]), c)] += F.v[F.at(i, j, k, c)];
                }
}

/* FillBoundary with periodicity: ghost cells take their image's value */
static void fill_boundary(Fab& F)
{
    for (int c = 0; c < F.ncomp; c++)
        for (int k = -F.ng[2]; k < F.n[2] + F.ng[2]; k++)
            for (int j = -F.ng[1]; j < F.n[1] + F.ng[1]; j++)
                for (int i = -F.ng[0]; i < F.n[0] + F.ng[0]; i++) {
                    bool valid = i >= 0 && i < F.n[0] && j >= 0 && j < F.n[1] && k >= 0 && k < F.n[2];
                    if (valid) continue;
                    F.v[F.at(i, j, k, c)] = F.v[F.at(wrapi(i, F.n[0]), wrapi(j, F.n[1]), wrapi(k, F.n[2]), c)];
                }
}

static void fab_from_mesh(Fab& F, const oracle_params* P, const double* mesh)
{
    Geo g = make_geo(P);
    F.define(P->ncell, g.ngrow, GIdx::ncomp);
    int64_t nc = (int64_t)P->ncell[0] * P->ncell[1] * P->ncell[2];
    for (int c = 0; c < GIdx::ncomp; c++)
        for (int k = 0; k < P->ncell[2]; k++)
            for (int j = 0; j < P->ncell[1]; j++)
                for (int i = 0; i < P->ncell[0]; i++)
                    F.v[F.at(i, j, k, c)] = mesh[c * nc + ((int64_t)k * P->ncell[1] + j) * P->ncell[0] + i];
    fill_boundary(F);
}

static void mesh_from_fab(const Fab& F, const oracle_params* P, double* mesh, int c_lo)
{
    int64_t nc = (int64_t)P->ncell[0] * P->ncell[1] * P->ncell[2];
    for (int c = c_lo; c < GIdx::ncomp; c++)
        for (int k = 0; k < P->ncell[2]; k++)
            for (int j = 0; j < P->ncell[1]; j++)
                for (int i = 0; i < P->ncell[0]; i++)
                    mesh[c * nc + ((int64_t)k * P->ncell[1] + j) * P->ncell[0] + i] = F.v[F.at(i, j, k, c)];
}

/* ---- deposit_to_mesh (Evolve.cpp:91-126) ---- */
static void deposit_range(const Geo& g, const double* parts, int64_t lo, int64_t hi, Fab& F)
{
    const auto plo = g.plo;
    const auto dxi = g.dxi;
    const int start_comp = GIdx::N00_Re;
    FabArr sarr{&F, start_comp};
    for (int64_t ip = lo; ip < hi; ip++) {
        PView p{const_cast<double*>(parts) + ip * NREAL};
        const amrex::Real delta_x = (p.pos(0) - plo[0]) * dxi[0];
        const amrex::Real delta_y = (p.pos(1) - plo[1]) * dxi[1];
        const amrex::Real delta_z = (p.pos(2) - plo[2]) * dxi[2];
        const ParticleInterpolator<2> sx(delta_x, g.ord[0]);
        const ParticleInterpolator<2> sy(delta_y, g.ord[1]);
        const ParticleInterpolator<2> sz(delta_z, g.ord[2]);
        for (int k = sz.first(); k <= sz.last(); ++k)
            for (int j = sy.first(); j <= sy.last(); ++j)
                for (int i = sx.first(); i <= sx.last(); ++i) {
#include "generated_files/Evolve.cpp_deposit_to_mesh_fill"
                }
    }
}

extern "C" void ref_deposit(const oracle_params* P, const double* parts, int64_t n, double* mesh, int nthreads)
{
    Geo g = make_geo(P);
    if (nthreads < 1) nthreads = 1;
    std::vector<Fab> fabs(nthreads);
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthreads) schedule(static, 1)
#endif
    for (int t = 0; t < nthreads; t++) {
        fabs[t].define(P->ncell, g.ngrow, GIdx::ncomp);
        deposit_range(g, parts, n * t / nthreads, n * (t + 1) / nthreads, fabs[t]);
    }
    for (int t = 1; t < nthreads; t++)
        for (size_t q = 0; q < fabs[0].v.size(); q++) fabs[0].v[q] += fabs[t].v[q];
    sum_boundary(fabs[0], GIdx::N00_Re, GIdx::ncomp);
    mesh_from_fab(fabs[0], P, mesh, GIdx::N00_Re);
}

/* ---- interpolate_rhs_from_mesh (Evolve.cpp:128-176) ---- */
static void interpolate_fab(const oracle_params* P, const Fab& F, const double* parts, int64_t n,
                            double* out, int nthreads)
{
    Geo g = make_geo(P);
    HParams hp = to_hparams(P);
    const HParams* parms = &hp;
    const auto plo = g.plo;
    const auto dxi = g.dxi;
    const Real inv_cell_volume = dxi[0] * dxi[1] * dxi[2];
    FabArr sarr{const_cast<Fab*>(&F), 0};
    if (nthreads < 1) nthreads = 1;
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthreads) schedule(static)
#endif
    for (int64_t ip = 0; ip < n; ip++) {
        std::memcpy(out + ip * NREAL, parts + ip * NREAL, sizeof(double) * NREAL);
        PView p{out + ip * NREAL};
#include "generated_files/Evolve.cpp_Vvac_fill"

        const amrex::Real delta_x = (p.pos(0) - plo[0]) * dxi[0];
        const amrex::Real delta_y = (p.pos(1) - plo[1]) * dxi[1];
        const amrex::Real delta_z = (p.pos(2) - plo[2]) * dxi[2];
        const ParticleInterpolator<2> sx(delta_x, g.ord[0]);
        const ParticleInterpolator<2> sy(delta_y, g.ord[1]);
        const ParticleInterpolator<2> sz(delta_z, g.ord[2]);
        for (int k = sz.first(); k <= sz.last(); ++k)
            for (int j = sy.first(); j <= sy.last(); ++j)
                for (int i = sx.first(); i <= sx.last(); ++i) {
#include "generated_files/Evolve.cpp_interpolate_from_mesh_fill"
                }

        p.rdata(PIdx::x) = p.rdata(PIdx::pupx) / p.rdata(PIdx::pupt) * PhysConst::c;
        p.rdata(PIdx::y) = p.rdata(PIdx::pupy) / p.rdata(PIdx::pupt) * PhysConst::c;
        p.rdata(PIdx::z) = p.rdata(PIdx::pupz) / p.rdata(PIdx::pupt) * PhysConst::c;
        p.rdata(PIdx::time) = 1.0;
        p.rdata(PIdx::pupx) = 0;
        p.rdata(PIdx::pupy) = 0;
        p.rdata(PIdx::pupz) = 0;
        p.rdata(PIdx::pupt) = 0;
        p.rdata(PIdx::N) = 0;
        p.rdata(PIdx::Nbar) = 0;
        p.rdata(PIdx::L) = 0;
        p.rdata(PIdx::Lbar) = 0;

#include "generated_files/Evolve.cpp_dfdt_fill"
    }
}

extern "C" void ref_interpolate_rhs(const oracle_params* P, const double* mesh, const double* parts,
                                    int64_t n, double* out, int nthreads)
{
    Fab F;
    fab_from_mesh(F, P, mesh);
    interpolate_fab(P, F, parts, n, out, nthreads);
}

/* ---- Renormalize (FlavoredNeutrinoContainer.cpp:89-113) ---- */
extern "C" int ref_renormalize(const oracle_params* P, double* parts, int64_t n, int64_t* bad)
{
    HParams hp = to_hparams(P);
    const HParams* parms = &hp;
    int status = 0;
    if (bad) *bad = -1;
    for (int64_t ip = 0; ip < n; ip++) {
        PView p{parts + ip * NREAL};
        Real sumP, length, error;
        g_err = 0;
#include "generated_files/FlavoredNeutrinoContainer.cpp_Renormalize_fill"
        if (g_err && bad && *bad < 0) *bad = ip;
        status |= g_err;
    }
    return status;
}

/* ---- L, Lbar from f (FlavoredNeutrinoContainerInit.cpp:651) ---- */
extern "C" void ref_set_trace_length(double* parts, int64_t n)
{
    for (int64_t ip = 0; ip < n; ip++) {
        PView p{parts + ip * NREAL};
#include "generated_files/FlavoredNeutrinoContainerInit.cpp_set_trace_length"
    }
}

/* ---- Vvac_max (FlavoredNeutrinoContainerInit.cpp:657-660) ---- */
extern "C" double ref_vvac_max(const oracle_params* P, const double* parts, int64_t n)
{
    HParams hp = to_hparams(P);
    const HParams* parms = &hp;
    Real pupt_min = INFINITY;
    for (int64_t ip = 0; ip < n; ip++) pupt_min = std::min(pupt_min, parts[ip * NREAL + 3 + PIdx::pupt]);
    Real Vvac_max;
#include "generated_files/FlavoredNeutrinoContainerInit.cpp_Vvac_fill"
    return Vvac_max;
}

/* ---- compute_dt (Evolve.cpp:22-89), reduction over the grown box ---- */
extern "C" int ref_compute_dt(const oracle_params* P, const double* mesh, double vvac_max, double* dt_out)
{
    Fab F;
    fab_from_mesh(F, P, mesh);
    Geo g = make_geo(P);
    const auto dx = g.dx;
    const Real cell_volume = dx[0] * dx[1] * dx[2];
    const auto dxi = g.dx;
    Real dt_translation = 0.0;
    if (P->cfl_factor > 0.0)
        dt_translation = std::min(std::min(dxi[0], dxi[1]), dxi[2]) / PhysConst::c * P->cfl_factor;
    Real dt_flavor = 0.0;
    if (P->flavor_cfl_factor > 0.0) {
        Real r0 = std::numeric_limits<Real>::lowest(), r1 = std::numeric_limits<Real>::lowest();
        FabArr fab{&F, 0};
        for (int k = -F.ng[2]; k < F.n[2] + F.ng[2]; k++)
            for (int j = -F.ng[1]; j < F.n[1] + F.ng[1]; j++)
                for (int i = -F.ng[0]; i < F.n[0] + F.ng[0]; i++) {
                    Real V_adaptive = 0, V_adaptive2 = 0, V_stupid = 0;
#include "generated_files/Evolve.cpp_compute_dt_fill"
                    r0 = std::max(r0, V_adaptive);
                    r1 = std::max(r1, V_stupid);
                }
        Real Vmax_adaptive = r0 + vvac_max;
        Real Vmax_stupid = r1 + vvac_max;
        Real dt_flavor_adaptive = PhysConst::hbar / Vmax_adaptive * P->flavor_cfl_factor;
        Real dt_flavor_stupid = PhysConst::hbar / Vmax_stupid * P->flavor_cfl_factor;
        dt_flavor = dt_flavor_stupid;
        if (P->max_adaptive_speedup > 1)
            dt_flavor = std::min(dt_flavor_stupid * P->max_adaptive_speedup, dt_flavor_adaptive);
    }
    Real dt = 0.0;
    if (dt_translation != 0.0 && dt_flavor != 0.0) dt = std::min(dt_translation, dt_flavor);
    else if (dt_translation != 0.0) dt = dt_translation;
    else if (dt_flavor != 0.0) dt = dt_flavor;
    else { *dt_out = 0.0; return ORACLE_ERR_DT; }
    *dt_out = dt;
    return ORACLE_OK;
}

/* ---- periodic Redistribute (restated AMReX enforcePeriodic) ---- */
extern "C" void ref_wrap(const oracle_params* P, double* parts, int64_t n)
{
    Real L[3] = {P->Lx, P->Ly, P->Lz};
    for (int64_t ip = 0; ip < n; ip++) {
        PView p{parts + ip * NREAL};
        p.pos(0) = p.rdata(PIdx::x);     /* SyncLocation(CoordinateToPosition) */
        p.pos(1) = p.rdata(PIdx::y);
        p.pos(2) = p.rdata(PIdx::z);
        for (int d = 0; d < 3; d++) {
            if (p.pos(d) >= L[d]) {
                while (p.pos(d) >= L[d]) p.pos(d) -= L[d];
                if (p.pos(d) < 0.0) p.pos(d) = 0.0;
            } else if (p.pos(d) < 0.0) {
                while (p.pos(d) < 0.0) p.pos(d) += L[d];
                if (p.pos(d) >= L[d]) p.pos(d) = 0.0;
            }
        }
        p.rdata(PIdx::x) = p.pos(0);     /* SyncLocation(PositionToCoordinate) */
        p.rdata(PIdx::y) = p.pos(1);
        p.rdata(PIdx::z) = p.pos(2);
    }
}

/* ---- explicit RK step (TimeIntegrator restated; see emu_oracle.c) ---- */
extern "C" int ref_rk_step(const oracle_params* P, int rk_type, double* parts, int64_t n, double dt,
                           double* mesh, double* scratch, int nthreads, int64_t* bad)
{
    static const double fe_a[1] = {0.0};
    static const double fe_b[1] = {1.0};
    static const double tz_a[4] = {0.0, 0.0, 1.0, 0.0};
    static const double tz_b[2] = {0.5, 0.5};
    static const double s3_a[9] = {0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.25, 0.25, 0.0};
    static const double s3_b[3] = {1. / 6., 1. / 6., 2. / 3.};
    static const double r4_a[16] = {0, 0, 0, 0, 0.5, 0, 0, 0, 0.0, 0.5, 0, 0, 0.0, 0.0, 1.0, 0};
    static const double r4_b[4] = {1. / 6., 1. / 3., 1. / 3., 1. / 6.};
    int ns;
    const double *A, *b;
    switch (rk_type) {
    case 0: ns = 1; A = fe_a; b = fe_b; break;
    case 2: ns = 2; A = tz_a; b = tz_b; break;
    case 3: ns = 3; A = s3_a; b = s3_b; break;
    default: ns = 4; A = r4_a; b = r4_b; break;
    }
    const size_t rec = (size_t)n * NREAL;
    double* S = scratch;
    double* K = scratch + rec;
    for (int i = 0; i < ns; i++) {
        std::memcpy(S, parts, sizeof(double) * rec);
        for (int j = 0; j < i; j++) {
            const double w = dt * A[i * ns + j];
            const double* Kj = K + (size_t)j * rec;
            for (int64_t ip = 0; ip < n; ip++)     /* ApplyFlavoredNeutrinoRHS */
                for (int a = 0; a < PIdx::nattribs; a++)
                    S[ip * NREAL + 3 + a] = w * Kj[ip * NREAL + 3 + a] + S[ip * NREAL + 3 + a];
        }
        ref_deposit(P, S, n, mesh, nthreads);
        Fab F;
        fab_from_mesh(F, P, mesh);
        interpolate_fab(P, F, S, n, K + (size_t)i * rec, nthreads);
    }
    for (int i = 0; i < ns; i++) {
        const double w = dt * b[i];
        const double* Ki = K + (size_t)i * rec;
        for (int64_t ip = 0; ip < n; ip++)
            for (int a = 0; a < PIdx::nattribs; a++)
                parts[ip * NREAL + 3 + a] = w * Ki[ip * NREAL + 3 + a] + parts[ip * NREAL + 3 + a];
    }
    ref_wrap(P, parts, n);
    return ref_renormalize(P, parts, n, bad);
}

extern "C" int ref_nflavors(void) { return PIdx::nattribs == 20 ? 2 : 3; }
