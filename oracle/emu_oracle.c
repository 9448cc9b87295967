/*
 * emu_oracle.c -- TEST INFRASTRUCTURE ONLY (see emu_oracle.h).
 *
 * Plain C99 FP64 restatement of the reference's per-step evolution path.
 * Each function cites the reference file:line it follows; paths are relative
 * to the Emu source tree.  Compiled with -ffp-contract=off so that the order
 * of operations written here is the order executed.
 */
#include "emu_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Source/Constants.H:6-26 */
static const double C_eV = 1.60218e-12;
static const double C_c = 2.99792458e10;
static const double C_hbar = 1.05457266e-27;
static const double C_Mp = 1.6726219e-24;

static double c2(void) { return C_c * C_c; }
static double c4(void) { return c2() * c2(); }
static double hbarc(void) { return C_hbar * C_c; }
static double GF(void)
{
    /* 1.1663787e-5 GeV^-2 / (1e9 eV)^2 * (hbar c)^3  [erg cm^3] */
    double hc = hbarc();
    return 1.1663787e-5 / (1e9 * 1e9 * C_eV * C_eV) * hc * hc * hc;
}

#define MAXNF 3
#define MAXH (MAXNF * MAXNF)

int oracle_nattribs(int nf) { return 8 + 2 * (2 + nf * nf); }
int oracle_nreal(int nf) { return 3 + oracle_nattribs(nf); }
int oracle_ncomp(int nf) { return 3 + 8 * nf * nf; }

/* PIdx offsets inside rdata (FlavoredNeutrinoContainer.H:18-25) */
enum { P_time = 0, P_x, P_y, P_z, P_pupx, P_pupy, P_pupz, P_pupt, P_N };
static int pidx_N(int nf, int s) { return 8 + s * (2 + nf * nf); }
static int pidx_L(int nf, int s) { return pidx_N(nf, s) + 1; }
static int pidx_f(int nf, int s) { return pidx_N(nf, s) + 2; }

/* Hermitian component order: upper triangle, row-major, Re then Im
 * (HermitianUtils.py:170-178).  hidx[i][j] = index of Re(i,j); Im at +1. */
static void herm_index(int nf, int re_idx[MAXNF][MAXNF], int im_idx[MAXNF][MAXNF])
{
    int c = 0;
    for (int i = 0; i < nf; i++)
        for (int j = i; j < nf; j++) {
            re_idx[i][j] = c++;
            im_idx[i][j] = (j > i) ? c++ : -1;
        }
}

/* is component e an imaginary part? */
static int herm_is_im(int nf, int e)
{
    int re[MAXNF][MAXNF], im[MAXNF][MAXNF];
    herm_index(nf, re, im);
    for (int i = 0; i < nf; i++)
        for (int j = i + 1; j < nf; j++)
            if (im[i][j] == e) return 1;
    return 0;
}

/* expand real components into a full complex matrix (re, im arrays) */
static void herm_expand(int nf, const double* h, double R[MAXNF][MAXNF], double I[MAXNF][MAXNF])
{
    int re[MAXNF][MAXNF], im[MAXNF][MAXNF];
    herm_index(nf, re, im);
    for (int i = 0; i < nf; i++)
        for (int j = i; j < nf; j++) {
            R[i][j] = h[re[i][j]];
            I[i][j] = (j > i) ? h[im[i][j]] : 0.0;
            R[j][i] = R[i][j];
            I[j][i] = -I[i][j];
        }
}

/* SU(n) vector length (HermitianUtils.py:102-123): sum |offdiag|^2 (Im^2 then
 * Re^2, pairs in (i,j) order) + sum_l (sqrt(2/(l(l+1)))/2 * (sum_{i<l} f_ii - l f_ll))^2 */
double oracle_su_length(int nf, const double* f)
{
    int re[MAXNF][MAXNF], im[MAXNF][MAXNF];
    herm_index(nf, re, im);
    double s = 0.0;
    for (int i = 0; i < nf; i++)
        for (int j = i + 1; j < nf; j++) {
            double a = f[im[i][j]], b = f[re[i][j]];
            s = s + a * a;
            s = s + b * b;
        }
    for (int l = 1; l < nf; l++) {
        double cl = sqrt(2.0 / (l * (l + 1.0))) / 2.0;
        double t = 0.0;
        for (int i = 0; i < l; i++) t = t + cl * f[re[i][i]];
        t = t - (cl * l) * f[re[l][l]];
        s = s + t * t;
    }
    return sqrt(s);
}

/* ParticleInterpolator.H:34-131 (nearest index uses truncation toward zero,
 * exactly as static_cast<int>) */
void oracle_shape(double delta, int order, int* first, double w[3])
{
    double dstar = (delta - 0.5 < 0.0) ? delta - 1.0 : delta;
    int nearest = (int)dstar;
    double fraction = delta - (double)(int)delta;
    double offset = (delta <= 0.0) ? fraction + 0.5 : fraction - 0.5;
    w[0] = w[1] = w[2] = 0.0;
    if (order >= 2) {
        *first = nearest - 1;
        w[0] = 0.5 * (0.5 - offset) * (0.5 - offset);
        w[1] = 0.75 - offset * offset;
        w[2] = 0.5 * (0.5 + offset) * (0.5 + offset);
    } else if (order == 1) {
        if (offset >= 0) {
            *first = nearest;
            w[0] = 1.0 - offset;
            w[1] = offset;
        } else {
            *first = nearest - 1;
            w[0] = -offset;
            w[1] = 1.0 + offset;
        }
    } else {
        *first = nearest;
        w[0] = 1.0;
    }
}

static int imod(int a, int n)
{
    int r = a % n;
    return r < 0 ? r + n : r;
}

/* per-dimension shape order: 0 for one-cell dimensions (Evolve.cpp:102-104, 134-136) */
static void dim_orders(const oracle_params* P, int ord[3])
{
    for (int d = 0; d < 3; d++) ord[d] = P->ncell[d] > 1 ? P->shape_order : 0;
}

static void geometry(const oracle_params* P, double dx[3], double dxi[3])
{
    double L[3] = {P->Lx, P->Ly, P->Lz};
    for (int d = 0; d < 3; d++) {
        dx[d] = L[d] / (double)P->ncell[d];   /* AMReX CellSize */
        dxi[d] = 1.0 / dx[d];                  /* AMReX InvCellSize */
    }
}

static int64_t ncells(const oracle_params* P)
{
    return (int64_t)P->ncell[0] * P->ncell[1] * P->ncell[2];
}

void oracle_init_mesh(const oracle_params* P, double* mesh)
{
    int64_t nc = ncells(P);
    int ncomp = oracle_ncomp(P->nflavors);
    memset(mesh, 0, sizeof(double) * nc * ncomp);
    for (int64_t c = 0; c < nc; c++) {
        mesh[0 * nc + c] = P->rho;
        mesh[1 * nc + c] = P->T;
        mesh[2 * nc + c] = P->Ye;
    }
}

/* GIdx component of (dir 0..3 = N,Fx,Fy,Fz ; species 0 nu / 1 nubar ; e) */
static int gidx(int nf, int dir, int s, int e) { return 3 + (dir * 2 + s) * nf * nf + e; }

/* deposit of a particle slice into an accumulation mesh (deposited comps only)
 * Evolve.cpp:91-126 and generate_code.py:150-169.  The reference deposits
 * into ghost cells and folds them back with SumBoundary; with periodic
 * boundaries that equals accumulating into (index mod ncell). */
static void deposit_slice(const oracle_params* P, const double* parts, int64_t lo, int64_t hi,
                          double* acc)
{
    const int nf = P->nflavors, nh = nf * nf, nr = oracle_nreal(nf);
    int ord[3];
    double dx[3], dxi[3];
    dim_orders(P, ord);
    geometry(P, dx, dxi);
    const int nx = P->ncell[0], ny = P->ncell[1], nz = P->ncell[2];
    const int64_t nc = ncells(P);
    for (int64_t p = lo; p < hi; p++) {
        const double* pp = parts + p * nr;
        const double* rd = pp + 3;
        int fx, fy, fz;
        double sx[3], sy[3], sz[3];
        oracle_shape((pp[0] - 0.0) * dxi[0], ord[0], &fx, sx);
        oracle_shape((pp[1] - 0.0) * dxi[1], ord[1], &fy, sy);
        oracle_shape((pp[2] - 0.0) * dxi[2], ord[2], &fz, sz);
        const int lx = fx + (ord[0] >= 2 ? 2 : ord[0]);
        const int ly = fy + (ord[1] >= 2 ? 2 : ord[1]);
        const int lz = fz + (ord[2] >= 2 ? 2 : ord[2]);
        for (int k = fz; k <= lz; k++)
            for (int j = fy; j <= ly; j++)
                for (int i = fx; i <= lx; i++) {
                    int64_t cell = ((int64_t)imod(k, nz) * ny + imod(j, ny)) * nx + imod(i, nx);
                    double w = sx[i - fx] * sy[j - fy] * sz[k - fz];
                    for (int s = 0; s < 2; s++) {
                        double Ns = rd[pidx_N(nf, s)];
                        const double* f = rd + pidx_f(nf, s);
                        for (int dir = 0; dir < 4; dir++)
                            for (int e = 0; e < nh; e++) {
                                double v = w * f[e] * Ns;
                                if (dir > 0) v = v * rd[P_pupx + dir - 1] / rd[P_pupt];
                                acc[(int64_t)(gidx(nf, dir, s, e) - 3) * nc + cell] += v;
                            }
                    }
                }
    }
}

void oracle_deposit(const oracle_params* P, const double* parts, int64_t n, double* mesh,
                    int nthreads)
{
    const int nf = P->nflavors;
    const int ndep = 8 * nf * nf;
    const int64_t nc = ncells(P);
    double* dep = mesh + 3 * nc;
    if (nthreads < 1) nthreads = 1;
    if (nthreads == 1 || n < 2 * nthreads) {
        memset(dep, 0, sizeof(double) * ndep * nc);
        deposit_slice(P, parts, 0, n, dep);
        return;
    }
    double* priv = (double*)calloc((size_t)nthreads * ndep * nc, sizeof(double));
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthreads) schedule(static, 1)
#endif
    for (int t = 0; t < nthreads; t++) {
        int64_t lo = n * t / nthreads, hi = n * (t + 1) / nthreads;
        deposit_slice(P, parts, lo, hi, priv + (size_t)t * ndep * nc);
    }
    memset(dep, 0, sizeof(double) * ndep * nc);
    for (int t = 0; t < nthreads; t++) {
        const double* src = priv + (size_t)t * ndep * nc;
        for (int64_t q = 0; q < (int64_t)ndep * nc; q++) dep[q] += src[q];
    }
    free(priv);
}

/* Flavor-basis mass-squared matrix (generate_code.py:174-227): U = U12*P for
 * NF=2, U = U23*U13*U12*P for NF=3, where U23 is built from theta13 (the
 * reference's own construction; theta23 never enters).  The Majorana phase
 * matrix P commutes with diag(m^2) and cancels, so it is omitted. */
static void mass_matrix(const oracle_params* P, double MR[MAXNF][MAXNF], double MI[MAXNF][MAXNF])
{
    const int nf = P->nflavors;
    double UR[MAXNF][MAXNF] = {{0}}, UI[MAXNF][MAXNF] = {{0}};
    double AR[MAXNF][MAXNF], AI[MAXNF][MAXNF];
    for (int i = 0; i < nf; i++) UR[i][i] = 1.0;
    /* U12 */
    double R12[MAXNF][MAXNF] = {{0}}, I12[MAXNF][MAXNF] = {{0}};
    for (int i = 0; i < nf; i++) R12[i][i] = 1.0;
    R12[0][0] = cos(P->theta12);
    R12[0][1] = sin(P->theta12);
    R12[1][0] = -sin(P->theta12);
    R12[1][1] = cos(P->theta12);
    if (nf == 2) {
        memcpy(UR, R12, sizeof UR);
        memcpy(UI, I12, sizeof UI);
    } else {
        double R13[MAXNF][MAXNF] = {{0}}, I13[MAXNF][MAXNF] = {{0}};
        double R23[MAXNF][MAXNF] = {{0}}, I23[MAXNF][MAXNF] = {{0}};
        for (int i = 0; i < nf; i++) R13[i][i] = R23[i][i] = 1.0;
        double s13 = sin(P->theta13), c13 = cos(P->theta13);
        R13[0][0] = c13;
        R13[0][2] = s13 * cos(-P->deltaCP);
        I13[0][2] = s13 * sin(-P->deltaCP);
        R13[2][0] = -s13 * cos(P->deltaCP);
        I13[2][0] = -s13 * sin(P->deltaCP);
        R13[2][2] = c13;
        R23[0][0] = c13;
        R23[0][2] = s13;
        R23[2][0] = -s13;
        R23[2][2] = c13;
        /* A = U23*U13 */
        for (int i = 0; i < nf; i++)
            for (int j = 0; j < nf; j++) {
                double r = 0, im = 0;
                for (int k = 0; k < nf; k++) {
                    r += R23[i][k] * R13[k][j] - I23[i][k] * I13[k][j];
                    im += R23[i][k] * I13[k][j] + I23[i][k] * R13[k][j];
                }
                AR[i][j] = r;
                AI[i][j] = im;
            }
        /* U = A*U12 */
        for (int i = 0; i < nf; i++)
            for (int j = 0; j < nf; j++) {
                double r = 0, im = 0;
                for (int k = 0; k < nf; k++) {
                    r += AR[i][k] * R12[k][j] - AI[i][k] * I12[k][j];
                    im += AR[i][k] * I12[k][j] + AI[i][k] * R12[k][j];
                }
                UR[i][j] = r;
                UI[i][j] = im;
            }
    }
    double m2[MAXNF] = {P->mass1 * P->mass1, P->mass2 * P->mass2, P->mass3 * P->mass3};
    /* M = U diag(m2) U^dagger */
    for (int i = 0; i < nf; i++)
        for (int j = 0; j < nf; j++) {
            double r = 0, im = 0;
            for (int k = 0; k < nf; k++) {
                /* U_ik m2_k conj(U_jk) */
                double ar = UR[i][k] * m2[k], ai = UI[i][k] * m2[k];
                r += ar * UR[j][k] + ai * UI[j][k];
                im += ai * UR[j][k] - ar * UI[j][k];
            }
            MR[i][j] = r;
            MI[i][j] = im;
        }
}

/* Evolve.cpp_Vvac_fill (generate_code.py:239-255): V = M2 c^4/(2 pupt);
 * antineutrinos take the complex conjugate. */
void oracle_vvac(const oracle_params* P, double pupt, double* V)
{
    const int nf = P->nflavors, nh = nf * nf;
    double MR[MAXNF][MAXNF], MI[MAXNF][MAXNF];
    int re[MAXNF][MAXNF], im[MAXNF][MAXNF];
    mass_matrix(P, MR, MI);
    herm_index(nf, re, im);
    for (int i = 0; i < nf; i++)
        for (int j = i; j < nf; j++) {
            V[re[i][j]] = MR[i][j] * c4() / (2. * pupt);
            V[nh + re[i][j]] = MR[i][j] * c4() / (2. * pupt);
            if (j > i) {
                V[im[i][j]] = MI[i][j] * c4() / (2. * pupt);
                V[nh + im[i][j]] = -1.0 * MI[i][j] * c4() / (2. * pupt);
            }
        }
}

/* FlavoredNeutrinoContainerInit.cpp:657-660 + generate_code.py:229-237 */
double oracle_vvac_max(const oracle_params* P, const double* parts, int64_t n)
{
    const int nf = P->nflavors, nr = oracle_nreal(nf);
    double pupt_min = INFINITY;
    for (int64_t p = 0; p < n; p++) {
        double v = parts[p * nr + 3 + P_pupt];
        if (v < pupt_min) pupt_min = v;
    }
    double h[MAXH] = {0};
    int re[MAXNF][MAXNF], im[MAXNF][MAXNF];
    herm_index(nf, re, im);
    h[re[0][0]] = P->mass1 * P->mass1;
    h[re[1][1]] = P->mass2 * P->mass2;
    if (nf == 3) h[re[2][2]] = P->mass3 * P->mass3;
    return oracle_su_length(nf, h) * c4() / pupt_min;
}

/* -i/hbar [H, F] in real components (generate_code.py:359-389) */
static void commutator_rhs(int nf, const double* h, const double* f, double* out)
{
    double HR[MAXNF][MAXNF], HI[MAXNF][MAXNF], FR[MAXNF][MAXNF], FI[MAXNF][MAXNF];
    int re[MAXNF][MAXNF], im[MAXNF][MAXNF];
    herm_expand(nf, h, HR, HI);
    herm_expand(nf, f, FR, FI);
    herm_index(nf, re, im);
    for (int i = 0; i < nf; i++)
        for (int j = i; j < nf; j++) {
            double cr = 0.0, ci = 0.0;   /* C = H F - F H */
            for (int k = 0; k < nf; k++) {
                cr += HR[i][k] * FR[k][j] - HI[i][k] * FI[k][j];
                ci += HR[i][k] * FI[k][j] + HI[i][k] * FR[k][j];
                cr -= FR[i][k] * HR[k][j] - FI[i][k] * HI[k][j];
                ci -= FR[i][k] * HI[k][j] + FI[i][k] * HR[k][j];
            }
            /* G = -i C / hbar */
            out[re[i][j]] = ci / C_hbar;
            if (j > i) out[im[i][j]] = -cr / C_hbar;
        }
}

/* interpolate_rhs_from_mesh for one particle: Evolve.cpp:128-176 and the
 * Vvac / interpolate / dfdt fills (generate_code.py:239-255, 296-389). */
static void interp_one(const oracle_params* P, const double* mesh, const double* pp, double* out,
                       const double* Vvac_unit)
{
    const int nf = P->nflavors, nh = nf * nf, nr = oracle_nreal(nf);
    int ord[3];
    double dx[3], dxi[3];
    dim_orders(P, ord);
    geometry(P, dx, dxi);
    const double inv_cell_volume = dxi[0] * dxi[1] * dxi[2];
    const int nx = P->ncell[0], ny = P->ncell[1], nz = P->ncell[2];
    const int64_t nc = ncells(P);
    const double* rd = pp + 3;
    const double pupt = rd[P_pupt];
    double V[2 * MAXH];
    /* Vvac_unit holds M2 (nu, nubar) ; scale per particle as the fill does */
    for (int e = 0; e < 2 * nh; e++) V[e] = Vvac_unit[e] * c4() / (2. * pupt);

    int fx, fy, fz;
    double sx[3], sy[3], sz[3];
    oracle_shape((pp[0] - 0.0) * dxi[0], ord[0], &fx, sx);
    oracle_shape((pp[1] - 0.0) * dxi[1], ord[1], &fy, sy);
    oracle_shape((pp[2] - 0.0) * dxi[2], ord[2], &fz, sz);
    const int lx = fx + (ord[0] >= 2 ? 2 : ord[0]);
    const int ly = fy + (ord[1] >= 2 ? 2 : ord[1]);
    const int lz = fz + (ord[2] >= 2 ? 2 : ord[2]);
    const double sqrt2GF = sqrt(2.) * GF();
    for (int k = fz; k <= lz; k++)
        for (int j = fy; j <= ly; j++)
            for (int i = fx; i <= lx; i++) {
                int64_t cell = ((int64_t)imod(k, nz) * ny + imod(j, ny)) * nx + imod(i, nx);
                const double coef = sqrt2GF * inv_cell_volume * sx[i - fx] * sy[j - fy] * sz[k - fz];
                for (int e = 0; e < nh; e++) {
                    double sgn = herm_is_im(nf, e) ? 1.0 : -1.0;
                    double SI = 1 * (mesh[(int64_t)gidx(nf, 0, 0, e) * nc + cell]
                                     - mesh[(int64_t)gidx(nf, 1, 0, e) * nc + cell] * rd[P_pupx] / pupt
                                     - mesh[(int64_t)gidx(nf, 2, 0, e) * nc + cell] * rd[P_pupy] / pupt
                                     - mesh[(int64_t)gidx(nf, 3, 0, e) * nc + cell] * rd[P_pupz] / pupt);
                    double SIbar = sgn * (mesh[(int64_t)gidx(nf, 0, 1, e) * nc + cell]
                                          - mesh[(int64_t)gidx(nf, 1, 1, e) * nc + cell] * rd[P_pupx] / pupt
                                          - mesh[(int64_t)gidx(nf, 2, 1, e) * nc + cell] * rd[P_pupy] / pupt
                                          - mesh[(int64_t)gidx(nf, 3, 1, e) * nc + cell] * rd[P_pupz] / pupt);
                    double inside = SI + SIbar;
                    if (e == 0) inside = inside + mesh[0 * nc + cell] * mesh[2 * nc + cell] / C_Mp / inv_cell_volume;
                    double term = coef * (inside);
                    V[e] += term;
                    if (sgn > 0) V[nh + e] += term; else V[nh + e] -= term;
                }
            }

    /* non-flavor derivatives (Evolve.cpp:160-172) */
    out[0] = pp[0];
    out[1] = pp[1];
    out[2] = pp[2];
    double* od = out + 3;
    for (int a = 0; a < nr - 3; a++) od[a] = 0.0;
    od[P_x] = rd[P_pupx] / rd[P_pupt] * C_c;
    od[P_y] = rd[P_pupy] / rd[P_pupt] * C_c;
    od[P_z] = rd[P_pupz] / rd[P_pupt] * C_c;
    od[P_time] = 1.0;
    for (int s = 0; s < 2; s++)
        commutator_rhs(nf, V + s * nh, rd + pidx_f(nf, s), od + pidx_f(nf, s));
}

static void vvac_unit(const oracle_params* P, double* Vu)
{
    const int nf = P->nflavors, nh = nf * nf;
    double MR[MAXNF][MAXNF], MI[MAXNF][MAXNF];
    int re[MAXNF][MAXNF], im[MAXNF][MAXNF];
    mass_matrix(P, MR, MI);
    herm_index(nf, re, im);
    for (int i = 0; i < nf; i++)
        for (int j = i; j < nf; j++) {
            Vu[re[i][j]] = 1 * MR[i][j];
            Vu[nh + re[i][j]] = 1 * MR[i][j];
            if (j > i) {
                Vu[im[i][j]] = 1 * MI[i][j];
                Vu[nh + im[i][j]] = -1 * MI[i][j];
            }
        }
}

void oracle_interpolate_rhs(const oracle_params* P, const double* mesh, const double* parts,
                            int64_t n, double* out, int nthreads)
{
    const int nr = oracle_nreal(P->nflavors);
    double Vu[2 * MAXH];
    vvac_unit(P, Vu);
    if (nthreads < 1) nthreads = 1;
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthreads) schedule(static)
#endif
    for (int64_t p = 0; p < n; p++) interp_one(P, mesh, parts + p * nr, out + p * nr, Vu);
}

/* generated Renormalize fill (generate_code.py:391-445), one species */
static int renorm_species(const oracle_params* P, double* f, double L)
{
    const int nf = P->nflavors, nh = nf * nf;
    int re[MAXNF][MAXNF], im[MAXNF][MAXNF];
    herm_index(nf, re, im);
    int status = 0;
    double sumP = 0;
    for (int i = 0; i < nf; i++) sumP += f[re[i][i]];
    double error = sumP - 1.0;
    if (fabs(error) > 100. * P->maxError) status |= ORACLE_ERR_TRACE;
    if (fabs(error) > P->maxError)
        for (int i = 0; i < nf; i++) f[re[i][i]] -= error / nf;
    for (int i = 0; i < nf; i++) {
        if (f[re[i][i]] < -100. * P->maxError) status |= ORACLE_ERR_NEGDIAG;
        if (f[re[i][i]] < -P->maxError) f[re[i][i]] = 0;
    }
    double length = oracle_su_length(nf, f);
    error = length - L;
    if (fabs(error) > 100. * P->maxError) status |= ORACLE_ERR_LENGTH;
    if (fabs(error) > P->maxError)
        for (int e = 0; e < nh; e++) f[e] /= length / L;
    return status;
}

int oracle_renormalize(const oracle_params* P, double* parts, int64_t n, int64_t* bad)
{
    const int nf = P->nflavors, nr = oracle_nreal(nf);
    int status = 0;
    if (bad) *bad = -1;
    for (int64_t p = 0; p < n; p++) {
        double* rd = parts + p * nr + 3;
        int st = 0;
        for (int s = 0; s < 2; s++) st |= renorm_species(P, rd + pidx_f(nf, s), rd[pidx_L(nf, s)]);
        if (st && bad && *bad < 0) *bad = p;
        status |= st;
    }
    return status;
}

/* SyncLocation + periodic Redistribute + SyncLocation (main.cpp:163-170;
 * FlavoredNeutrinoContainer.cpp:8-41).  Positions are shifted by whole
 * domain lengths into [0, L). */
void oracle_wrap(const oracle_params* P, double* parts, int64_t n)
{
    const int nr = oracle_nreal(P->nflavors);
    double L[3] = {P->Lx, P->Ly, P->Lz};
    for (int64_t p = 0; p < n; p++) {
        double* pp = parts + p * nr;
        for (int d = 0; d < 3; d++) {
            double x = pp[3 + P_x + d];          /* CoordinateToPosition */
            /* shift by whole periods: x -/+ L for x in [-L, 2L) */
            if (x >= L[d] || x < 0.0) {
                if (!isfinite(x)) {
                    x = 0.0;
                } else {
                    x = fmod(x, L[d]);
                    if (x < 0.0) x += L[d];
                    if (x >= L[d] || x < 0.0) x = 0.0;
                }
            }
            pp[d] = x;                           /* Redistribute */
            pp[3 + P_x + d] = x;                 /* PositionToCoordinate */
        }
    }
}

/* compute_dt: Evolve.cpp:22-89 and generate_code.py:257-294 */
int oracle_compute_dt(const oracle_params* P, const double* mesh, double vvac_max, double* dt_out)
{
    const int nf = P->nflavors, nh = nf * nf;
    double dx[3], dxi[3];
    geometry(P, dx, dxi);
    const double cell_volume = dx[0] * dx[1] * dx[2];
    const int64_t nc = ncells(P);
    double dt_translation = 0.0;
    if (P->cfl_factor > 0.0) {
        double m = dx[0] < dx[1] ? dx[0] : dx[1];
        m = m < dx[2] ? m : dx[2];
        dt_translation = m / C_c * P->cfl_factor;
    }
    double dt_flavor = 0.0;
    if (P->flavor_cfl_factor > 0.0) {
        int re[MAXNF][MAXNF], im[MAXNF][MAXNF];
        herm_index(nf, re, im);
        double vmax_adaptive = -INFINITY, vmax_stupid = -INFINITY;
        for (int64_t c = 0; c < nc; c++) {
            double rho = mesh[0 * nc + c], Ye = mesh[2 * nc + c];
            /* spherically symmetric part: N - conj(Nbar), plus matter on 00 */
            double h[MAXH];
            for (int e = 0; e < nh; e++) {
                double a = mesh[(int64_t)gidx(nf, 0, 0, e) * nc + c];
                double b = mesh[(int64_t)gidx(nf, 0, 1, e) * nc + c];
                h[e] = herm_is_im(nf, e) ? a + b : a - b;
            }
            h[0] += rho * Ye / C_Mp * cell_volume;
            double l = oracle_su_length(nf, h);
            double V2 = l * l;
            for (int d = 1; d <= 3; d++) {
                for (int e = 0; e < nh; e++)
                    h[e] = mesh[(int64_t)gidx(nf, d, 0, e) * nc + c] - mesh[(int64_t)gidx(nf, d, 1, e) * nc + c];
                l = oracle_su_length(nf, h);
                V2 += l * l;
            }
            double V_adaptive = sqrt(V2) * M_SQRT2 * GF() / cell_volume;
            double V_stupid = 0;
            for (int i = 0; i < nf; i++) {
                double a = mesh[(int64_t)gidx(nf, 0, 0, re[i][i]) * nc + c];
                double b = mesh[(int64_t)gidx(nf, 0, 1, re[i][i]) * nc + c];
                V_stupid = V_stupid > a ? V_stupid : a;
                V_stupid = V_stupid > b ? V_stupid : b;
            }
            double mat = cell_volume * Ye * rho / C_Mp;
            V_stupid = V_stupid > mat ? V_stupid : mat;
            V_stupid *= 2.0 * nf * M_SQRT2 * GF() / cell_volume;
            if (V_adaptive > vmax_adaptive) vmax_adaptive = V_adaptive;
            if (V_stupid > vmax_stupid) vmax_stupid = V_stupid;
        }
        vmax_adaptive += vvac_max;
        vmax_stupid += vvac_max;
        double dt_flavor_adaptive = C_hbar / vmax_adaptive * P->flavor_cfl_factor;
        double dt_flavor_stupid = C_hbar / vmax_stupid * P->flavor_cfl_factor;
        dt_flavor = dt_flavor_stupid;
        if (P->max_adaptive_speedup > 1) {
            double a = dt_flavor_stupid * P->max_adaptive_speedup;
            dt_flavor = a < dt_flavor_adaptive ? a : dt_flavor_adaptive;
        }
    }
    double dt = 0.0;
    if (dt_translation != 0.0 && dt_flavor != 0.0)
        dt = dt_translation < dt_flavor ? dt_translation : dt_flavor;
    else if (dt_translation != 0.0)
        dt = dt_translation;
    else if (dt_flavor != 0.0)
        dt = dt_flavor;
    else {
        *dt_out = 0.0;
        return ORACLE_ERR_DT;
    }
    *dt_out = dt;
    return ORACLE_OK;
}

/* Explicit Runge-Kutta step with AMReX's TimeIntegrator semantics (the
 * integrator lives in the un-vendored AMReX fork; its contract is visible in
 * main.cpp:129-213 and FlavoredNeutrinoContainer.H:33-47):
 *   stage i: S = copy(S_old); for j < i: S.rdata += (dt*a_ij) * K_j.rdata
 *            deposit(S); K_i = copy(S); interpolate_rhs(K_i)
 *   S_new = copy(S_old); for i: S_new.rdata += (dt*b_i) * K_i.rdata
 * Positions (pos) are the start-of-step positions in every stage.  Then the
 * post-timestep hook wraps positions and renormalises. */
int oracle_rk_step(const oracle_params* P, int rk_type, double* parts, int64_t n, double dt,
                   double* mesh, double* scratch, int nthreads, int64_t* bad)
{
    static const double fe_a[1][1] = {{0.0}};
    static const double fe_b[1] = {1.0};
    static const double tz_a[2][2] = {{0.0, 0.0}, {1.0, 0.0}};
    static const double tz_b[2] = {0.5, 0.5};
    static const double s3_a[3][3] = {{0.0, 0.0, 0.0}, {1.0, 0.0, 0.0}, {0.25, 0.25, 0.0}};
    static const double s3_b[3] = {1. / 6., 1. / 6., 2. / 3.};
    static const double r4_a[4][4] = {{0, 0, 0, 0}, {0.5, 0, 0, 0}, {0.0, 0.5, 0, 0}, {0.0, 0.0, 1.0, 0}};
    static const double r4_b[4] = {1. / 6., 1. / 3., 1. / 3., 1. / 6.};
    int ns;
    const double* A;
    const double* b;
    switch (rk_type) {
    case 0: ns = 1; A = &fe_a[0][0]; b = fe_b; break;
    case 2: ns = 2; A = &tz_a[0][0]; b = tz_b; break;
    case 3: ns = 3; A = &s3_a[0][0]; b = s3_b; break;
    default: ns = 4; A = &r4_a[0][0]; b = r4_b; break;
    }
    const int nr = oracle_nreal(P->nflavors);
    const size_t rec = (size_t)n * nr;
    double* S = scratch;            /* stage state */
    double* K = scratch + rec;      /* ns RHS containers */
    for (int i = 0; i < ns; i++) {
        memcpy(S, parts, sizeof(double) * rec);
        for (int j = 0; j < i; j++) {
            const double w = dt * A[i * ns + j];
            const double* Kj = K + (size_t)j * rec;
            for (int64_t p = 0; p < n; p++)
                for (int a = 3; a < nr; a++) S[p * nr + a] = w * Kj[p * nr + a] + S[p * nr + a];
        }
        oracle_deposit(P, S, n, mesh, nthreads);
        oracle_interpolate_rhs(P, mesh, S, n, K + (size_t)i * rec, nthreads);
    }
    for (int i = 0; i < ns; i++) {
        const double w = dt * b[i];
        const double* Ki = K + (size_t)i * rec;
        for (int64_t p = 0; p < n; p++)
            for (int a = 3; a < nr; a++) parts[p * nr + a] = w * Ki[p * nr + a] + parts[p * nr + a];
    }
    oracle_wrap(P, parts, n);
    return oracle_renormalize(P, parts, n, bad);
}

int oracle_rk4_step(const oracle_params* P, double* parts, int64_t n, double dt, double* mesh,
                    double* scratch, int nthreads, int64_t* bad)
{
    return oracle_rk_step(P, 4, parts, n, dt, mesh, scratch, nthreads, bad);
}
