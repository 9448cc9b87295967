/*
 * emu_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of Emu's per-step particle evolution path, used as the
 * parity checker for the CUDA library (emu_b200/csrc) and as the timed CPU
 * baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs may
 * load it.  The product path never calls into this file.
 *
 * Parity pin: every function here is compared, on seeded inputs, with the
 * reference's own generated kernel bodies (Scripts/symbolic_hermitians/
 * generate_code.py) compiled into oracle/_ref by oracle/build_oracle.py, and
 * with the analytic checks of Scripts/tests/msw_test.py and
 * Scripts/tests/fast_flavor_test.py (tests/test_oracle_*.py).
 *
 * Data layout (the interchange format of the whole project):
 *   particle record = [pos_x, pos_y, pos_z, rdata[0..nattribs)]  (FP64)
 *     rdata follows PIdx (Source/FlavoredNeutrinoContainer.H:12-26 plus the
 *     generated H_fill): time,x,y,z,pupx,pupy,pupz,pupt,N,L,f..,Nbar,Lbar,f..bar
 *     with the Hermitian components in upper-triangle row-major order, Re
 *     before Im (Scripts/symbolic_hermitians/HermitianUtils.py:170-178).
 *     This is the real-component order of the reference's particle output
 *     (Scripts/visualization/amrex_plot_tools.py:12-90).
 *   mesh = ncomp planes of nx*ny*nz valid cells, i fastest, component slowest
 *     (the Array4 order), components in GIdx order (Source/Evolve.H:11-27):
 *     rho,T,Ye, then N,Nbar,Fx,Fxbar,Fy,Fybar,Fz,Fzbar each with NF*NF reals.
 */
#ifndef EMU_ORACLE_H_
#define EMU_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_params {
    int nflavors;            /* NUM_FLAVORS: 2 or 3 */
    int shape_order;         /* SHAPE_FACTOR_ORDER: 0, 1 or 2 */
    int ncell[3];
    double Lx, Ly, Lz;       /* domain is [0,L) per dimension, periodic */
    double rho, Ye, T;       /* g/ccm, 1, MeV (uniform background) */
    double mass1, mass2, mass3;               /* grams (already eV/c^2 converted) */
    double theta12, theta13, theta23;         /* radians */
    double alpha1, alpha2, deltaCP;           /* radians */
    double cfl_factor, flavor_cfl_factor, max_adaptive_speedup, maxError;
} oracle_params;

/* status codes (match include/emu_b200.h) */
#define ORACLE_OK            0
#define ORACLE_ERR_TRACE     1   /* |trace-1| > 100*maxError */
#define ORACLE_ERR_NEGDIAG   2   /* diagonal < -100*maxError */
#define ORACLE_ERR_LENGTH    4   /* |length-L| > 100*maxError */
#define ORACLE_ERR_DT        8   /* no timestep limiter active */

int oracle_nattribs(int nflavors);
int oracle_nreal(int nflavors);       /* 3 + nattribs */
int oracle_ncomp(int nflavors);       /* 3 + 8*NF*NF */

/* ParticleInterpolator<order>(delta): first cell and up to 3 weights. */
void oracle_shape(double delta, int order, int* first, double w[3]);

/* deposit_to_mesh: overwrites the deposited components of mesh (GIdx >= 3),
 * keeps rho/T/Ye.  Particles are deposited in index order; with nthreads > 1
 * each thread deposits a contiguous slice into a private mesh and the slices
 * are summed in slice order, so the result is deterministic. */
void oracle_deposit(const oracle_params* P, const double* parts, int64_t n,
                    double* mesh, int nthreads);

/* set rho/T/Ye planes of a mesh to the uniform background (main.cpp:81-85) */
void oracle_init_mesh(const oracle_params* P, double* mesh);

/* interpolate_rhs_from_mesh: out[p] = d/dt of every rdata attribute of
 * particle p (pos copied through), given the deposited mesh. */
void oracle_interpolate_rhs(const oracle_params* P, const double* mesh,
                            const double* parts, int64_t n, double* out,
                            int nthreads);

/* Vacuum potential of one particle: V[0..NF*NF) nu, V[NF*NF..2NF*NF) nubar,
 * in Hermitian component order. */
void oracle_vvac(const oracle_params* P, double pupt, double* V);

/* Vvac_max (FlavoredNeutrinoContainerInit.cpp:657-660) */
double oracle_vvac_max(const oracle_params* P, const double* parts, int64_t n);

/* Renormalize (FlavoredNeutrinoContainer.cpp:89-113); returns OR of status
 * bits, *bad = first offending particle (or -1). */
int oracle_renormalize(const oracle_params* P, double* parts, int64_t n,
                       int64_t* bad);

/* periodic wrap of positions + SyncLocation (main.cpp:163-170) */
void oracle_wrap(const oracle_params* P, double* parts, int64_t n);

/* compute_dt (Evolve.cpp:22-89) from a deposited mesh */
int oracle_compute_dt(const oracle_params* P, const double* mesh,
                      double vvac_max, double* dt);

/* One RK4 step with the AMReX TimeIntegrator stage semantics, followed by the
 * post-timestep hook (wrap, Renormalize).  mesh receives the stage-4 deposit
 * (the mesh the reference keeps after a step).  scratch must hold
 * 5*n*nreal doubles.  Returns status bits; *bad as in oracle_renormalize. */
int oracle_rk4_step(const oracle_params* P, double* parts, int64_t n,
                    double dt, double* mesh, double* scratch, int nthreads,
                    int64_t* bad);

/* Forward Euler / trapezoid / SSPRK3 / RK4 via the same Butcher-tableau
 * machinery (integration.type=0 -> rk_type 0; rk.type 2,3,4). */
int oracle_rk_step(const oracle_params* P, int rk_type, double* parts,
                   int64_t n, double dt, double* mesh, double* scratch,
                   int nthreads, int64_t* bad);

/* SU(n) flavor-vector length of one Hermitian matrix (HermitianUtils.py:102-123) */
double oracle_su_length(int nflavors, const double* f);

#ifdef __cplusplus
}
#endif
#endif
