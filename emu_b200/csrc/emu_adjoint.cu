// emu_adjoint.cu -- discrete adjoint of the FP64 RK4 evolution (no
// counterpart in the reference, which has no derivatives).
//
// Objective (emu_adjoint_objective):
//   J = sum_cells |N_emu(cell)|^2 / V_cell
// with N_emu the neutrino e-mu off-diagonal number per cell deposited from
// the current particle state (mesh components N01_Re, N01_Im of the
// deposit_to_mesh layout, Evolve.cpp:91-126), i.e. the domain integral of
// |n_emu|^2.
//
// Gradient (emu_adjoint_backward): the exact vector-Jacobian product of the
// recorded run (the dt of every step is held at its recorded value):
//   stage s:  M_s = D(Y_s N)              deposit, start-of-step weights
//             K_s = -i/hbar [H(M_s), Y_s] interpolate + commutator
//             Y_{s+1} = Y_0 + a_s dt K_s
//   Y_n = Y_0 + dt sum_s b_s K_s,  Y_new = Renormalize(Y_n)
// Backward per step, stage s = 4..1 (lam = dJ/d.):
//   lam_K4 = b4 dt lam_n,  lam_Ks = b_s dt lam_n + a_{s+1} dt lam_Y{s+1}
//   lam_Ys = C_Y^T(H_s) lam_Ks  +  N D^T( I^T( C_H^T(Y_s) lam_Ks ) )
//   lam_Y0 = lam_n + sum_{s>=2} lam_Ys + lam_Y1,  lam_N += Y_s . D^T(...)
// C_Y^T, C_H^T: the commutator is bilinear, so each adjoint component is the
// commutator with a unit vector contracted with lam (exact).  I^T scatters
// like a deposit (same mesh layout, velocity sign flipped, factor
// sqrt(2) G_F / V_cell); D^T gathers like an interpolation.  The
// Renormalize adjoint replays its branches (trace fix, diagonal clamp,
// length rescale) at the forward values.
//
// Memory: checkpoints of (Y_0, x) every `interval` steps; a segment is
// recomputed forward into per-step (Y_0, x) slots, then each step's stage
// states Y_2..Y_4, Y_n and meshes M_1..M_4 are recomputed before its
// backward.  Particles keep their slot order for the whole recorded run (no
// re-sort).
#include "emu_context.cuh"
#include "emu_kernels_impl.cuh"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

using emu_ctx::check_launch;
using emu_ctx::fail;

struct emu_adjoint {
    long long cap = 0;
    int NS = 0;
    int nsteps = 0, interval = 0, nck = 0;
    bool recorded = false;
    bool store = false;         // stage states of a whole segment fit (else one step at a time)
    int sub = 0;                // per-step mode: sub-checkpoint spacing inside a segment (0: none)
    // the whole run's step states, stage states and meshes fit: the recorded
    // forward stores them (cooperative segment kernel computing dt on the
    // device) and the backward recomputes nothing; full_steps = capacity
    bool full = false;
    int full_steps = 0;
    double t0 = 0.0;
    std::vector<double> dts;
    std::vector<char> resorted; // segment c began with a cell re-sort (permutation perm[c])
    double* dts_dev = nullptr;
    double* ck = nullptr;       // nck x (NS + 3) x cap: Y_0 then x, y, z per checkpoint
    unsigned* perm = nullptr;   // nck x cap gather permutations of the segment-start re-sorts
    double* seg = nullptr;      // seg_slots x (NS + 3) x cap: Y_0, x of every step of a segment
                                // (with sub-checkpoints: of a sub-segment, then the sub-checkpoints)
    double* sst = nullptr;      // stored stage states (4 x NS x cap per step)
    double* mst = nullptr;      // stored meshes M_1..M_4 per step
    double* stat = nullptr;     // two working copies of the static particle fields
    double* work = nullptr;
    double* lmesh[4] = {};      // adjoint meshes (rotating)
    double* nex = nullptr;      // ncells x 2 objective components
    long long seg_slots = 0, ck_slots = 0;
    int interval_cap = 0;       // longest segment the slots serve
    size_t bytes = 0;           // device memory held
    double *acc = nullptr, *lamY0 = nullptr, *lamN = nullptr, *lamn = nullptr, *lamYd = nullptr;
    double *wf = nullptr, *lamtmp = nullptr, *wpos = nullptr, *wtime = nullptr;
    double* rows = nullptr;     // n x NS staging for host transfers
    unsigned* map[2] = {};      // recorded forward: slot -> slot at the segment start, through the re-sorts
    bool final_mapped = false;  // perm slot nck: the map of the run's last segment (re-sorts in it)
    // per-step mode with re-sorts: the backward's recompute re-sorts as the
    // forward did; second state buffers, the re-sort permutation of every
    // step of a sub-segment, the composed map of every sub-segment
    double *wf2 = nullptr, *wpos2 = nullptr;
    unsigned* gperm = nullptr;
    unsigned* smap = nullptr;
    int gslots = 0, sslots = 0;
    int rps_slots = 0;          // segment slots the sub-segment layout uses
    // and, when the free memory allows, the meshes M_1..M_4 of every step of
    // a sub-segment (gslots x 4 x nmesh) as the state pass deposits them: the
    // sweep's stage recompute then only interpolates
    double* smesh = nullptr;
};

namespace emu {
namespace {

// ---- per-particle adjoint pieces ------------------------------------------

// VJP of K = C(H, F) = -i/hbar [H, F] (bilinear in H and F):
//   lamF_b = sum_c lam_c C_c(H, e_b),  lamH_a = sum_c lam_c C_c(e_a, F)
template <int NF>
__device__ __forceinline__ void commutator_vjp(const double* h, const double* f, const double* lam, double* lamH,
                                               double* lamF, double inv_hbar)
{
    constexpr int NH = NF * NF;
#pragma unroll
    for (int b = 0; b < NH; b++) {
        double e[NH], o[NH];
#pragma unroll
        for (int k = 0; k < NH; k++) e[k] = (k == b) ? 1.0 : 0.0;
        commutator<NF, double>(h, e, o, inv_hbar);
        double sf = 0.0;
#pragma unroll
        for (int c = 0; c < NH; c++) sf += lam[c] * o[c];
        lamF[b] = sf;
        commutator<NF, double>(e, f, o, inv_hbar);
        double sh = 0.0;
#pragma unroll
        for (int c = 0; c < NH; c++) sh += lam[c] * o[c];
        lamH[b] = sh;
    }
}

// VJP of renormalize<NF>() at input fin (one species): replays the forward
// branch decisions with the same arithmetic.
template <int NF>
__device__ __forceinline__ void renormalize_vjp(const double* fin, double L, double maxError, const double* lam_out,
                                                double* lam_in)
{
    using H = Herm<NF>;
    constexpr int NH = NF * NF;
    double f[NH];
#pragma unroll
    for (int e = 0; e < NH; e++) f[e] = fin[e];
    double sumP = 0.0;
#pragma unroll
    for (int i = 0; i < NF; i++) sumP = __dadd_rn(sumP, f[H::re(i, i)]);
    const double err = sumP - 1.0;
    const bool trace_fix = fabs(err) > maxError;
    if (trace_fix) {
#pragma unroll
        for (int i = 0; i < NF; i++) f[H::re(i, i)] = __dsub_rn(f[H::re(i, i)], __ddiv_rn(err, (double)NF));
    }
    bool clamped[NF];
#pragma unroll
    for (int i = 0; i < NF; i++) {
        clamped[i] = f[H::re(i, i)] < -maxError;
        if (clamped[i]) f[H::re(i, i)] = 0;
    }
    const double length = su_length<NF>(f);
    const bool rescale = fabs(length - L) > maxError;
    double lam[NH];
#pragma unroll
    for (int e = 0; e < NH; e++) lam[e] = lam_out[e];
    if (rescale) {
        // f' = f L / length(f):  lam_f = (L/len) lam - (L/len^2) (lam . f) grad len
        double g[NH];
#pragma unroll
        for (int e = 0; e < NH; e++) g[e] = H::is_diag(e) ? 0.0 : f[e] / length;
#pragma unroll
        for (int l = 1; l < NF; l++) {
            const double cl = (l == 1) ? 0.5 : 0.28867513459481287;
            double t = 0.0;
#pragma unroll
            for (int i = 0; i < l; i++) t += cl * f[H::re(i, i)];
            t -= cl * l * f[H::re(l, l)];
#pragma unroll
            for (int i = 0; i < l; i++) g[H::re(i, i)] += t * cl / length;
            g[H::re(l, l)] -= t * cl * l / length;
        }
        double dot = 0.0;
#pragma unroll
        for (int e = 0; e < NH; e++) dot += lam[e] * f[e];
        const double a = L / length, b = L / (length * length) * dot;
#pragma unroll
        for (int e = 0; e < NH; e++) lam[e] = a * lam[e] - b * g[e];
    }
#pragma unroll
    for (int i = 0; i < NF; i++)
        if (clamped[i]) lam[H::re(i, i)] = 0.0;
    if (trace_fix) {
        double m = 0.0;
#pragma unroll
        for (int i = 0; i < NF; i++) m += lam[H::re(i, i)];
        m /= NF;
#pragma unroll
        for (int i = 0; i < NF; i++) lam[H::re(i, i)] -= m;
    }
#pragma unroll
    for (int e = 0; e < NH; e++) lam_in[e] = lam[e];
}

// D^T: G_c = sum_cells w * (lm[c] + vx lm[NS+c] + vy lm[2NS+c] + vz lm[3NS+c])
// (the transpose of the deposit's N / F layout)
template <int NF, class SWt>
__device__ __forceinline__ void gather_deposit_adjoint(const DevParams& P, const double* __restrict__ lm,
                                                       const Stencil<double>& st, double vx, double vy, double vz,
                                                       double* G)
{
    constexpr int NS = 2 * NF * NF, ND = 8 * NF * NF;
#pragma unroll
    for (int c = 0; c < NS; c++) G[c] = 0.0;
    STENCIL_LOOP(SWt, {
        const long long cell = cell_of(P, st.b[0], st.b[1], st.b[2], ii, jj, kk);
        const double* __restrict__ m = lm + cell * ND;
        const double w = (st.wx[ii] * st.wy[jj]) * st.wz[kk];
#pragma unroll
        for (int c = 0; c < NS; c++)
            G[c] += w * (__ldg(m + c) + vx * __ldg(m + NS + c) + vy * __ldg(m + 2 * NS + c) +
                         vz * __ldg(m + 3 * NS + c));
    })
}

// ---- kernels ----------------------------------------------------------------

// Stage recompute: K = RHS(Yin, M_s); s < 4: acc, Y_{s+1} = Y0 + a dt K and
// its deposit; s == 4: Y_n = acc + b4 dt K.  Same arithmetic as the forward
// stage kernel.
template <int NF, class SWt>
__device__ __forceinline__ void adj_fwd_stage_body(const DevParams& P, const DevState& S, int s, double dt,
                                                   const double* __restrict__ Yin, const double* __restrict__ Y0,
                                                   double* __restrict__ acc, double* __restrict__ Yout,
                                                   const double* __restrict__ mesh_in, double* __restrict__ mesh_out)
{
    constexpr int NH = NF * NF, NS = 2 * NH;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < S.n;
    const long long cap = S.cap;
    Stencil<double> st{};
    double fN[NS] = {};
    double vx = 0, vy = 0, vz = 0;
    if (active) {
        make_stencil<double>(P, S.pos[0][p], S.pos[1][p], S.pos[2][p], st);
        vx = S.vhat[0][p];
        vy = S.vhat[1][p];
        vz = S.vhat[2][p];
        double V[NS];
        potential_fp64<NF, SWt>(P, mesh_in, st, vx, vy, vz, S.vscale[p], V);
        const double bw = dt * kRK4B[s - 1];
        const double aw = s < 4 ? dt * kRK4A[s] : 0.0;
#pragma unroll
        for (int sp = 0; sp < 2; sp++) {
            double f[NH], K[NH];
#pragma unroll
            for (int e = 0; e < NH; e++) f[e] = Yin[(sp * NH + e) * cap + p];
            commutator<NF, double>(V + sp * NH, f, K, P.inv_hbar);
            const double Ns = S.Nn[sp][p];
#pragma unroll
            for (int e = 0; e < NH; e++) {
                const long long o = (sp * NH + e) * cap + p;
                if (s < 4) {
                    const double y0 = (s == 1) ? f[e] : Y0[o];
                    const double a0 = (s == 1) ? y0 : acc[o];
                    acc[o] = __dadd_rn(__dmul_rn(bw, K[e]), a0);
                    const double fn = __dadd_rn(__dmul_rn(aw, K[e]), y0);
                    Yout[o] = fn;
                    fN[sp * NH + e] = fn * Ns;
                } else {
                    Yout[o] = __dadd_rn(__dmul_rn(bw, K[e]), acc[o]);
                }
            }
        }
    }
    if (s < 4 && mesh_out)   // (null: the stage meshes are stored)
        tile_deposit_block<NF, SWt, double>(P, mesh_out, active, st, fN, vx, vy, vz,
                                            [](double a, int) -> double { return a; });
}

template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock) k_adj_fwd_stage(DevParams P, DevState S, int s, double dt,
                                                          const double* __restrict__ Yin, const double* __restrict__ Y0,
                                                          double* __restrict__ acc, double* __restrict__ Yout,
                                                          const double* __restrict__ mesh_in,
                                                          double* __restrict__ mesh_out)
{
    adj_fwd_stage_body<NF, SW<WX, WY, WZ>>(P, S, s, dt, Yin, Y0, acc, Yout, mesh_in, mesh_out);
}

// deposit of (f N) at S.pos (k_deposit's body)
template <int NF, class SWt>
__device__ __forceinline__ void adj_deposit_body(const DevParams& P, const DevState& S, const double* __restrict__ f,
                                                 double* __restrict__ mesh)
{
    constexpr int NH = NF * NF, NS = 2 * NH;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < S.n;
    Stencil<double> st{};
    double fN[NS] = {};
    double vx = 0, vy = 0, vz = 0;
    if (active) {
        make_stencil<double>(P, S.pos[0][p], S.pos[1][p], S.pos[2][p], st);
        vx = S.vhat[0][p];
        vy = S.vhat[1][p];
        vz = S.vhat[2][p];
#pragma unroll
        for (int c = 0; c < NS; c++) fN[c] = f[c * S.cap + p] * S.Nn[c / NH][p];
    }
    tile_deposit_block<NF, SWt, double>(P, mesh, active, st, fN, vx, vy, vz,
                                        [](double a, int) -> double { return a; }, true);
}

struct AdjStagePtrs {
    const double* Ys;       // stage state Y_s (s >= 1)
    const double* Ynext;    // Y_{s+1} (Y_0 for s = 0), gathered stage
    const double* Yn;       // pre-Renormalize state (s = 4)
    const double* mesh_s;   // forward mesh M_s (s >= 1)
    const double* lm_in;    // adjoint mesh of stage s+1 (s < 4)
    double* lm_out;         // adjoint mesh of stage s (s >= 1), zeroed
    double* lm_zero;        // adjoint mesh zeroed for the next launch
    long long nmesh;
    double* lamY0;          // in (s = 4): lam of the renormalised state; accumulates lam_Y0
    double* lamn;           // lam of Y_n
    double* lamYd;          // direct part C_Y^T lam_K of stage s
    double* lamN;           // [2][cap] accumulated dJ/dN, dJ/dNbar
};

// One backward launch: (s < 4) finish stage s+1 by gathering its adjoint
// mesh, (s >= 1) start stage s: commutator VJP and the scatter of lam_H.
// s = 4 starts from the Renormalize VJP.
template <int NF, class SWt>
__device__ __forceinline__ void adj_stage_body(const DevParams& P, const DevState& S, int s, double dt,
                                               const AdjStagePtrs& A)
{
    using H = Herm<NF>;
    constexpr int NH = NF * NF, NS = 2 * NH;
    zero_slice(A.lm_zero, A.nmesh);
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < S.n;
    const long long cap = S.cap;
    Stencil<double> st{};
    double g[NS] = {};
    double vx = 0, vy = 0, vz = 0;
    if (active) {
        make_stencil<double>(P, S.pos[0][p], S.pos[1][p], S.pos[2][p], st);
        vx = S.vhat[0][p];
        vy = S.vhat[1][p];
        vz = S.vhat[2][p];
        const double Nsp[2] = {S.Nn[0][p], S.Nn[1][p]};
        double lamK[NS], ln[NS];
        if (s == 4) {
#pragma unroll
            for (int sp = 0; sp < 2; sp++) {
                double y[NH], lr[NH];
#pragma unroll
                for (int e = 0; e < NH; e++) {
                    y[e] = A.Yn[(sp * NH + e) * cap + p];
                    lr[e] = A.lamY0[(sp * NH + e) * cap + p];
                }
                renormalize_vjp<NF>(y, S.Ll[sp][p], P.maxError, lr, ln + sp * NH);
            }
            const double b4 = dt * kRK4B[3];
#pragma unroll
            for (int c = 0; c < NS; c++) {
                A.lamn[c * cap + p] = ln[c];
                A.lamY0[c * cap + p] = ln[c];
                lamK[c] = b4 * ln[c];
            }
        } else {
            double G[NS];
            gather_deposit_adjoint<NF, SWt>(P, A.lm_in, st, vx, vy, vz, G);
            double dN[2] = {0.0, 0.0};
#pragma unroll
            for (int c = 0; c < NS; c++) {
                const int sp = c / NH;
                const long long o = c * cap + p;
                const double ly = A.lamYd[o] + Nsp[sp] * G[c];   // lam of Y_{s+1}
                dN[sp] += A.Ynext[o] * G[c];
                A.lamY0[o] += ly;
                if (s >= 1) lamK[c] = dt * kRK4B[s - 1] * A.lamn[o] + dt * kRK4A[s] * ly;
            }
            A.lamN[p] += dN[0];
            A.lamN[cap + p] += dN[1];
        }
        if (s >= 1) {
            double V[NS];
            potential_fp64<NF, SWt>(P, A.mesh_s, st, vx, vy, vz, S.vscale[p], V);
            double lH[NS];
#pragma unroll
            for (int sp = 0; sp < 2; sp++) {
                double y[NH], ly[NH];
#pragma unroll
                for (int e = 0; e < NH; e++) y[e] = A.Ys[(sp * NH + e) * cap + p];
                commutator_vjp<NF>(V + sp * NH, y, lamK + sp * NH, lH + sp * NH, ly, P.inv_hbar);
#pragma unroll
                for (int e = 0; e < NH; e++) A.lamYd[(sp * NH + e) * cap + p] = ly[e];
            }
            // I^T: V[e] += coef inside_e, V[NH+e] += (im ? +1 : -1) coef inside_e,
            // inside_e = SI_e (+/-) Sb_e with SI from the N/F fields of nu and
            // Sb from those of nubar (velocity terms enter with a minus sign)
#pragma unroll
            for (int e = 0; e < NH; e++) {
                const double li = P.sqrt2GF_inv_vol * (H::is_im(e) ? lH[e] + lH[NH + e] : lH[e] - lH[NH + e]);
                g[e] = li;
                g[NH + e] = H::is_im(e) ? li : -li;
            }
        }
    }
    if (s >= 1)
        tile_deposit_block<NF, SWt, double>(P, A.lm_out, active, st, g, -vx, -vy, -vz,
                                            [](double a, int) -> double { return a; });
}

template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock) k_adj_stage(DevParams P, DevState S, int s, double dt, AdjStagePtrs A)
{
    adj_stage_body<NF, SW<WX, WY, WZ>>(P, S, s, dt, A);
}

// Stage 4 of a recorded step with the step's completion: Y_n = acc + b4 dt K
// (stored), Y_new = Renormalize(Y_n), positions advanced and wrapped, and
// the deposit of Y_new at the new positions (the next step's M_1).  Same
// arithmetic as the forward stage kernel.
template <int NF, class SWt>
__device__ __forceinline__ void adj_fwd_stage4_next_body(const DevParams& P, const DevState& S, double dt,
                                                         const double* __restrict__ Y4, const double* __restrict__ acc,
                                                         double* __restrict__ Yn, double* __restrict__ Ynext,
                                                         double* __restrict__ xnext, const double* __restrict__ mesh_in,
                                                         double* __restrict__ mesh_next, StepCtl* report = nullptr)
{
    constexpr int NH = NF * NF, NS = 2 * NH;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < S.n;
    const long long cap = S.cap;
    Stencil<double> st{};
    double fN[NS] = {};
    double vx = 0, vy = 0, vz = 0;
    if (active) {
        const double x = S.pos[0][p], y = S.pos[1][p], z = S.pos[2][p];
        make_stencil<double>(P, x, y, z, st);
        vx = S.vhat[0][p];
        vy = S.vhat[1][p];
        vz = S.vhat[2][p];
        double V[NS];
        potential_fp64<NF, SWt>(P, mesh_in, st, vx, vy, vz, S.vscale[p], V);
        const double bw = dt * kRK4B[3];
        int stt = 0;
#pragma unroll
        for (int sp = 0; sp < 2; sp++) {
            double f[NH], K[NH];
#pragma unroll
            for (int e = 0; e < NH; e++) f[e] = Y4[(sp * NH + e) * cap + p];
            commutator<NF, double>(V + sp * NH, f, K, P.inv_hbar);
#pragma unroll
            for (int e = 0; e < NH; e++) {
                const long long o = (sp * NH + e) * cap + p;
                f[e] = __dadd_rn(__dmul_rn(bw, K[e]), acc[o]);
                Yn[o] = f[e];
            }
            if (Ynext) {
                stt |= renormalize<NF>(f, S.Ll[sp][p], P.maxError);
                const double Ns = S.Nn[sp][p];
#pragma unroll
                for (int e = 0; e < NH; e++) {
                    Ynext[(sp * NH + e) * cap + p] = f[e];
                    fN[sp * NH + e] = f[e] * Ns;
                }
            }
        }
        if (xnext) {
            double xn[3] = {x, y, z};
            const double kxv[3] = {vx * kC, vy * kC, vz * kC};
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const double w = dt * kRK4B[i];
#pragma unroll
                for (int d = 0; d < 3; d++) xn[d] = __dadd_rn(__dmul_rn(w, kxv[d]), xn[d]);
            }
#pragma unroll
            for (int d = 0; d < 3; d++) {
                xn[d] = wrap_coord(xn[d], P.L[d]);
                xnext[d * cap + p] = xn[d];
            }
            make_stencil<double>(P, xn[0], xn[1], xn[2], st);
        }
        if (report) report_bad(report, stt, S.id[p]);
    }
    if (mesh_next)
        tile_deposit_block<NF, SWt, double>(P, mesh_next, active, st, fN, vx, vy, vz,
                                            [](double a, int) -> double { return a; }, true);
}

template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock) k_adj_fwd_stage4_next(DevParams P, DevState S, double dt,
                                                                const double* __restrict__ Y4,
                                                                const double* __restrict__ acc, double* __restrict__ Yn,
                                                                double* __restrict__ Ynext, double* __restrict__ xnext,
                                                                const double* __restrict__ mesh_in,
                                                                double* __restrict__ mesh_next)
{
    adj_fwd_stage4_next_body<NF, SW<WX, WY, WZ>>(P, S, dt, Y4, acc, Yn, Ynext, xnext, mesh_in, mesh_next);
}

// One checkpoint segment of len steps, stored step by step:
//   seg  + j*seg_stride:  Y_0 (NS x cap) then x, y, z (cap each) of step j
//   sst  + j*sst_stride:  Y_2, Y_3, Y_4, Y_n (NS x cap each)
//   mst  + j*mst_stride:  M_1..M_4 (nmesh each)
struct SegPtrs {
    double* seg;
    long long seg_stride;
    double* sst;
    long long sst_stride;
    double* mst;
    long long mst_stride;
    const double* dts;
    double* dts_out;   // record: the forward run itself, dt from the device step control, stored here
    int record;
    int k0, len, NS;
    double* acc;
    double* lm[4];
    long long nmesh;
    double* lamY0;
    double* lamn;
    double* lamYd;
    double* lamN;
};

__host__ __device__ inline DevState seg_state(const DevState& S, const SegPtrs& G, int j)
{
    DevState Q = S;
    double* base = G.seg + j * G.seg_stride + (long long)G.NS * S.cap;
    for (int d = 0; d < 3; d++) Q.pos[d] = base + d * S.cap;
    return Q;
}

__host__ __device__ inline double* seg_f(const SegPtrs& G, int j) { return G.seg + j * G.seg_stride; }

__host__ __device__ inline double* seg_y(const SegPtrs& G, int j, int s, long long cap)
{
    // s = 2, 3, 4 stage states, 5 = Y_n
    return G.sst + j * G.sst_stride + (long long)(s - 2) * G.NS * cap;
}

__host__ __device__ inline double* seg_m(const SegPtrs& G, int j, int i) { return G.mst + j * G.mst_stride + i * G.nmesh; }

__host__ __device__ inline AdjStagePtrs seg_stage_ptrs(const SegPtrs& G, int j, int s, long long cap)
{
    const double* Y[6] = {seg_f(G, j), seg_f(G, j), seg_y(G, j, 2, cap), seg_y(G, j, 3, cap), seg_y(G, j, 4, cap),
                          seg_y(G, j, 5, cap)};
    AdjStagePtrs A{};
    A.Ys = s >= 1 ? Y[s] : nullptr;
    A.Ynext = s < 4 ? Y[s + 1] : nullptr;
    A.Yn = Y[5];
    A.mesh_s = s >= 1 ? seg_m(G, j, s - 1) : nullptr;
    A.lm_in = s < 4 ? G.lm[(s + 1) % 4] : nullptr;
    A.lm_out = s >= 1 ? G.lm[s % 4] : nullptr;
    A.lm_zero = s >= 1 ? G.lm[(s + 3) % 4] : nullptr;
    A.nmesh = G.nmesh;
    A.lamY0 = G.lamY0;
    A.lamn = G.lamn;
    A.lamYd = G.lamYd;
    A.lamN = G.lamN;
    return A;
}

// Forward over a whole segment in one cooperative launch (Y_0 and x of step
// 0 and its deposit M_1 are in place; every stored mesh starts at zero):
// four phases per step separated by bounded grid barriers.
template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock, 4) k_adj_seg_fwd_coop(DevParams P, DevState S, SegPtrs G, StepCtl* ctl)
{
    using SWt = SW<WX, WY, WZ>;
    const long long cap = S.cap;
#pragma unroll 1
    for (int j = 0; j < G.len; j++) {
        const DevState Q = seg_state(S, G, j);
        // recording: this step's dt from the device control (every block
        // reads it before any block can reach the reduction that replaces it)
        const double dt = G.record ? __ldcg(&ctl->dt) : G.dts[G.k0 + j];
        if (G.record && blockIdx.x == 0 && threadIdx.x == 0) G.dts_out[G.k0 + j] = dt;
        const double* Y0 = seg_f(G, j);
#pragma unroll 1
        for (int s = 1; s <= 3; s++) {
            adj_fwd_stage_body<NF, SWt>(P, Q, s, dt, s == 1 ? Y0 : seg_y(G, j, s, cap), Y0, G.acc,
                                        seg_y(G, j, s + 1, cap), seg_m(G, j, s - 1), seg_m(G, j, s));
            grid_barrier(ctl, P.wait_polls);
        }
        // recording: compute_dt on the stage-4 mesh (main.cpp:193-198), the
        // next step's dt; M_4 is complete and every block holds this step's
        // dt, so it overlaps stage 4 and shares its barrier
        if (G.record) dt_reduce_and_finish<NF, double>(P, seg_m(G, j, 3), ctl, DT_ADVANCE, reduce_blocks(P));
        // (recording: the state after the segment goes to slot len too)
        const bool more = j + 1 < G.len, next = more || G.record;
        adj_fwd_stage4_next_body<NF, SWt>(P, Q, dt, seg_y(G, j, 4, cap), G.acc, seg_y(G, j, 5, cap),
                                          next ? seg_f(G, j + 1) : nullptr,
                                          next ? seg_f(G, j + 1) + (long long)G.NS * cap : nullptr, seg_m(G, j, 3),
                                          more ? seg_m(G, j + 1, 0) : nullptr, G.record ? ctl : nullptr);
        grid_barrier(ctl, P.wait_polls);
        if (G.record && __ldcg(&ctl->done) && more) break;   // (uniform: read after the barrier)
    }
}

// composition of a re-sort (new slot i holds old slot g[i]) into the map of
// slots to segment-start slots
__global__ void k_compose_map(const unsigned* __restrict__ map_old, const unsigned* __restrict__ g,
                              unsigned* __restrict__ map_new, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) map_new[i] = map_old ? map_old[g[i]] : g[i];
}

// particle time of a recorded segment: time += dt_j * b_i, stage by stage and
// step by step, in the order of the step kernels
__global__ void k_time_advance(DevState S, const double* __restrict__ dts, int k0, int len)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= S.n) return;
    double tn = S.time[p];
    for (int j = 0; j < len; j++) {
        const double dt = dts[k0 + j];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const double w = dt * kRK4B[i];
            tn = __dadd_rn(w, tn);
        }
    }
    S.time[p] = tn;
}

// Backward over a whole segment in one cooperative launch: five phases per
// step, last step first.
template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock, 4) k_adj_seg_bwd_coop(DevParams P, DevState S, SegPtrs G, StepCtl* ctl)
{
    using SWt = SW<WX, WY, WZ>;
    const long long cap = S.cap;
#pragma unroll 1
    for (int j = G.len - 1; j >= 0; j--) {
        const DevState Q = seg_state(S, G, j);
        const double dt = G.dts[G.k0 + j];
#pragma unroll 1
        for (int s = 4; s >= 0; s--) {
            adj_stage_body<NF, SWt>(P, Q, s, dt, seg_stage_ptrs(G, j, s, cap));
            grid_barrier(ctl, P.wait_polls);
        }
    }
}

// copy (f, x) of the recompute state into a segment slot and set the
// control dt of the step about to be recomputed
__global__ void k_seg_save(DevState R, double* __restrict__ slot, int NS, const double* __restrict__ dts, int k,
                           StepCtl* ctl)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0 && ctl) ctl->dt = dts[k];
    if (p >= R.n || !slot) return;   // (no slot: only the dt of step k)
    const long long cap = R.cap;
    for (int c = 0; c < NS; c++) slot[c * cap + p] = R.f0[c * cap + p];
    for (int d = 0; d < 3; d++) slot[(NS + d) * cap + p] = R.pos[d][p];
}

// static particle fields (and the carried adjoint state) from one slot
// order to another: dst[perm[i]] = src[i] (perm = NULL: same order)
__global__ void k_static_scatter(DevState src, DevState dst, const unsigned* __restrict__ perm,
                                 const double* __restrict__ lsrc, double* __restrict__ ldst, int nl)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= src.n) return;
    const long long j = perm ? (long long)perm[i] : i;
    const long long cap = src.cap;
    for (int d = 0; d < 3; d++) dst.vhat[d][j] = src.vhat[d][i];
    for (int d = 0; d < 4; d++) dst.pup[d][j] = src.pup[d][i];
    for (int sp = 0; sp < 2; sp++) {
        dst.Nn[sp][j] = src.Nn[sp][i];
        dst.Ll[sp][j] = src.Ll[sp][i];
    }
    dst.vscale[j] = src.vscale[i];
    dst.id[j] = src.id[i];
    if (lsrc)
        for (int c = 0; c < nl; c++) ldst[c * cap + j] = lsrc[c * cap + i];
}

// the same, gathering: dst[i] = src[perm[i]] (the forward direction of a re-sort)
__global__ void k_static_gather(DevState src, DevState dst, const unsigned* __restrict__ perm)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= src.n) return;
    const long long j = perm[i];
    for (int d = 0; d < 3; d++) dst.vhat[d][i] = src.vhat[d][j];
    for (int d = 0; d < 4; d++) dst.pup[d][i] = src.pup[d][j];
    for (int sp = 0; sp < 2; sp++) {
        dst.Nn[sp][i] = src.Nn[sp][j];
        dst.Ll[sp][i] = src.Ll[sp][j];
    }
    dst.vscale[i] = src.vscale[j];
    dst.id[i] = src.id[j];
}

// nc component arrays of stride cap: dst[c][i] = src[c][perm[i]]
__global__ void k_rows_gather(const double* __restrict__ src, double* __restrict__ dst, const unsigned* __restrict__ perm,
                              int nc, long long cap, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long j = perm[i];
    for (int c = 0; c < nc; c++) dst[c * cap + i] = src[c * cap + j];
}

// objective: lam_M = 2/V_cell M on the nu e-mu components, zero elsewhere;
// the two components per cell go to nex for the host sum
template <int NF>
__global__ void k_adj_nex(DevParams P, const double* __restrict__ mesh, double* __restrict__ lm,
                          double* __restrict__ nex)
{
    constexpr int ND = 8 * NF * NF;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncells) return;
    const double inv_vol = P.dxi[0] * P.dxi[1] * P.dxi[2];
    const int kre = Herm<NF>::re(0, 1), kim = Herm<NF>::im(0, 1);
    const double a = mesh[c * ND + kre], b = mesh[c * ND + kim];
    nex[2 * c] = a;
    nex[2 * c + 1] = b;
    lm[c * ND + kre] = 2.0 * inv_vol * a;
    lm[c * ND + kim] = 2.0 * inv_vol * b;
}

// lam of one state (f, N) from an adjoint mesh: lam_f = N D^T lam_M,
// lam_N = f . D^T lam_M
template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock) k_adj_gather(DevParams P, DevState S, const double* __restrict__ lm,
                                                       double* __restrict__ lamf, double* __restrict__ lamN)
{
    constexpr int NH = NF * NF, NS = 2 * NH;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= S.n) return;
    const long long cap = S.cap;
    Stencil<double> st;
    make_stencil<double>(P, S.pos[0][p], S.pos[1][p], S.pos[2][p], st);
    double G[NS];
    gather_deposit_adjoint<NF, SW<WX, WY, WZ>>(P, lm, st, S.vhat[0][p], S.vhat[1][p], S.vhat[2][p], G);
    double dN[2] = {0.0, 0.0};
#pragma unroll
    for (int c = 0; c < NS; c++) {
        const int sp = c / NH;
        lamf[c * cap + p] = S.Nn[sp][p] * G[c];
        dN[sp] += S.f0[c * cap + p] * G[c];
    }
    lamN[p] = dN[0];
    lamN[cap + p] = dN[1];
}

// slot-order SoA [ncomp][cap] <-> load-order rows [n][ncomp]
__global__ void k_soa_to_rows(const long long* __restrict__ id, const double* __restrict__ src, int ncomp,
                              long long cap, long long n, double* __restrict__ dst)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const long long r = id[p];
    for (int c = 0; c < ncomp; c++) dst[r * ncomp + c] = src[c * cap + p];
}

__global__ void k_rows_to_soa(const long long* __restrict__ id, const double* __restrict__ src, int ncomp,
                              long long cap, long long n, double* __restrict__ dst)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const long long r = id[p];
    for (int c = 0; c < ncomp; c++) dst[c * cap + p] = src[r * ncomp + c];
}

// ---- launchers ----------------------------------------------------------------
template <int NF>
void launch_adj_fwd_stage_t(const DevParams& P, const DevState& S, int s, double dt, const double* Yin,
                            const double* Y0, double* acc, double* Yout, const double* mesh_in, double* mesh_out,
                            cudaStream_t st)
{
    EMU_W_DISPATCH(P, {
        constexpr int bytes = tile_smem_bytes<NF, SW<WXv, WYv, WZv>, double>();
        smem_optin(k_adj_fwd_stage<NF, WXv, WYv, WZv>, bytes);
        k_adj_fwd_stage<NF, WXv, WYv, WZv><<<grid_for(S.n), kBlock, bytes, st>>>(P, S, s, dt, Yin, Y0, acc, Yout,
                                                                                 mesh_in, mesh_out);
    });
}

template <int NF>
void launch_adj_stage_t(const DevParams& P, const DevState& S, int s, double dt, const AdjStagePtrs& A,
                        cudaStream_t st)
{
    EMU_W_DISPATCH(P, {
        constexpr int bytes = tile_smem_bytes<NF, SW<WXv, WYv, WZv>, double>();
        smem_optin(k_adj_stage<NF, WXv, WYv, WZv>, bytes);
        k_adj_stage<NF, WXv, WYv, WZv><<<grid_for(S.n), kBlock, bytes, st>>>(P, S, s, dt, A);
    });
}

template <int NF>
void launch_adj_gather_t(const DevParams& P, const DevState& S, const double* lm, double* lamf, double* lamN,
                         cudaStream_t st)
{
    EMU_W_DISPATCH(P, { k_adj_gather<NF, WXv, WYv, WZv><<<grid_for(S.n), kBlock, 0, st>>>(P, S, lm, lamf, lamN); });
}

template <int NF, class K>
bool coop_fits(K kern, int bytes, long long n)
{
    smem_optin(kern, bytes);
    int per_sm = 0, dev = 0, nsm = 0;
    const bool ok = cudaGetDevice(&dev) == cudaSuccess &&
                    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
                    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, bytes) == cudaSuccess &&
                    (long long)per_sm * nsm >= (long long)grid_for(n);
    cudaGetLastError();
    return ok;
}

template <int NF>
bool adj_coop_fits_t(const DevParams& P, long long n)
{
    bool ok = false;
    EMU_W_DISPATCH(P, {
        constexpr int bytes = tile_smem_bytes<NF, SW<WXv, WYv, WZv>, double>();
        ok = coop_fits<NF>(k_adj_seg_fwd_coop<NF, WXv, WYv, WZv>, bytes, n) &&
             coop_fits<NF>(k_adj_seg_bwd_coop<NF, WXv, WYv, WZv>, bytes, n);
    });
    return ok;
}

template <int NF>
cudaError_t launch_adj_seg_coop_t(bool forward, const DevParams& P, const DevState& S, const SegPtrs& G,
                                  StepCtl* ctl, cudaStream_t st)
{
    cudaError_t err = cudaSuccess;
    EMU_W_DISPATCH(P, {
        constexpr int bytes = tile_smem_bytes<NF, SW<WXv, WYv, WZv>, double>();
        smem_optin(k_adj_seg_fwd_coop<NF, WXv, WYv, WZv>, bytes);
        smem_optin(k_adj_seg_bwd_coop<NF, WXv, WYv, WZv>, bytes);
        const void* kern = forward ? (const void*)k_adj_seg_fwd_coop<NF, WXv, WYv, WZv>
                                   : (const void*)k_adj_seg_bwd_coop<NF, WXv, WYv, WZv>;
        DevParams Pc = P;
        DevState Sc = S;
        SegPtrs Gc = G;
        StepCtl* c = ctl;
        void* args[] = {&Pc, &Sc, &Gc, &c};
        err = cudaLaunchCooperativeKernel(kern, dim3(grid_for(S.n)), dim3(kBlock), args, bytes, st);
    });
    return err;
}

template <int NF>
void launch_adj_fwd_stage4_next_t(const DevParams& P, const DevState& S, double dt, const double* Y4,
                                  const double* acc, double* Yn, double* Ynext, double* xnext, const double* mesh_in,
                                  double* mesh_next, cudaStream_t st)
{
    EMU_W_DISPATCH(P, {
        constexpr int bytes = tile_smem_bytes<NF, SW<WXv, WYv, WZv>, double>();
        smem_optin(k_adj_fwd_stage4_next<NF, WXv, WYv, WZv>, bytes);
        k_adj_fwd_stage4_next<NF, WXv, WYv, WZv><<<grid_for(S.n), kBlock, bytes, st>>>(P, S, dt, Y4, acc, Yn, Ynext,
                                                                                       xnext, mesh_in, mesh_next);
    });
}

// two flavors only: the three-flavor backward body needs more than the
// 128 registers a co-resident grid of 4 CTAs per SM allows
bool adj_coop_fits(int nf, const DevParams& P, long long n)
{
    return nf == 2 && adj_coop_fits_t<2>(P, n);
}

void launch_compose_map(const unsigned* map_old, const unsigned* g, unsigned* map_new, long long n, cudaStream_t st)
{
    k_compose_map<<<grid_for(n), kBlock, 0, st>>>(map_old, g, map_new, n);
}

void launch_time_advance(const DevState& S, const double* dts, int k0, int len, cudaStream_t st)
{
    k_time_advance<<<grid_for(S.n), kBlock, 0, st>>>(S, dts, k0, len);
}

cudaError_t launch_adj_seg_coop(int nf, bool forward, const DevParams& P, const DevState& S, const SegPtrs& G,
                                StepCtl* ctl, cudaStream_t st)
{
    return nf == 2 ? launch_adj_seg_coop_t<2>(forward, P, S, G, ctl, st) : cudaErrorInvalidValue;
}

void launch_adj_fwd_stage4_next(int nf, const DevParams& P, const DevState& S, double dt, const double* Y4,
                                const double* acc, double* Yn, double* Ynext, double* xnext, const double* mesh_in,
                                double* mesh_next, cudaStream_t st)
{
    if (nf == 2) launch_adj_fwd_stage4_next_t<2>(P, S, dt, Y4, acc, Yn, Ynext, xnext, mesh_in, mesh_next, st);
    else launch_adj_fwd_stage4_next_t<3>(P, S, dt, Y4, acc, Yn, Ynext, xnext, mesh_in, mesh_next, st);
}

void launch_adj_fwd_stage(int nf, const DevParams& P, const DevState& S, int s, double dt, const double* Yin,
                          const double* Y0, double* acc, double* Yout, const double* mesh_in, double* mesh_out,
                          cudaStream_t st)
{
    if (nf == 2) launch_adj_fwd_stage_t<2>(P, S, s, dt, Yin, Y0, acc, Yout, mesh_in, mesh_out, st);
    else launch_adj_fwd_stage_t<3>(P, S, s, dt, Yin, Y0, acc, Yout, mesh_in, mesh_out, st);
}

void launch_adj_stage(int nf, const DevParams& P, const DevState& S, int s, double dt, const AdjStagePtrs& A,
                      cudaStream_t st)
{
    if (nf == 2) launch_adj_stage_t<2>(P, S, s, dt, A, st);
    else launch_adj_stage_t<3>(P, S, s, dt, A, st);
}

void launch_adj_gather(int nf, const DevParams& P, const DevState& S, const double* lm, double* lamf, double* lamN,
                       cudaStream_t st)
{
    if (nf == 2) launch_adj_gather_t<2>(P, S, lm, lamf, lamN, st);
    else launch_adj_gather_t<3>(P, S, lm, lamf, lamN, st);
}

void launch_adj_nex(int nf, const DevParams& P, const double* mesh, double* lm, double* nex, cudaStream_t st)
{
    if (nf == 2) k_adj_nex<2><<<grid_for(P.ncells), kBlock, 0, st>>>(P, mesh, lm, nex);
    else k_adj_nex<3><<<grid_for(P.ncells), kBlock, 0, st>>>(P, mesh, lm, nex);
}

}  // namespace
}  // namespace emu

// ============================================================================
// host side
// ============================================================================
namespace {

long long mesh_elems(const emu_context* c) { return c->P.ncells * c->ND; }

void free_adj(emu_adjoint* a)
{
    if (!a) return;
    for (void* p : {(void*)a->dts_dev, (void*)a->ck, (void*)a->seg, (void*)a->work, (void*)a->nex, (void*)a->rows,
                    (void*)a->perm, (void*)a->stat, (void*)a->sst, (void*)a->mst, (void*)a->map[0], (void*)a->map[1],
                    (void*)a->wf2, (void*)a->wpos2, (void*)a->gperm, (void*)a->smap, (void*)a->smesh})
        if (p) emu_ctx::dev_free(p);
    for (int i = 0; i < 4; i++)
        if (a->lmesh[i]) emu_ctx::dev_free(a->lmesh[i]);
    delete a;
}

// static-field view of one of the two working blocks (12 doubles + id per slot)
DevState stat_view(emu_adjoint* a, int w, const DevState& like)
{
    DevState W = like;
    char* p = reinterpret_cast<char*>(a->stat) + (size_t)w * 13 * 8 * a->cap;
    auto take = [&](long long count) {
        double* r = reinterpret_cast<double*>(p);
        p += (size_t)count * 8;
        return r;
    };
    for (int d = 0; d < 3; d++) W.vhat[d] = take(a->cap);
    for (int d = 0; d < 4; d++) W.pup[d] = take(a->cap);
    for (int sp = 0; sp < 2; sp++) W.Nn[sp] = take(a->cap);
    for (int sp = 0; sp < 2; sp++) W.Ll[sp] = take(a->cap);
    W.vscale = take(a->cap);
    W.id = reinterpret_cast<long long*>(take(a->cap));
    return W;
}

// Sub-segments of a segment of len steps over B segment slots (per-step
// mode with re-sorts).  Sub-segment i >= 1 starts from its sub-checkpoint in
// slot i - 1 and keeps its later states in slots i, i + 1, ... (the
// sub-checkpoints of the sub-segments after it are consumed by then);
// sub-segment 0 starts from the segment checkpoint and keeps its later
// states in slots 0, 1, ...  So sub-segment i holds at most B + 1 (i = 0) or
// B - i + 1 steps.  The fewest sub-segments, the later ones as long as
// allowed: the sub-checkpoint pass stops at the last one's start.  Returns
// the starts relative to the segment (nsub + 1 entries, the last = len), or
// nothing when B slots cannot hold len steps.
std::vector<int> rps_layout(int len, int B)
{
    auto most = [&](int i) { return i == 0 ? B + 1 : B - i + 1; };
    int nsub = 0;
    long long tot = 0;
    while (tot < len) {
        if (most(nsub) <= 0) return {};
        tot += most(nsub);
        nsub++;
    }
    std::vector<int> L(nsub);
    int rem = len;
    for (int i = nsub - 1; i >= 1; i--) {
        L[i] = std::min(most(i), rem - i);   // (at least one step left for each earlier one)
        rem -= L[i];
    }
    L[0] = rem;
    std::vector<int> sb(nsub + 1, 0);
    for (int i = 0; i < nsub; i++) sb[i + 1] = sb[i] + L[i];
    return sb;
}

// device arrays for a recorded run of nsteps with checkpoints every interval
int ensure_adj(emu_context* ctx, int nsteps, int interval)
{
    const long long cap = ctx->cap;
    const int NS = ctx->NS;
    const int nck = (nsteps + interval - 1) / interval;
    const long long nm = mesh_elems(ctx);
    emu_adjoint* a = ctx->adj;
    if (a && (a->cap != cap || a->NS != NS || a->ck_slots < nck || a->interval_cap < interval ||
              (int)a->dts.size() < nsteps || (a->full && a->full_steps < nsteps))) {
        free_adj(a);
        a = ctx->adj = nullptr;
    }
    if (!a) {
        a = new emu_adjoint();
        ctx->adj = a;
        a->cap = cap;
        a->NS = NS;
        a->dts.resize(std::max(nsteps, 1));
        a->ck_slots = std::max(nck, 1);
        a->interval_cap = interval;
        a->resorted.assign(a->ck_slots, 0);
        const size_t slot = (size_t)(NS + 3) * cap;
        // stage states and meshes of every step of a segment when they take
        // at most a quarter of the free memory (and 16 GiB); otherwise one
        // step's worth, recomputed step by step
        size_t fre = 0, tot = 0;
        cudaMemGetInfo(&fre, &tot);
        size_t budget = std::min(fre / 4, (size_t)16 << 30);
        if (const char* env = std::getenv("EMU_ADJOINT_STORE_MAX_BYTES")) budget = (size_t)std::strtoull(env, nullptr, 10);
        const size_t per_step = sizeof(double) * ((size_t)4 * NS * cap + (size_t)4 * nm);
        a->store = (size_t)interval * per_step <= budget;
        const char* fenv = std::getenv("EMU_ADJOINT_FULL_STORE");
        a->full = a->store && (!fenv || std::atoi(fenv) != 0) &&
                  emu::adj_coop_fits(ctx->nf, ctx->P, ctx->S[ctx->cur].n) &&
                  (size_t)nsteps * (per_step + sizeof(double) * slot) <= budget;
        a->full_steps = a->full ? nsteps : 0;
        const size_t st_steps = a->full ? (size_t)nsteps : a->store ? (size_t)interval : 1;
        // per-step mode: the states of every step of a segment (interval
        // slots), or, when the checkpoints and those slots would not fit in
        // the free memory, sub-checkpoints every J ~ sqrt(interval) steps
        // (J + interval / J slots; each step is recomputed once more)
        a->sub = 0;
        a->seg_slots = a->full ? nsteps + 1 : interval;
        if (!a->store) {
            const size_t other = sizeof(double) * ((size_t)st_steps * 4 * (NS * cap + nm) + (size_t)(6 * NS + 8) * cap +
                                                   (size_t)4 * nm + (size_t)NS * cap + 2 * 13 * cap +
                                                   (size_t)(NS + 3) * cap) +
                                 sizeof(unsigned) * (size_t)cap * (a->ck_slots + 3 + 2 * (size_t)interval);
            const size_t single = sizeof(double) * slot * (size_t)(a->ck_slots + interval) + other;
            int J = 0;
            if (single > fre / 20 * 19) J = (int)std::ceil(std::sqrt((double)interval));
            if (const char* env = std::getenv("EMU_ADJOINT_SUBCHECKPOINT")) J = std::atoi(env);
            if (J > 0 && J < interval) {
                a->sub = J;
                a->seg_slots = J + (interval + J - 1) / J;
            }
        }
        // per-step mode with re-sorts: the sub-segment layout over the
        // segment slots (EMU_ADJOINT_SEG_SLOTS: fewer slots, for tests)
        std::vector<int> rps_sb;
        if (!a->store && ctx->prm.resort_interval > 0) {
            int B = a->seg_slots;
            if (const char* env = std::getenv("EMU_ADJOINT_SEG_SLOTS")) B = std::max(1, std::min(B, std::atoi(env)));
            rps_sb = rps_layout(interval, B);
            if (rps_sb.empty()) {
                free_adj(a);
                ctx->adj = nullptr;
                return fail(ctx, EMU_ERR_ARG, "adjoint: too few segment slots for the checkpoint interval");
            }
            a->rps_slots = B;
        }
        a->bytes = 0;
        auto alloc = [&](auto** ptr, size_t b) {
            a->bytes += b;
            return emu_ctx::dev_malloc(reinterpret_cast<void**>(ptr), b);
        };
        CU(alloc(&a->dts_dev, sizeof(double) * a->dts.size()));
        CU(alloc(&a->ck, sizeof(double) * slot * a->ck_slots));
        CU(alloc(&a->seg, sizeof(double) * slot * a->seg_slots));
        CU(alloc(&a->perm, sizeof(unsigned) * cap * (a->ck_slots + 1)));
        CU(alloc(&a->stat, (size_t)2 * 13 * 8 * cap));
        CU(alloc(&a->sst, sizeof(double) * st_steps * 4 * NS * cap));
        CU(alloc(&a->mst, sizeof(double) * st_steps * 4 * nm));
        // acc, lamY0, lamn, lamYd, wf, lamtmp: 6 NS; lamN 2, lamtmp 2; wpos 3; wtime 1
        CU(alloc(&a->work, sizeof(double) * (size_t)(6 * NS + 8) * cap));
        for (int i = 0; i < 4; i++) CU(alloc(&a->lmesh[i], sizeof(double) * nm));
        CU(alloc(&a->nex, sizeof(double) * 2 * ctx->P.ncells));
        CU(alloc(&a->rows, sizeof(double) * (size_t)NS * cap));
        for (int i = 0; i < 2; i++) CU(alloc(&a->map[i], sizeof(unsigned) * cap));
        if (!a->store && ctx->prm.resort_interval > 0) {
            // (a shorter last segment may form one sub-segment of up to
            // B + 1 steps; a full one has the most sub-segments)
            a->gslots = std::min(a->rps_slots + 1, interval);
            a->sslots = (int)rps_sb.size() - 1;
            CU(alloc(&a->wf2, sizeof(double) * (size_t)NS * cap));
            CU(alloc(&a->wpos2, sizeof(double) * (size_t)3 * cap));
            CU(alloc(&a->gperm, sizeof(unsigned) * (size_t)a->gslots * cap));
            CU(alloc(&a->smap, sizeof(unsigned) * (size_t)a->sslots * cap));
            size_t f2 = 0, t2 = 0;
            cudaMemGetInfo(&f2, &t2);
            const size_t mb = sizeof(double) * (size_t)a->gslots * 4 * nm;
            const char* menv = std::getenv("EMU_ADJOINT_STORE_MESHES");
            if ((!menv || std::atoi(menv) != 0) && mb + ((size_t)2 << 30) <= f2) CU(alloc(&a->smesh, mb));
        }
        double* w = a->work;
        a->acc = w; w += (size_t)NS * cap;
        a->lamY0 = w; w += (size_t)NS * cap;
        a->lamN = w; w += (size_t)2 * cap;        // lamN follows lamY0: one (NS+2) x cap block
        a->lamn = w; w += (size_t)NS * cap;
        a->lamYd = w; w += (size_t)NS * cap;
        a->wf = w; w += (size_t)NS * cap;
        a->lamtmp = w; w += (size_t)(NS + 2) * cap;
        a->wpos = w; w += (size_t)3 * cap;
        a->wtime = w;
    }
    a->nsteps = nsteps;
    a->interval = interval;
    a->nck = nck;
    return EMU_OK;
}

double* slot_f(emu_adjoint* a, double* base, long long i) { return base + (size_t)i * (a->NS + 3) * a->cap; }
double* slot_x(emu_adjoint* a, double* base, long long i, int d)
{
    return slot_f(a, base, i) + (size_t)(a->NS + d) * a->cap;
}

int save_slot(emu_context* ctx, emu_adjoint* a, double* base, long long i, const double* f, double* const pos[3])
{
    const size_t fb = sizeof(double) * (size_t)a->NS * a->cap, xb = sizeof(double) * a->cap;
    CU(cudaMemcpyAsync(slot_f(a, base, i), f, fb, cudaMemcpyDeviceToDevice, ctx->stream));
    for (int d = 0; d < 3; d++)
        CU(cudaMemcpyAsync(slot_x(a, base, i, d), pos[d], xb, cudaMemcpyDeviceToDevice, ctx->stream));
    return EMU_OK;
}

int check_ready(emu_context* ctx, const char* who)
{
    if (!ctx->loaded) return fail(ctx, EMU_ERR_STATE, std::string(who) + ": no particles loaded");
    if (ctx->mixed) return fail(ctx, EMU_ERR_ARG, std::string(who) + ": the adjoint is FP64 only");
    if (ctx->comm || ctx->local) return fail(ctx, EMU_ERR_ARG, std::string(who) + ": the adjoint runs on one GPU");
    if (!(ctx->prm.integration_type == 1 && ctx->prm.rk_type == 4))
        return fail(ctx, EMU_ERR_ARG, std::string(who) + ": the adjoint differentiates RK4 only");
    return EMU_OK;
}

// deposit of (f, x) into mesh (zeroed first)
int deposit_into(emu_context* ctx, const DevState& S, const double* f, double* mesh)
{
    CU(cudaMemsetAsync(mesh, 0, sizeof(double) * mesh_elems(ctx), ctx->stream));
    emu::launch_deposit(ctx->nf, ctx->P, S, f, mesh, ctx->stream);
    return check_launch(ctx, "adjoint deposit");
}

// forward over steps [0, len) of G (step 0's Y_0, x in place, stored meshes
// zeroed), storing stage states and meshes, then the backward sweep.
// meshes_given: G's meshes M_1..M_4 already hold the step's deposits (one
// step, not cooperative); the forward only recomputes the stage states.
int segment_sweep(emu_context* ctx, const DevState& W, const emu::SegPtrs& G, bool coop, bool meshes_given = false)
{
    const int nf = ctx->nf;
    const long long cap = ctx->cap;
    cudaStream_t st = ctx->stream;
    int r;
    if (!meshes_given &&
        (r = deposit_into(ctx, emu::seg_state(W, G, 0), emu::seg_f(G, 0), emu::seg_m(G, 0, 0))))
        return r;
    if (coop) {
        cudaError_t e = emu::launch_adj_seg_coop(nf, true, ctx->P, W, G, ctx->ctl, st);
        if (e == cudaSuccess) e = emu::launch_adj_seg_coop(nf, false, ctx->P, W, G, ctx->ctl, st);
        if (e != cudaSuccess) return fail(ctx, EMU_ERR_CUDA, std::string("adjoint segment: ") + cudaGetErrorString(e));
        return check_launch(ctx, "adjoint segment");
    }
    for (int j = 0; j < G.len; j++) {
        const DevState Q = emu::seg_state(W, G, j);
        const double dt = ctx->adj->dts[G.k0 + j];
        const double* Y0 = emu::seg_f(G, j);
        for (int s = 1; s <= 3; s++)
            emu::launch_adj_fwd_stage(nf, ctx->P, Q, s, dt, s == 1 ? Y0 : emu::seg_y(G, j, s, cap), Y0, G.acc,
                                      emu::seg_y(G, j, s + 1, cap), emu::seg_m(G, j, s - 1),
                                      meshes_given ? nullptr : emu::seg_m(G, j, s), st);
        const bool more = j + 1 < G.len;
        emu::launch_adj_fwd_stage4_next(nf, ctx->P, Q, dt, emu::seg_y(G, j, 4, cap), G.acc, emu::seg_y(G, j, 5, cap),
                                        more ? emu::seg_f(G, j + 1) : nullptr,
                                        more ? emu::seg_f(G, j + 1) + (long long)G.NS * cap : nullptr,
                                        emu::seg_m(G, j, 3), more ? emu::seg_m(G, j + 1, 0) : nullptr, st);
    }
    for (int j = G.len - 1; j >= 0; j--) {
        const DevState Q = emu::seg_state(W, G, j);
        const double dt = ctx->adj->dts[G.k0 + j];
        for (int s = 4; s >= 0; s--) emu::launch_adj_stage(nf, ctx->P, Q, s, dt, emu::seg_stage_ptrs(G, j, s, cap), st);
    }
    return check_launch(ctx, "adjoint segment");
}

// The recorded forward run when every step's states fit (a->full): per
// segment a cell re-sort at its start (as the step loop), then one
// cooperative launch that advances the segment with dt from the device step
// control, storing Y_0 and x, the stage states and the meshes of every step
// (what the backward would otherwise recompute), then the particle time and
// the state after the segment back into the context.
int record_full(emu_context* ctx, emu_adjoint* a, int nsteps, int interval)
{
    const int NS = ctx->NS;
    const long long cap = ctx->cap, nm = mesh_elems(ctx);
    cudaStream_t st = ctx->stream;
    int r;
    emu::SegPtrs G{};
    G.seg_stride = (long long)(NS + 3) * cap;
    G.sst_stride = (long long)4 * NS * cap;
    G.mst_stride = 4 * nm;
    G.dts = a->dts_dev;
    G.dts_out = a->dts_dev;
    G.record = 1;
    G.NS = NS;
    G.acc = a->acc;
    G.nmesh = nm;
    const int nseg = (nsteps + interval - 1) / interval;
    for (int c = 0; c < nseg; c++) {
        const int k0 = c * interval, len = std::min(k0 + interval, nsteps) - k0;
        if (c > 0 && ctx->prm.resort_interval > 0) {
            if ((r = emu_ctx::resort_now(ctx, a->perm + (size_t)c * a->cap))) return r;
            a->resorted[c] = 1;
        }
        const DevState& S = ctx->S[ctx->cur];
        if ((r = save_slot(ctx, a, a->ck, c, S.f0, S.pos))) return r;
        if ((r = save_slot(ctx, a, a->seg, k0, S.f0, S.pos))) return r;
        G.seg = a->seg + (size_t)k0 * G.seg_stride;
        G.sst = a->sst + (size_t)k0 * G.sst_stride;
        G.mst = a->mst + (size_t)k0 * G.mst_stride;
        G.k0 = k0;
        G.len = len;
        CU(cudaMemsetAsync(G.mst, 0, sizeof(double) * (size_t)len * 4 * nm, st));
        if ((r = deposit_into(ctx, emu::seg_state(S, G, 0), emu::seg_f(G, 0), emu::seg_m(G, 0, 0)))) return r;
        cudaError_t e = emu::launch_adj_seg_coop(ctx->nf, true, ctx->P, S, G, ctx->ctl, st);
        if (e != cudaSuccess) return fail(ctx, EMU_ERR_CUDA, std::string("recorded segment: ") + cudaGetErrorString(e));
        emu::launch_time_advance(S, a->dts_dev, k0, len, st);
        CU(cudaMemcpyAsync(S.f0, emu::seg_f(G, len), sizeof(double) * (size_t)NS * cap, cudaMemcpyDeviceToDevice, st));
        for (int d = 0; d < 3; d++)
            CU(cudaMemcpyAsync(S.pos[d], emu::seg_f(G, len) + (size_t)(NS + d) * cap, sizeof(double) * cap,
                               cudaMemcpyDeviceToDevice, st));
        if ((r = check_launch(ctx, "recorded segment"))) return r;
    }
    // the context as after the step loop: the new state's deposit in mesh 0,
    // the last step's stage-4 mesh as the current mesh
    if ((r = deposit_into(ctx, ctx->S[ctx->cur], ctx->S[ctx->cur].f0, ctx->mesh[0]))) return r;
    CU(cudaMemsetAsync(ctx->mesh[1], 0, sizeof(double) * nm, st));
    CU(cudaMemcpyAsync(ctx->mesh[3], a->mst + (size_t)(nsteps - 1) * G.mst_stride + 3 * nm, sizeof(double) * nm,
                       cudaMemcpyDeviceToDevice, st));
    ctx->cur_mesh = 3;
    return EMU_OK;
}

}  // namespace

void emu_ctx::adjoint_free(emu_context* ctx)
{
    if (ctx) {
        free_adj(ctx->adj);
        ctx->adj = nullptr;
    }
}

int emu_adjoint_reserve(emu_context* ctx, int nsteps, int checkpoint_interval, int64_t* device_bytes,
                        int* stage_store, int* sub_interval)
{
    if (!ctx) return EMU_ERR_ARG;
    int r;
    if ((r = check_ready(ctx, "emu_adjoint_reserve"))) return r;
    if (nsteps < 1 || checkpoint_interval < 1)
        return fail(ctx, EMU_ERR_ARG, "emu_adjoint_reserve: nsteps and checkpoint_interval must be >= 1");
    if ((r = ensure_adj(ctx, nsteps, checkpoint_interval))) return r;
    const emu_adjoint* a = ctx->adj;
    if (device_bytes) *device_bytes = (int64_t)a->bytes;
    if (stage_store) *stage_store = a->full ? 2 : a->store ? 1 : 0;
    if (sub_interval) *sub_interval = a->sub;
    return EMU_OK;
}

int emu_adjoint_forward(emu_context* ctx, int nsteps, int checkpoint_interval, double start_time, double* dts,
                        emu_run_info* info)
{
    if (!ctx) return EMU_ERR_ARG;
    int r;
    if ((r = check_ready(ctx, "emu_adjoint_forward"))) return r;
    if (nsteps < 1 || checkpoint_interval < 1)
        return fail(ctx, EMU_ERR_ARG, "emu_adjoint_forward: nsteps and checkpoint_interval must be >= 1");
    if (!ctx->prm.fused) return fail(ctx, EMU_ERR_ARG, "emu_adjoint_forward: requires fused RK4 (fused >= 1)");
    if ((r = ensure_adj(ctx, nsteps, checkpoint_interval))) return r;
    emu_adjoint* a = ctx->adj;
    a->recorded = false;
    ctx->adj_valid = false;
    a->t0 = start_time;
    std::fill(a->resorted.begin(), a->resorted.end(), 0);
    a->final_mapped = false;
    if ((r = emu_evolve_begin(ctx, start_time, INFINITY, nsteps))) return r;
    if (a->full) {
        if ((r = record_full(ctx, a, nsteps, checkpoint_interval))) return r;
    } else {
    emu::launch_ctl_hist(ctx->ctl, a->dts_dev, ctx->stream);   // the step kernels record their dt
    // cell re-sorts on the step loop's schedule; the backward recomputes each
    // segment in its start order, so a segment's re-sorts are composed into
    // one map (slot -> slot at the segment start) that the backward undoes at
    // the next boundary
    int nmap = 0, mcur = 0;
    const long long n = ctx->S[ctx->cur].n;
    for (int k = 0; k < nsteps; k++) {
        if (k % checkpoint_interval == 0) {
            const int c = k / checkpoint_interval;
            if (c > 0 && nmap > 0) {
                CU(cudaMemcpyAsync(a->perm + (size_t)c * a->cap, a->map[mcur], sizeof(unsigned) * n,
                                   cudaMemcpyDeviceToDevice, ctx->stream));
                a->resorted[c] = 1;
            }
            nmap = 0;
            const DevState& S = ctx->S[ctx->cur];
            if ((r = save_slot(ctx, a, a->ck, c, S.f0, S.pos))) return r;
        }
        if ((r = emu_ctx::step_device(ctx))) return r;
        const int ri = ctx->prm.resort_interval;
        if (ri > 0 && k + 1 < nsteps && (k + 1) % ri == 0) {
            if ((r = emu_ctx::resort_now(ctx, nullptr))) return r;
            emu::launch_compose_map(nmap ? a->map[mcur] : nullptr, ctx->idx2, a->map[1 - mcur], n, ctx->stream);
            mcur = 1 - mcur;
            nmap++;
        }
    }
    a->final_mapped = nmap > 0;
    if (nmap > 0)
        CU(cudaMemcpyAsync(a->perm + (size_t)a->nck * a->cap, a->map[mcur], sizeof(unsigned) * n,
                           cudaMemcpyDeviceToDevice, ctx->stream));
    emu::launch_ctl_hist(ctx->ctl, nullptr, ctx->stream);
    }
    ctx->steps_since_sort = 0;
    emu_run_info ri{};
    r = emu_evolve_end(ctx, &ri);
    if (info) *info = ri;
    if (r) return r;
    if (ri.steps_done != nsteps)
        return fail(ctx, EMU_ERR_STATE, "emu_adjoint_forward: the run stopped after " + std::to_string(ri.steps_done) +
                                            " steps");
    CU(cudaMemcpyAsync(a->dts.data(), a->dts_dev, sizeof(double) * nsteps, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    if (dts) std::copy(a->dts.begin(), a->dts.begin() + nsteps, dts);
    a->recorded = true;
    ctx->adj_valid = true;
    return EMU_OK;
}

int emu_adjoint_objective(emu_context* ctx, double* J, double* lam_f, double* lam_N)
{
    if (!ctx || !J) return fail(ctx, EMU_ERR_ARG, "emu_adjoint_objective: bad arguments");
    int r;
    if ((r = check_ready(ctx, "emu_adjoint_objective"))) return r;
    if ((r = ensure_adj(ctx, ctx->adj ? std::max(ctx->adj->nsteps, 1) : 1,
                        ctx->adj ? std::max(ctx->adj->interval, 1) : 1)))
        return r;
    emu_adjoint* a = ctx->adj;
    const DevState& S = ctx->S[ctx->cur];
    const long long n = S.n, cap = ctx->cap, nc = ctx->P.ncells;
    double* mesh = a->lmesh[0];
    double* lm = a->lmesh[1];
    if ((r = deposit_into(ctx, S, S.f0, mesh))) return r;
    CU(cudaMemsetAsync(lm, 0, sizeof(double) * mesh_elems(ctx), ctx->stream));
    emu::launch_adj_nex(ctx->nf, ctx->P, mesh, lm, a->nex, ctx->stream);
    double* lamf = a->lamtmp;   // scratch
    double* lamN = a->lamtmp + (size_t)ctx->NS * cap;
    emu::launch_adj_gather(ctx->nf, ctx->P, S, lm, lamf, lamN, ctx->stream);
    if ((r = check_launch(ctx, "adjoint objective"))) return r;
    std::vector<double> nex((size_t)2 * nc);
    CU(cudaMemcpyAsync(nex.data(), a->nex, sizeof(double) * 2 * nc, cudaMemcpyDeviceToHost, ctx->stream));
    const unsigned g = (unsigned)((n + emu::kBlock - 1) / emu::kBlock);
    if (lam_f) {
        emu::k_soa_to_rows<<<g, emu::kBlock, 0, ctx->stream>>>(S.id, lamf, ctx->NS, cap, n, a->rows);
        CU(cudaMemcpyAsync(lam_f, a->rows, sizeof(double) * (size_t)n * ctx->NS, cudaMemcpyDeviceToHost,
                           ctx->stream));
    }
    CU(cudaStreamSynchronize(ctx->stream));
    if (lam_N) {
        emu::k_soa_to_rows<<<g, emu::kBlock, 0, ctx->stream>>>(S.id, lamN, 2, cap, n, a->rows);
        CU(cudaMemcpyAsync(lam_N, a->rows, sizeof(double) * (size_t)n * 2, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
    }
    if ((r = check_launch(ctx, "adjoint objective output"))) return r;
    const double inv_vol = ctx->P.dxi[0] * ctx->P.dxi[1] * ctx->P.dxi[2];
    double s = 0.0;
    for (long long c = 0; c < nc; c++) s += nex[2 * c] * nex[2 * c] + nex[2 * c + 1] * nex[2 * c + 1];
    *J = s * inv_vol;
    return EMU_OK;
}

int emu_adjoint_backward(emu_context* ctx, const double* lam_f_final, const double* lam_N_final, double* lam_f0,
                         double* lam_N0)
{
    if (!ctx || !lam_f_final || !lam_f0 || !lam_N0)
        return fail(ctx, EMU_ERR_ARG, "emu_adjoint_backward: bad arguments");
    int r;
    if ((r = check_ready(ctx, "emu_adjoint_backward"))) return r;
    emu_adjoint* a = ctx->adj;
    if (!a || !a->recorded || !ctx->adj_valid)
        return fail(ctx, EMU_ERR_STATE, "emu_adjoint_backward: no recorded run for the loaded particles");
    const DevState& S = ctx->S[ctx->cur];
    const long long n = S.n, cap = ctx->cap;
    const int NS = ctx->NS, nf = ctx->nf;
    cudaStream_t st = ctx->stream;
    const unsigned g = (unsigned)((n + emu::kBlock - 1) / emu::kBlock);
    const long long nm = mesh_elems(ctx);

    // adjoint state of the final (renormalised) state, in the final slot order
    CU(cudaMemcpyAsync(a->rows, lam_f_final, sizeof(double) * (size_t)n * NS, cudaMemcpyHostToDevice, st));
    emu::k_rows_to_soa<<<g, emu::kBlock, 0, st>>>(S.id, a->rows, NS, cap, n, a->lamY0);
    CU(cudaStreamSynchronize(st));
    if (lam_N_final) {
        CU(cudaMemcpyAsync(a->rows, lam_N_final, sizeof(double) * (size_t)n * 2, cudaMemcpyHostToDevice, st));
        emu::k_rows_to_soa<<<g, emu::kBlock, 0, st>>>(S.id, a->rows, 2, cap, n, a->lamN);
    } else {
        CU(cudaMemsetAsync(a->lamN, 0, sizeof(double) * 2 * cap, st));
    }
    // working copy of the static fields, carried back through the re-sorts
    int w = 0;
    emu::k_static_scatter<<<g, emu::kBlock, 0, st>>>(S, stat_view(a, 0, S), nullptr, nullptr, nullptr, 0);
    CU(cudaMemsetAsync(a->lmesh[0], 0, sizeof(double) * nm, st));
    emu::launch_ctl_set(ctx->ctl, 0.0, 0.0, INFINITY, INT_MAX, 0, st);
    if ((r = check_launch(ctx, "adjoint input"))) return r;
    const bool coop = a->store && emu::adj_coop_fits(nf, ctx->P, n);
    // per-step mode with re-sorts (the recomputes re-sort as the forward did)
    const bool rps = !a->store && ctx->prm.resort_interval > 0 && a->gperm;

    emu::SegPtrs G{};
    G.seg_stride = (long long)(NS + 3) * cap;
    G.sst = a->sst;
    G.mst = a->mst;
    G.sst_stride = a->store ? (long long)4 * NS * cap : 0;
    G.mst_stride = a->store ? 4 * nm : 0;
    G.dts = a->dts_dev;
    G.NS = NS;
    G.acc = a->acc;
    for (int i = 0; i < 4; i++) G.lm[i] = a->lmesh[i];
    G.nmesh = nm;
    G.lamY0 = a->lamY0;
    G.lamn = a->lamn;
    G.lamYd = a->lamYd;
    G.lamN = a->lamN;

    for (int seg = a->nck - 1; seg >= 0; seg--) {
        const int k0 = seg * a->interval, k1 = std::min(k0 + a->interval, a->nsteps), len = k1 - k0;
        DevState W = stat_view(a, w, S);   // static fields in this segment's slot order
        W.fs = S.fs;
        W.acc = S.acc;
        if (a->full) {
            // the recorded forward stored every step: only the sweep
            G.seg = a->seg + (size_t)k0 * G.seg_stride;
            G.sst = a->sst + (size_t)k0 * G.sst_stride;
            G.mst = a->mst + (size_t)k0 * G.mst_stride;
            G.k0 = k0;
            G.len = len;
            cudaError_t e = emu::launch_adj_seg_coop(nf, false, ctx->P, W, G, ctx->ctl, st);
            if (e != cudaSuccess)
                return fail(ctx, EMU_ERR_CUDA, std::string("adjoint segment: ") + cudaGetErrorString(e));
            if ((r = check_launch(ctx, "adjoint segment"))) return r;
        } else if (a->store) {
            G.seg = a->seg;
            G.k0 = k0;
            G.len = len;
            CU(cudaMemcpyAsync(a->seg, slot_f(a, a->ck, seg), sizeof(double) * G.seg_stride, cudaMemcpyDeviceToDevice,
                               st));
            CU(cudaMemsetAsync(a->mst, 0, sizeof(double) * (size_t)len * 4 * nm, st));
            if ((r = segment_sweep(ctx, W, G, coop))) return r;
        } else if (rps) {
            // per-step mode with re-sorts: the recomputes re-sort where the
            // step loop did (a stable sort of the same positions gives the
            // forward's orders), each step's permutation is kept, and the
            // sweep undoes it on the static fields and the adjoint state
            // before the step; W enters in the next segment's start order
            const int ri = ctx->prm.resort_interval;
            double* const* M = ctx->mesh;
            // sub-segment starts (absolute steps; sb[nsub] = k1), see rps_layout
            std::vector<int> sb = rps_layout(len, a->rps_slots);
            if (sb.empty()) return fail(ctx, EMU_ERR_STATE, "adjoint: sub-segment layout");
            const int nsub = (int)sb.size() - 1;
            for (int& b : sb) b += k0;
            // the step state at step k of sub-segment i: its start is the
            // segment checkpoint (i = 0) or the sub-checkpoint in slot i - 1;
            // the later ones follow in slots (i = 0 ? 0 : i), ...
            auto state_slot = [&](int i, int k) -> double* {
                const int j = k - sb[i];
                if (j == 0) return i == 0 ? slot_f(a, a->ck, seg) : slot_f(a, a->seg, i - 1);
                return slot_f(a, a->seg, (i == 0 ? 0 : i) + j - 1);
            };
            double *rf = a->wf, *rf2 = a->wf2, *rp = a->wpos, *rp2 = a->wpos2;
            auto Wv = [&]() {
                DevState V = stat_view(a, w, S);
                V.fs = S.fs;
                V.acc = S.acc;
                return V;
            };
            auto Rv = [&]() {
                DevState V = Wv();
                V.f0 = rf;
                for (int d = 0; d < 3; d++) V.pos[d] = rp + (size_t)d * cap;
                V.time = a->wtime;
                return V;
            };
            // the static fields (and with lambda the adjoint state) through a
            // permutation: undo = scatter, else gather
            auto move_static = [&](const unsigned* perm, bool undo, bool with_lambda) -> int {
                const DevState src = Wv(), dst = stat_view(a, 1 - w, S);
                if (undo)
                    emu::k_static_scatter<<<g, emu::kBlock, 0, st>>>(src, dst, perm, with_lambda ? a->lamY0 : nullptr,
                                                                     a->lamtmp, NS + 2);
                else
                    emu::k_static_gather<<<g, emu::kBlock, 0, st>>>(src, dst, perm);
                if (undo && with_lambda)
                    CU(cudaMemcpyAsync(a->lamY0, a->lamtmp, sizeof(double) * (size_t)(NS + 2) * cap,
                                       cudaMemcpyDeviceToDevice, st));
                w = 1 - w;
                return EMU_OK;
            };
            // the recompute state after step k is re-sorted when the step
            // loop re-sorted there: 1 (permutation copied to gout), 0 not due
            auto resort_after = [&](int k, unsigned* gout, int& res) -> int {
                res = 0;
                if (!(k + 1 < a->nsteps && (k + 1) % ri == 0)) return EMU_OK;
                int rr;
                if ((rr = emu_ctx::sort_state_perm(ctx, Rv()))) return rr;
                emu::k_rows_gather<<<g, emu::kBlock, 0, st>>>(rf, rf2, ctx->idx2, NS, cap, n);
                emu::k_rows_gather<<<g, emu::kBlock, 0, st>>>(rp, rp2, ctx->idx2, 3, cap, n);
                std::swap(rf, rf2);
                std::swap(rp, rp2);
                if ((rr = move_static(ctx->idx2, false, false))) return rr;
                if (gout) CU(cudaMemcpyAsync(gout, ctx->idx2, sizeof(unsigned) * n, cudaMemcpyDeviceToDevice, st));
                res = 1;
                return EMU_OK;
            };
            // the recompute state from a slot, its deposit into m1 and m2
            // zeroed (stage 1 deposits there)
            auto restore = [&](const double* slot, double* m1, double* m2) -> int {
                CU(cudaMemcpyAsync(rf, slot, sizeof(double) * NS * cap, cudaMemcpyDeviceToDevice, st));
                CU(cudaMemcpyAsync(rp, slot + (size_t)NS * cap, sizeof(double) * 3 * cap, cudaMemcpyDeviceToDevice,
                                   st));
                CU(cudaMemsetAsync(m2, 0, sizeof(double) * nm, st));
                return deposit_into(ctx, Rv(), rf, m1);
            };
            // one step: stage s reads q[s-1], deposits into q[s] and zeroes
            // q[s+1] (q[4], q[5]: M_1 and M_2 of the next step)
            auto advance_q = [&](double* const q[6]) {
                const DevState R = Rv();
                for (int s = 1; s <= 4; s++)
                    emu::launch_rk4_stage(nf, ctx->P, R, s, q[s - 1], q[s], q[s + 1], nm, ctx->ctl, -1, st);
            };
            double* const Mr[6] = {M[0], M[1], M[2], M[3], M[0], M[1]};   // the context's rotating meshes
            auto advance = [&]() { advance_q(Mr); };
            // stored meshes of sub-segment step j (M_1..M_4 at q = 0..3)
            auto Mk = [&](int j, int q) -> double* { return a->smesh + ((size_t)j * 4 + q) * nm; };
            const bool mapped = seg + 1 < a->nck ? a->resorted[seg + 1] != 0 : a->final_mapped;
            if (mapped && (r = move_static(a->perm + (size_t)(seg + 1) * cap, true, false))) return r;
            // sub-checkpoints (seg slot i - 1 for sub-segment i >= 1) and the
            // composed map of every sub-segment but the last (smap slot i:
            // slot at sub-checkpoint i + 1 -> slot at sub-checkpoint i)
            std::vector<int> ncomp(nsub, 0);
            if (nsub > 1) {
                if ((r = restore(slot_f(a, a->ck, seg), M[0], M[1]))) return r;
                const int kl = sb[nsub - 1];
                int mc = 0;
                int i = 0;   // the sub-segment of step k
                for (int k = k0; k <= kl; k++) {
                    while (k >= sb[i + 1]) i++;
                    const bool save = i >= 1 && k == sb[i];
                    emu::k_seg_save<<<g, emu::kBlock, 0, st>>>(
                        Rv(), save ? slot_f(a, a->seg, i - 1) : nullptr, NS, a->dts_dev, k, ctx->ctl);
                    if (k == kl) break;
                    advance();
                    int res;
                    if ((r = resort_after(k, nullptr, res))) return r;
                    if (res) {
                        emu::launch_compose_map(ncomp[i] ? a->map[mc] : nullptr, ctx->idx2, a->map[1 - mc], n, st);
                        mc = 1 - mc;
                        ncomp[i]++;
                    }
                    if (k + 1 == sb[i + 1] && ncomp[i])
                        CU(cudaMemcpyAsync(a->smap + (size_t)i * cap, a->map[mc], sizeof(unsigned) * n,
                                           cudaMemcpyDeviceToDevice, st));
                }
                if ((r = check_launch(ctx, "adjoint sub-checkpoints"))) return r;
            }
            for (int i = nsub - 1; i >= 0; i--) {
                const int s0 = sb[i], s1 = sb[i + 1];
                if (i < nsub - 1 && ncomp[i] && (r = move_static(a->smap + (size_t)i * cap, true, false))) return r;
                const double* slot0 = state_slot(i, s0);
                const bool keep = a->smesh != nullptr;
                if ((r = keep ? restore(slot0, Mk(0, 0), Mk(0, 1)) : restore(slot0, M[0], M[1]))) return r;
                std::vector<int> has(s1 - s0, 0), meshed(s1 - s0, 0);
                for (int k = s0; k < s1; k++) {
                    const int j = k - s0;
                    // (the start state is already in its slot)
                    emu::k_seg_save<<<g, emu::kBlock, 0, st>>>(Rv(), j == 0 ? nullptr : state_slot(i, k), NS,
                                                                a->dts_dev, k, ctx->ctl);
                    const bool due = k + 1 < a->nsteps && (k + 1) % ri == 0;
                    if (k + 1 < s1 || due) {
                        // (the last step too when a re-sort follows it: its
                        // permutation maps onto the next sub-segment's order)
                        if (keep) {
                            const bool nx = k + 1 < s1;
                            double* const q[6] = {Mk(j, 0), Mk(j, 1), Mk(j, 2),
                                                  Mk(j, 3), nx ? Mk(j + 1, 0) : M[0], nx ? Mk(j + 1, 1) : M[1]};
                            advance_q(q);
                            meshed[j] = 1;
                        } else {
                            advance();
                        }
                        if ((r = resort_after(k, a->gperm + (size_t)j * cap, has[j]))) return r;
                    }
                }
                if ((r = check_launch(ctx, "adjoint segment recompute"))) return r;
                for (int k = s1 - 1; k >= s0; k--) {
                    const int j = k - s0;
                    if (has[j] && (r = move_static(a->gperm + (size_t)j * cap, true, true))) return r;
                    G.seg = state_slot(i, k);
                    G.k0 = k;
                    G.len = 1;
                    if (meshed[j]) {
                        G.mst = Mk(j, 0);
                        r = segment_sweep(ctx, Wv(), G, false, true);
                        G.mst = a->mst;
                    } else {
                        CU(cudaMemsetAsync(a->mst, 0, sizeof(double) * 4 * nm, st));
                        r = segment_sweep(ctx, Wv(), G, false);
                    }
                    if (r) return r;
                }
            }
        } else {
            // (Y_0, x) of every step of a sub-segment (the whole segment
            // unless memory asked for sub-checkpoints), recomputed from the
            // segment checkpoint or a sub-checkpoint, then each step as a
            // one-step segment (its stage states recomputed)
            DevState R = W;
            R.f0 = a->wf;
            for (int d = 0; d < 3; d++) R.pos[d] = a->wpos + (size_t)d * cap;
            R.time = a->wtime;
            double* const* M = ctx->mesh;
            const int J = (a->sub > 0 && a->sub < len) ? a->sub : len;   // steps per sub-segment
            const int nsub = (len + J - 1) / J;
            // sub-checkpoint i >= 1 (state at step k0 + i J) sits in seg slot J + i
            auto restore = [&](const double* slot) -> int {
                CU(cudaMemcpyAsync(a->wf, slot, sizeof(double) * NS * cap, cudaMemcpyDeviceToDevice, st));
                CU(cudaMemcpyAsync(a->wpos, slot + (size_t)NS * cap, sizeof(double) * 3 * cap,
                                   cudaMemcpyDeviceToDevice, st));
                CU(cudaMemsetAsync(M[1], 0, sizeof(double) * nm, st));
                return deposit_into(ctx, R, R.f0, M[0]);
            };
            auto advance = [&]() {
                for (int s = 1; s <= 4; s++)
                    emu::launch_rk4_stage(nf, ctx->P, R, s, M[s - 1], M[s % 4], M[(s + 1) % 4], nm, ctx->ctl, -1, st);
            };
            if (nsub > 1) {
                if ((r = restore(slot_f(a, a->ck, seg)))) return r;
                const int kl = k0 + (nsub - 1) * J;
                for (int k = k0; k <= kl; k++) {
                    const bool save = k > k0 && (k - k0) % J == 0;
                    emu::k_seg_save<<<g, emu::kBlock, 0, st>>>(
                        R, save ? slot_f(a, a->seg, J + (k - k0) / J) : nullptr, NS, a->dts_dev, k, ctx->ctl);
                    if (k < kl) advance();
                }
                if ((r = check_launch(ctx, "adjoint sub-checkpoints"))) return r;
            }
            for (int i = nsub - 1; i >= 0; i--) {
                const int s0 = k0 + i * J, s1 = std::min(s0 + J, k1);
                if ((r = restore(i == 0 ? slot_f(a, a->ck, seg) : slot_f(a, a->seg, J + i)))) return r;
                for (int k = s0; k < s1; k++) {
                    emu::k_seg_save<<<g, emu::kBlock, 0, st>>>(R, slot_f(a, a->seg, k - s0), NS, a->dts_dev, k,
                                                                ctx->ctl);
                    if (k + 1 == s1) break;
                    advance();
                }
                if ((r = check_launch(ctx, "adjoint segment recompute"))) return r;
                for (int k = s1 - 1; k >= s0; k--) {
                    G.seg = slot_f(a, a->seg, k - s0);
                    G.k0 = k;
                    G.len = 1;
                    CU(cudaMemsetAsync(a->mst, 0, sizeof(double) * 4 * nm, st));
                    if ((r = segment_sweep(ctx, W, G, false))) return r;
                }
            }
        }
        if (!rps && seg > 0 && a->resorted[seg]) {
            // undo the re-sorts of the previous segment (composed map)
            const unsigned* perm = a->perm + (size_t)seg * cap;
            emu::k_static_scatter<<<g, emu::kBlock, 0, st>>>(W, stat_view(a, 1 - w, S), perm, a->lamY0, a->lamtmp,
                                                             NS + 2);
            CU(cudaMemcpyAsync(a->lamY0, a->lamtmp, sizeof(double) * (size_t)(NS + 2) * cap, cudaMemcpyDeviceToDevice,
                               st));
            w = 1 - w;
        }
    }
    CU(cudaMemcpyAsync(ctx->ctl_host, ctx->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    if ((r = check_launch(ctx, "adjoint sweep"))) return r;
    if (ctx->ctl_host->status & EMU_ERR_TIMEOUT)
        return fail(ctx, EMU_ERR_TIMEOUT, "emu_adjoint_backward: a grid barrier timed out");
    // outputs in load order (the order of the run's first segment)
    const DevState W0 = stat_view(a, w, S);
    emu::k_soa_to_rows<<<g, emu::kBlock, 0, st>>>(W0.id, a->lamY0, NS, cap, n, a->rows);
    CU(cudaMemcpyAsync(lam_f0, a->rows, sizeof(double) * (size_t)n * NS, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    emu::k_soa_to_rows<<<g, emu::kBlock, 0, st>>>(W0.id, a->lamN, 2, cap, n, a->rows);
    CU(cudaMemcpyAsync(lam_N0, a->rows, sizeof(double) * (size_t)n * 2, cudaMemcpyDeviceToHost, st));
    // the forward meshes were reused: restore the current state's deposit
    double* const* M = ctx->mesh;
    CU(cudaMemsetAsync(M[1], 0, sizeof(double) * nm, st));
    if ((r = deposit_into(ctx, S, S.f0, M[0]))) return r;
    ctx->cur_mesh = 0;
    CU(cudaStreamSynchronize(st));
    return check_launch(ctx, "adjoint output");
}
