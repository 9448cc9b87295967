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
#include <string>
#include <vector>

using emu_ctx::check_launch;
using emu_ctx::fail;

struct emu_adjoint {
    long long cap = 0;
    int NS = 0;
    int nsteps = 0, interval = 0, nck = 0;
    bool recorded = false;
    double t0 = 0.0;
    std::vector<double> dts;
    double* dts_dev = nullptr;
    double* ck = nullptr;       // nck x (NS + 3) x cap: Y_0 then x, y, z
    double* seg = nullptr;      // interval x (NS + 3) x cap
    double* work = nullptr;     // stage states, adjoint state, recompute state
    double* lmesh[4] = {};      // adjoint meshes (rotating)
    double* nex = nullptr;      // ncells x 2 objective components
    long long seg_slots = 0, ck_slots = 0;
    // views into work
    double *Y[5] = {}, *Yn = nullptr, *acc = nullptr;
    double *lamY0 = nullptr, *lamn = nullptr, *lamYd = nullptr, *lamN = nullptr;
    double *wf = nullptr, *wpos = nullptr, *wtime = nullptr;
    double* rows = nullptr;     // n x NS staging for host transfers
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
template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock) k_adj_fwd_stage(DevParams P, DevState S, int s, double dt,
                                                          const double* __restrict__ Yin, const double* __restrict__ Y0,
                                                          double* __restrict__ acc, double* __restrict__ Yout,
                                                          const double* __restrict__ mesh_in,
                                                          double* __restrict__ mesh_out)
{
    using SWt = SW<WX, WY, WZ>;
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
    if (s < 4)
        tile_deposit_block<NF, SWt, double>(P, mesh_out, active, st, fN, vx, vy, vz,
                                            [](double a, int) -> double { return a; });
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
template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock) k_adj_stage(DevParams P, DevState S, int s, double dt, AdjStagePtrs A)
{
    using H = Herm<NF>;
    using SWt = SW<WX, WY, WZ>;
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
    if (a->dts_dev) cudaFree(a->dts_dev);
    if (a->ck) cudaFree(a->ck);
    if (a->seg) cudaFree(a->seg);
    if (a->work) cudaFree(a->work);
    for (int i = 0; i < 4; i++)
        if (a->lmesh[i]) cudaFree(a->lmesh[i]);
    if (a->nex) cudaFree(a->nex);
    if (a->rows) cudaFree(a->rows);
    delete a;
}

// device arrays for a recorded run of nsteps with checkpoints every interval
int ensure_adj(emu_context* ctx, int nsteps, int interval)
{
    const long long cap = ctx->cap;
    const int NS = ctx->NS;
    const int nck = (nsteps + interval - 1) / interval;
    emu_adjoint* a = ctx->adj;
    if (a && (a->cap != cap || a->NS != NS || a->ck_slots < nck || a->seg_slots < interval ||
              (int)a->dts.size() < nsteps)) {
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
        a->seg_slots = interval;
        const size_t slot = (size_t)(NS + 3) * cap;
        CU(cudaMalloc(&a->dts_dev, sizeof(double) * a->dts.size()));
        CU(cudaMalloc(&a->ck, sizeof(double) * slot * a->ck_slots));
        CU(cudaMalloc(&a->seg, sizeof(double) * slot * a->seg_slots));
        // Y2..Y4, Yn, acc, lamY0, lamn, lamYd, wf: 9 NS; lamN 2; wpos 3; wtime 1
        CU(cudaMalloc(&a->work, sizeof(double) * (size_t)(9 * NS + 6) * cap));
        for (int i = 0; i < 4; i++) CU(cudaMalloc(&a->lmesh[i], sizeof(double) * mesh_elems(ctx)));
        CU(cudaMalloc(&a->nex, sizeof(double) * 2 * ctx->P.ncells));
        CU(cudaMalloc(&a->rows, sizeof(double) * (size_t)NS * cap));
        double* w = a->work;
        for (int s = 2; s <= 4; s++) { a->Y[s] = w; w += (size_t)NS * cap; }
        a->Yn = w; w += (size_t)NS * cap;
        a->acc = w; w += (size_t)NS * cap;
        a->lamY0 = w; w += (size_t)NS * cap;
        a->lamn = w; w += (size_t)NS * cap;
        a->lamYd = w; w += (size_t)NS * cap;
        a->wf = w; w += (size_t)NS * cap;
        a->lamN = w; w += (size_t)2 * cap;
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

// copy (f, x) of a DevState-like view into a slot and back
int save_slot(emu_context* ctx, emu_adjoint* a, double* base, long long i, const double* f, double* const pos[3])
{
    const size_t fb = sizeof(double) * (size_t)a->NS * a->cap, xb = sizeof(double) * a->cap;
    CU(cudaMemcpyAsync(slot_f(a, base, i), f, fb, cudaMemcpyDeviceToDevice, ctx->stream));
    for (int d = 0; d < 3; d++)
        CU(cudaMemcpyAsync(slot_x(a, base, i, d), pos[d], xb, cudaMemcpyDeviceToDevice, ctx->stream));
    return EMU_OK;
}

int load_slot(emu_context* ctx, emu_adjoint* a, double* base, long long i, double* f, double* const pos[3])
{
    const size_t fb = sizeof(double) * (size_t)a->NS * a->cap, xb = sizeof(double) * a->cap;
    CU(cudaMemcpyAsync(f, slot_f(a, base, i), fb, cudaMemcpyDeviceToDevice, ctx->stream));
    for (int d = 0; d < 3; d++)
        CU(cudaMemcpyAsync(pos[d], slot_x(a, base, i, d), xb, cudaMemcpyDeviceToDevice, ctx->stream));
    return EMU_OK;
}

int check_ready(emu_context* ctx, const char* who)
{
    if (!ctx->loaded) return fail(ctx, EMU_ERR_STATE, std::string(who) + ": no particles loaded");
    if (ctx->mixed) return fail(ctx, EMU_ERR_ARG, std::string(who) + ": the adjoint is FP64 only");
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

}  // namespace

void emu_ctx::adjoint_free(emu_context* ctx)
{
    if (ctx) {
        free_adj(ctx->adj);
        ctx->adj = nullptr;
    }
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
    if ((r = emu_evolve_begin(ctx, start_time, INFINITY, nsteps))) return r;
    const DevState& S = ctx->S[ctx->cur];
    for (int k = 0; k < nsteps; k++) {
        if (k % checkpoint_interval == 0 &&
            (r = save_slot(ctx, a, a->ck, k / checkpoint_interval, S.f0, S.pos)))
            return r;
        CU(cudaMemcpyAsync(a->dts_dev + k, &ctx->ctl->dt, sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        if ((r = emu_ctx::step_device(ctx))) return r;
    }
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
    double* lamf = a->Yn;         // scratch
    double* lamN = a->lamN;
    emu::launch_adj_gather(ctx->nf, ctx->P, S, lm, lamf, lamN, ctx->stream);
    if ((r = check_launch(ctx, "adjoint objective"))) return r;
    std::vector<double> nex((size_t)2 * nc);
    CU(cudaMemcpyAsync(nex.data(), a->nex, sizeof(double) * 2 * nc, cudaMemcpyDeviceToHost, ctx->stream));
    const unsigned g = (unsigned)((n + emu::kBlock - 1) / emu::kBlock);
    std::vector<double> tmpN;
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

    // adjoint state of the final (renormalised) state, in slot order
    CU(cudaMemcpyAsync(a->rows, lam_f_final, sizeof(double) * (size_t)n * NS, cudaMemcpyHostToDevice, st));
    emu::k_rows_to_soa<<<g, emu::kBlock, 0, st>>>(S.id, a->rows, NS, cap, n, a->lamY0);
    CU(cudaStreamSynchronize(st));
    if (lam_N_final) {
        CU(cudaMemcpyAsync(a->rows, lam_N_final, sizeof(double) * (size_t)n * 2, cudaMemcpyHostToDevice, st));
        emu::k_rows_to_soa<<<g, emu::kBlock, 0, st>>>(S.id, a->rows, 2, cap, n, a->lamN);
    } else {
        CU(cudaMemsetAsync(a->lamN, 0, sizeof(double) * 2 * cap, st));
    }
    CU(cudaMemsetAsync(a->lmesh[0], 0, sizeof(double) * nm, st));
    if ((r = check_launch(ctx, "adjoint input"))) return r;

    // recompute view: the run's static fields with private state arrays
    DevState R = S;
    R.f0 = a->wf;
    for (int d = 0; d < 3; d++) R.pos[d] = a->wpos + (size_t)d * cap;
    R.time = a->wtime;
    double* const wpos[3] = {R.pos[0], R.pos[1], R.pos[2]};
    double* const* M = ctx->mesh;   // M_1..M_4 live in mesh[0..3]

    for (int seg = a->nck - 1; seg >= 0; seg--) {
        const int k0 = seg * a->interval, k1 = std::min(k0 + a->interval, a->nsteps);
        // forward over the segment from its checkpoint, saving (Y_0, x) per step
        if ((r = load_slot(ctx, a, a->ck, seg, a->wf, wpos))) return r;
        CU(cudaMemsetAsync(M[1], 0, sizeof(double) * nm, st));
        if ((r = deposit_into(ctx, R, R.f0, M[0]))) return r;
        for (int k = k0; k < k1; k++) {
            if ((r = save_slot(ctx, a, a->seg, k - k0, a->wf, wpos))) return r;
            if (k + 1 < k1) {
                emu::launch_ctl_set(ctx->ctl, a->dts[k], 0.0, INFINITY, INT_MAX, 0, st);
                for (int s = 1; s <= 4; s++)
                    emu::launch_rk4_stage(nf, ctx->P, R, s, M[s - 1], M[s % 4], M[(s + 1) % 4], nm, ctx->ctl, -1, st);
            }
        }
        if ((r = check_launch(ctx, "adjoint segment recompute"))) return r;
        // backward through the segment's steps
        for (int k = k1 - 1; k >= k0; k--) {
            const double dt = a->dts[k];
            DevState Q = S;   // weights from the step's start positions
            for (int d = 0; d < 3; d++) Q.pos[d] = slot_x(a, a->seg, k - k0, d);
            const double* Y0 = slot_f(a, a->seg, k - k0);
            const double* Ys[5] = {Y0, Y0, a->Y[2], a->Y[3], a->Y[4]};
            for (int i = 1; i < 4; i++) CU(cudaMemsetAsync(M[i], 0, sizeof(double) * nm, st));
            if ((r = deposit_into(ctx, Q, Y0, M[0]))) return r;
            for (int s = 1; s <= 4; s++)
                emu::launch_adj_fwd_stage(nf, ctx->P, Q, s, dt, Ys[s], Y0, a->acc, s < 4 ? a->Y[s + 1] : a->Yn,
                                          M[s - 1], s < 4 ? M[s] : nullptr, st);
            for (int s = 4; s >= 0; s--) {
                emu::AdjStagePtrs A{};
                A.Ys = s >= 1 ? Ys[s] : nullptr;
                A.Ynext = s < 4 ? Ys[s + 1] : nullptr;
                A.Yn = a->Yn;
                A.mesh_s = s >= 1 ? M[s - 1] : nullptr;
                A.lm_in = s < 4 ? a->lmesh[(s + 1) % 4] : nullptr;
                A.lm_out = s >= 1 ? a->lmesh[s % 4] : nullptr;
                A.lm_zero = s >= 1 ? a->lmesh[(s + 3) % 4] : nullptr;
                A.nmesh = nm;
                A.lamY0 = a->lamY0;
                A.lamn = a->lamn;
                A.lamYd = a->lamYd;
                A.lamN = a->lamN;
                emu::launch_adj_stage(nf, ctx->P, Q, s, dt, A, st);
            }
            if ((r = check_launch(ctx, "adjoint step"))) return r;
        }
    }
    // outputs in load order
    emu::k_soa_to_rows<<<g, emu::kBlock, 0, st>>>(S.id, a->lamY0, NS, cap, n, a->rows);
    CU(cudaMemcpyAsync(lam_f0, a->rows, sizeof(double) * (size_t)n * NS, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    emu::k_soa_to_rows<<<g, emu::kBlock, 0, st>>>(S.id, a->lamN, 2, cap, n, a->rows);
    CU(cudaMemcpyAsync(lam_N0, a->rows, sizeof(double) * (size_t)n * 2, cudaMemcpyDeviceToHost, st));
    // the forward meshes were reused: restore the current state's deposit
    CU(cudaMemsetAsync(M[1], 0, sizeof(double) * nm, st));
    if ((r = deposit_into(ctx, S, S.f0, M[0]))) return r;
    ctx->cur_mesh = 0;
    CU(cudaStreamSynchronize(st));
    return check_launch(ctx, "adjoint output");
}
