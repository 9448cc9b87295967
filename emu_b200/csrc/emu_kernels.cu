// emu_kernels.cu -- CUDA kernels (sm_100a) for Emu's per-step evolution path.
//
// Kernels, one thread per particle, particles cell-sorted so that warps share
// stencils:
//   k_rk4_stage<NF>        fused RK4 stage (FP64): interpolate the stage mesh,
//                          -i[H,rho], RK bookkeeping, deposit of the next stage
//                          state (stage 4: combine, wrap, Renormalize, deposit
//                          of the new state for the next step)
//   k_rk4_stage_mixed<NF>  the same with FP32 interpolation/SI commutator, FP64
//                          vacuum+matter commutator and state, int64 deposit
//   k_finalize_mixed<NF>   int64 mesh -> FP32 potential mesh (+ dt reduction)
//   k_dt<NF>               compute_dt reduction and device-side step control
//   k_deposit / k_rhs / k_stage_state / k_combine: unfused building blocks
//                          used by the C ABI calls and by FE/trapezoid/SSPRK3
#include "emu_kernels.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <climits>
#include <cstdio>

namespace emu {

namespace {

__device__ __constant__ double kRK4A[4] = {0.0, 0.5, 0.5, 1.0};   // a_{s,s-1}
__device__ __constant__ double kRK4B[4] = {1. / 6., 1. / 3., 1. / 3., 1. / 6.};

inline unsigned grid_for(long long n, int block = kBlock)
{
    long long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    return (unsigned)g;
}

// ---------------------------------------------------------------------------
// FP64 potential of one particle (Evolve.cpp:163-193 with the Vvac and
// interpolate fills): V starts at the vacuum term and accumulates
// coef*inside per stencil cell, nubar with the reference's sign rule.
template <int NF>
__device__ __forceinline__ void potential_fp64(const DevParams& P, const double* __restrict__ mesh,
                                               const Stencil<double>& st, double vx, double vy, double vz,
                                               double vscale, double* V)
{
    using H = Herm<NF>;
    constexpr int NH = NF * NF, ND = 8 * NH;
#pragma unroll
    for (int e = 0; e < NH; e++) {
        V[e] = P.M2[0][e] * vscale;
        V[NH + e] = P.M2[1][e] * vscale;
    }
    for (int kk = 0; kk < P.w[2]; kk++)
        for (int jj = 0; jj < P.w[1]; jj++)
            for (int ii = 0; ii < P.w[0]; ii++) {
                const long long cell = cell_of(P, st.b[0], st.b[1], st.b[2], ii, jj, kk);
                const double* __restrict__ m = mesh + cell * ND;
                const double coef = ((P.sqrt2GF_inv_vol * st.wx[ii]) * st.wy[jj]) * st.wz[kk];
#pragma unroll
                for (int e = 0; e < NH; e++) {
                    const double SI = m[e] - __ldg(m + 2 * NH + e) * vx - __ldg(m + 4 * NH + e) * vy -
                                      __ldg(m + 6 * NH + e) * vz;
                    const double Sb = __ldg(m + NH + e) - __ldg(m + 3 * NH + e) * vx -
                                      __ldg(m + 5 * NH + e) * vy - __ldg(m + 7 * NH + e) * vz;
                    double inside = H::is_im(e) ? SI + Sb : SI - Sb;
                    if (e == 0) inside = inside + P.matter;
                    const double t = coef * inside;
                    V[e] += t;
                    if (H::is_im(e)) V[NH + e] += t; else V[NH + e] -= t;
                }
            }
}

template <int NF>
__device__ __forceinline__ void load_state(const double* __restrict__ f, long long cap, long long p, double* out)
{
#pragma unroll
    for (int c = 0; c < 2 * NF * NF; c++) out[c] = f[c * cap + p];
}

template <int NF>
__device__ __forceinline__ void store_state(double* __restrict__ f, long long cap, long long p, const double* in)
{
#pragma unroll
    for (int c = 0; c < 2 * NF * NF; c++) f[c * cap + p] = in[c];
}

// deposit of a state vector (FP64 accumulation): component q = (dir*2+s)*NH+e
template <int NF>
__device__ __forceinline__ void deposit_fp64(const DevParams& P, double* mesh, bool active, const Stencil<double>& st,
                                             const double* fN, double vx, double vy, double vz)
{
    constexpr int NH = NF * NF, ND = 8 * NH;
    const int key = active ? stencil_key(P, st.b) : -1;
    warp_deposit<ND, 4, double, double>(
        P, mesh, key, st,
        [&](int q) -> double {
            const int dir = q / (2 * NH), sp = (q / NH) & 1, e = q % NH;
            const double b = fN[sp * NH + e];
            return dir == 0 ? b : b * (dir == 1 ? vx : (dir == 2 ? vy : vz));
        },
        [](double w, double v, int) -> double { return w * v; });
}

// periodic wrap of one coordinate into [0, L) (Redistribute with periodic
// boundaries).  For x in [-L, 2L) this is the single shift x -/+ L; fmod
// keeps the cost bounded for any input, and non-finite positions go to 0.
__device__ __forceinline__ double wrap_coord(double x, double L)
{
    if (x >= L || x < 0.0) {
        if (!isfinite(x)) return 0.0;
        x = fmod(x, L);
        if (x < 0.0) x += L;
        if (x >= L || x < 0.0) x = 0.0;
    }
    return x;
}

__device__ __forceinline__ void report_bad(StepCtl* ctl, int st, long long id)
{
    if (st) {
        atomicOr(&ctl->status, st);
        atomicMin(&ctl->bad, id);
    }
}

// grid-stride zeroing fused into a kernel
template <class T>
__device__ __forceinline__ void zero_slice(T* buf, long long n)
{
    if (!buf) return;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) buf[i] = (T)0;
}

// ===========================================================================
// fused FP64 RK4 stage
// ===========================================================================
template <int NF>
__global__ void __launch_bounds__(kBlock) k_rk4_stage(DevParams P, DevState S, int s, const double* __restrict__ mesh_in,
                                                      double* __restrict__ mesh_out, double* mesh_zero, long long nzero,
                                                      StepCtl* ctl)
{
    constexpr int NH = NF * NF, NS = 2 * NH;
    if (ctl->done) return;
    zero_slice(mesh_zero, nzero);
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < S.n;
    const double dt = ctl->dt;
    const long long cap = S.cap;

    Stencil<double> st;
    double fN[NS];
    double vx = 0, vy = 0, vz = 0;
    if (active) {
        const double x = S.pos[0][p], y = S.pos[1][p], z = S.pos[2][p];
        vx = S.vhat[0][p];
        vy = S.vhat[1][p];
        vz = S.vhat[2][p];
        double f[NS], V[NS], K[NS];
        load_state<NF>(s == 1 ? S.f0 : S.fs, cap, p, f);
        make_stencil<double>(P, x, y, z, st);
        potential_fp64<NF>(P, mesh_in, st, vx, vy, vz, S.vscale[p], V);
        commutator<NF, double>(V, f, K, P.inv_hbar);
        commutator<NF, double>(V + NH, f + NH, K + NH, P.inv_hbar);
        const double bw = dt * kRK4B[s - 1];
        double* fn = f;   // reuse as the next state
        if (s < 4) {
            const double aw = dt * kRK4A[s];
#pragma unroll
            for (int c = 0; c < NS; c++) {
                const double y0 = (s == 1) ? f[c] : S.f0[c * cap + p];
                const double a0 = (s == 1) ? y0 : S.acc[c * cap + p];
                S.acc[c * cap + p] = __dadd_rn(__dmul_rn(bw, K[c]), a0);
                fn[c] = __dadd_rn(__dmul_rn(aw, K[c]), y0);
                S.fs[c * cap + p] = fn[c];
            }
        } else {
#pragma unroll
            for (int c = 0; c < NS; c++) fn[c] = __dadd_rn(__dmul_rn(bw, K[c]), S.acc[c * cap + p]);
            // x, time: the integrator applies the same derivative at every
            // stage: x += (dt*b_i) * (pup/pupt*c), time += (dt*b_i) * 1
            double xn[3] = {x, y, z};
            const double kxv[3] = {vx * kC, vy * kC, vz * kC};
            double tn = S.time[p];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const double w = dt * kRK4B[i];
#pragma unroll
                for (int d = 0; d < 3; d++) xn[d] = __dadd_rn(__dmul_rn(w, kxv[d]), xn[d]);
                tn = __dadd_rn(w, tn);
            }
#pragma unroll
            for (int d = 0; d < 3; d++) {
                xn[d] = wrap_coord(xn[d], P.L[d]);
                S.pos[d][p] = xn[d];
            }
            S.time[p] = tn;
            int stt = renormalize<NF>(fn, S.Ll[0][p], P.maxError);
            stt |= renormalize<NF>(fn + NH, S.Ll[1][p], P.maxError);
            report_bad(ctl, stt, S.id[p]);
            store_state<NF>(S.f0, cap, p, fn);
            make_stencil<double>(P, xn[0], xn[1], xn[2], st);
        }
        const double N0 = S.Nn[0][p], N1 = S.Nn[1][p];
#pragma unroll
        for (int e = 0; e < NH; e++) {
            fN[e] = fn[e] * N0;
            fN[NH + e] = fn[NH + e] * N1;
        }
    }
    deposit_fp64<NF>(P, mesh_out, active, st, fN, vx, vy, vz);
}

// ===========================================================================
// unfused building blocks (FP64)
// ===========================================================================
template <int NF>
__global__ void __launch_bounds__(kBlock) k_deposit(DevParams P, DevState S, const double* __restrict__ f,
                                                    double* __restrict__ mesh)
{
    constexpr int NH = NF * NF, NS = 2 * NH;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < S.n;
    Stencil<double> st;
    double fN[NS];
    double vx = 0, vy = 0, vz = 0;
    if (active) {
        make_stencil<double>(P, S.pos[0][p], S.pos[1][p], S.pos[2][p], st);
        vx = S.vhat[0][p];
        vy = S.vhat[1][p];
        vz = S.vhat[2][p];
        const double N0 = S.Nn[0][p], N1 = S.Nn[1][p];
#pragma unroll
        for (int e = 0; e < NH; e++) {
            fN[e] = f[e * S.cap + p] * N0;
            fN[NH + e] = f[(NH + e) * S.cap + p] * N1;
        }
    }
    deposit_fp64<NF>(P, mesh, active, st, fN, vx, vy, vz);
}

template <int NF>
__global__ void __launch_bounds__(kBlock) k_rhs(DevParams P, DevState S, const double* __restrict__ f,
                                                const double* __restrict__ mesh, double* __restrict__ K)
{
    constexpr int NH = NF * NF, NS = 2 * NH;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= S.n) return;
    Stencil<double> st;
    double fl[NS], V[NS], k[NS];
    load_state<NF>(f, S.cap, p, fl);
    make_stencil<double>(P, S.pos[0][p], S.pos[1][p], S.pos[2][p], st);
    potential_fp64<NF>(P, mesh, st, S.vhat[0][p], S.vhat[1][p], S.vhat[2][p], S.vscale[p], V);
    commutator<NF, double>(V, fl, k, P.inv_hbar);
    commutator<NF, double>(V + NH, fl + NH, k + NH, P.inv_hbar);
    store_state<NF>(K, S.cap, p, k);
}

// Y = f0; for j: Y = coef_j * K_j + Y   (TimeIntegrator stage state)
template <int NF>
__global__ void __launch_bounds__(kBlock) k_stage_state(DevState S, const double* __restrict__ K, int nterms,
                                                        double c0, double c1, double c2, double* __restrict__ out)
{
    constexpr int NS = 2 * NF * NF;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= S.n) return;
    const double c[3] = {c0, c1, c2};
    const long long kstride = (long long)NS * S.cap;
#pragma unroll
    for (int q = 0; q < NS; q++) {
        double y = S.f0[q * S.cap + p];
        for (int j = 0; j < nterms; j++) y = __dadd_rn(__dmul_rn(c[j], K[j * kstride + q * S.cap + p]), y);
        out[q * S.cap + p] = y;
    }
}

// f0 = f0 + sum_i (dt*b_i) K_i ; x, time likewise ; wrap ; Renormalize
template <int NF>
__global__ void __launch_bounds__(kBlock) k_combine(DevParams P, DevState S, const double* __restrict__ K, int ns,
                                                    double w0, double w1, double w2, double w3, StepCtl* ctl)
{
    constexpr int NH = NF * NF, NS = 2 * NH;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= S.n) return;
    const double w[4] = {w0, w1, w2, w3};
    const long long kstride = (long long)NS * S.cap;
    double f[NS];
#pragma unroll
    for (int q = 0; q < NS; q++) {
        double y = S.f0[q * S.cap + p];
        for (int i = 0; i < ns; i++) y = __dadd_rn(__dmul_rn(w[i], K[i * kstride + q * S.cap + p]), y);
        f[q] = y;
    }
    const double kxv[3] = {S.vhat[0][p] * kC, S.vhat[1][p] * kC, S.vhat[2][p] * kC};
    double tn = S.time[p];
    for (int d = 0; d < 3; d++) {
        double x = S.pos[d][p];
        for (int i = 0; i < ns; i++) x = __dadd_rn(__dmul_rn(w[i], kxv[d]), x);
        S.pos[d][p] = wrap_coord(x, P.L[d]);
    }
    for (int i = 0; i < ns; i++) tn = __dadd_rn(w[i], tn);
    S.time[p] = tn;
    int stt = renormalize<NF>(f, S.Ll[0][p], P.maxError);
    stt |= renormalize<NF>(f + NH, S.Ll[1][p], P.maxError);
    report_bad(ctl, stt, S.id[p]);
    store_state<NF>(S.f0, S.cap, p, f);
}

template <int NF>
__global__ void __launch_bounds__(kBlock) k_renorm(DevParams P, DevState S, StepCtl* ctl)
{
    constexpr int NH = NF * NF, NS = 2 * NH;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= S.n) return;
    double f[NS];
    load_state<NF>(S.f0, S.cap, p, f);
    int stt = renormalize<NF>(f, S.Ll[0][p], P.maxError);
    stt |= renormalize<NF>(f + NH, S.Ll[1][p], P.maxError);
    report_bad(ctl, stt, S.id[p]);
    store_state<NF>(S.f0, S.cap, p, f);
}

// ===========================================================================
// compute_dt (Evolve.cpp:57-124) with device-side step control
// ===========================================================================
__device__ __forceinline__ void block_max2(double& a, double& b)
{
    __shared__ double sa[kBlock / 32], sb[kBlock / 32];
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        a = fmax(a, __shfl_xor_sync(kFull, a, off));
        b = fmax(b, __shfl_xor_sync(kFull, b, off));
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sa[w] = a; sb[w] = b; }
    __syncthreads();
    if (w == 0) {
        a = l < (int)(blockDim.x >> 5) ? sa[l] : 0.0;
        b = l < (int)(blockDim.x >> 5) ? sb[l] : 0.0;
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) {
            a = fmax(a, __shfl_xor_sync(kFull, a, off));
            b = fmax(b, __shfl_xor_sync(kFull, b, off));
        }
    }
}

template <int NF>
__device__ __forceinline__ double su_len2_dev(const double* h)
{
    using H = Herm<NF>;
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < NF; i++)
#pragma unroll
        for (int j = i + 1; j < NF; j++) s += h[H::im(i, j)] * h[H::im(i, j)] + h[H::re(i, j)] * h[H::re(i, j)];
#pragma unroll
    for (int l = 1; l < NF; l++) {
        const double cl = (l == 1) ? 0.5 : 0.28867513459481287;
        double t = 0.0;
#pragma unroll
        for (int i = 0; i < l; i++) t += cl * h[H::re(i, i)];
        t -= cl * l * h[H::re(l, l)];
        s += t * t;
    }
    return s;
}

// per-cell V_adaptive and V_stupid from the deposited number fields
template <int NF, class Get>
__device__ __forceinline__ void cell_potentials(const DevParams& P, Get get, double& Va, double& Vs)
{
    using H = Herm<NF>;
    constexpr int NH = NF * NF;
    double h[NH];
#pragma unroll
    for (int e = 0; e < NH; e++) h[e] = H::is_im(e) ? get(e) + get(NH + e) : get(e) - get(NH + e);
    h[0] += P.rho * P.Ye / kMp * P.cell_volume;
    double V2 = su_len2_dev<NF>(h);
#pragma unroll
    for (int d = 1; d <= 3; d++) {
#pragma unroll
        for (int e = 0; e < NH; e++) h[e] = get(2 * d * NH + e) - get((2 * d + 1) * NH + e);
        V2 += su_len2_dev<NF>(h);
    }
    Va = sqrt(V2) * M_SQRT2 * P.GF / P.cell_volume;
    double vs = 0.0;
#pragma unroll
    for (int i = 0; i < NF; i++) {
        vs = fmax(vs, get(H::re(i, i)));
        vs = fmax(vs, get(NH + H::re(i, i)));
    }
    vs = fmax(vs, P.cell_volume * P.Ye * P.rho / kMp);
    Vs = vs * (2.0 * NF * M_SQRT2 * P.GF / P.cell_volume);
}

// the last block to finish turns the reduced potentials into the next dt
__device__ void dt_finish(const DevParams& P, StepCtl* ctl, int mode)
{
    const double va = __longlong_as_double((long long)ctl->vmax_bits[0]) + P.vvac_max;
    const double vs = __longlong_as_double((long long)ctl->vmax_bits[1]) + P.vvac_max;
    double dt_flavor = 0.0;
    if (P.flavor_cfl_factor > 0.0) {
        const double dta = kHbar / va * P.flavor_cfl_factor;
        const double dts = kHbar / vs * P.flavor_cfl_factor;
        dt_flavor = dts;
        if (P.max_adaptive_speedup > 1) dt_flavor = fmin(dts * P.max_adaptive_speedup, dta);
    }
    double dt = 0.0;
    const double dtt = P.dt_translation;
    if (dtt != 0.0 && dt_flavor != 0.0) dt = fmin(dtt, dt_flavor);
    else if (dtt != 0.0) dt = dtt;
    else if (dt_flavor != 0.0) dt = dt_flavor;
    else ctl->status |= ST_DT;
    if (mode == DT_ADVANCE) {
        ctl->t = ctl->t + ctl->dt;
        ctl->step += 1;
        if (ctl->last || ctl->step >= ctl->max_step) ctl->done = 1;
    }
    if (mode != DT_QUERY) {
        // TimeIntegrator::integrate: clip the step to land on end_time
        if (ctl->end_time - ctl->t < dt) {
            dt = ctl->end_time - ctl->t;
            ctl->last = 1;
        }
        if (ctl->status & ST_DT) ctl->done = 1;
    }
    ctl->dt = dt;
    ctl->vmax_bits[0] = 0ull;
    ctl->vmax_bits[1] = 0ull;
    ctl->blocks_done = 0u;
}

template <class T>
__device__ __forceinline__ double mesh_value(const DevParams& P, const T* m, int q, int NH)
{
    return (double)m[q];
}
template <>
__device__ __forceinline__ double mesh_value<long long>(const DevParams& P, const long long* m, int q, int NH)
{
    return (double)m[q] * P.q_unscale[(q / NH) & 1];
}

template <int NF, class T>
__global__ void __launch_bounds__(kBlock) k_dt(DevParams P, const T* __restrict__ mesh, StepCtl* ctl, int mode)
{
    constexpr int NH = NF * NF, ND = 8 * NH;
    if (mode == DT_ADVANCE && ctl->done) return;
    double va = 0.0, vs = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    if (P.flavor_cfl_factor > 0.0) {
        for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < P.ncells; c += stride) {
            const T* m = mesh + c * ND;
            double a, b;
            cell_potentials<NF>(P, [&](int q) { return mesh_value<T>(P, m, q, NH); }, a, b);
            va = fmax(va, a);
            vs = fmax(vs, b);
        }
    }
    block_max2(va, vs);
    __shared__ bool is_last;
    if (threadIdx.x == 0) {
        atomicMax(&ctl->vmax_bits[0], (unsigned long long)__double_as_longlong(va));
        atomicMax(&ctl->vmax_bits[1], (unsigned long long)__double_as_longlong(vs));
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->blocks_done, 1u);
        is_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last && threadIdx.x == 0) {
        __threadfence();
        dt_finish(P, ctl, mode);
    }
}

// ===========================================================================
// mixed precision
// ===========================================================================
// finalize an int64 mesh into FP32 potentials G[cell][d][e] =
// sqrt(2)GF/dV * (M_d,nu,e + sgn_e M_d,nubar,e) and zero the other int64
// mesh (the one the next stage deposits into).
template <int NF>
__global__ void __launch_bounds__(kBlock) k_finalize_mixed(DevParams P, const long long* __restrict__ q,
                                                           long long* __restrict__ qzero, float* __restrict__ g,
                                                           StepCtl* ctl)
{
    using H = Herm<NF>;
    constexpr int NH = NF * NF, ND = 8 * NH;
    if (ctl->done) return;
    zero_slice(qzero, qzero ? P.ncells * ND : 0);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < P.ncells; c += stride) {
        const long long* m = q + c * ND;
#pragma unroll
        for (int d = 0; d < 4; d++)
#pragma unroll
            for (int e = 0; e < NH; e++) {
                const double a = (double)m[2 * d * NH + e] * P.q_unscale[0];
                const double b = (double)m[(2 * d + 1) * NH + e] * P.q_unscale[1];
                const double comb = H::is_im(e) ? a + b : a - b;
                g[c * 4 * NH + d * NH + e] = (float)(P.sqrt2GF_inv_vol * comb);
            }
    }
}

// int64 fixed-point deposit of an FP64 state (state rounded to FP32 first)
template <int NF>
__device__ __forceinline__ void deposit_q(const DevParams& P, long long* mesh, bool active, const Stencil<float>& st,
                                          const float* fN, float vx, float vy, float vz)
{
    constexpr int NH = NF * NF, ND = 8 * NH;
    const int key = active ? stencil_key(P, st.b) : -1;
    const float s0 = (float)P.q_scale[0], s1 = (float)P.q_scale[1];
    warp_deposit<ND, 4, long long, float>(
        P, mesh, key, st,
        [&](int q) -> float {
            const int dir = q / (2 * NH), sp = (q / NH) & 1, e = q % NH;
            const float b = fN[sp * NH + e];
            return dir == 0 ? b : b * (dir == 1 ? vx : (dir == 2 ? vy : vz));
        },
        [&](float w, float v, int q) -> long long {
            return __float2ll_rn((w * v) * (((q / NH) & 1) ? s1 : s0));
        });
}

template <int NF>
__global__ void __launch_bounds__(kBlock) k_deposit_q(DevParams P, DevState S, const double* __restrict__ f,
                                                      long long* __restrict__ mesh)
{
    constexpr int NH = NF * NF, NS = 2 * NH;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < S.n;
    Stencil<float> st;
    float fN[NS];
    float vx = 0, vy = 0, vz = 0;
    if (active) {
        make_stencil<float>(P, S.pos[0][p], S.pos[1][p], S.pos[2][p], st);
        vx = S.vhat32[0][p];
        vy = S.vhat32[1][p];
        vz = S.vhat32[2][p];
        const float N0 = S.N32[0][p], N1 = S.N32[1][p];
#pragma unroll
        for (int e = 0; e < NH; e++) {
            fN[e] = (float)f[e * S.cap + p] * N0;
            fN[NH + e] = (float)f[(NH + e) * S.cap + p] * N1;
        }
    }
    deposit_q<NF>(P, mesh, active, st, fN, vx, vy, vz);
}

// FP32 self-interaction potential from the finalized mesh: H_SI,e
// (nu); the nubar potential is sgn_e * H_SI,e (generate_code.py:317-355)
template <int NF>
__device__ __forceinline__ void potential_si32(const DevParams& P, const float* __restrict__ g, const Stencil<float>& st,
                                               float vx, float vy, float vz, float* hs)
{
    constexpr int NH = NF * NF;
#pragma unroll
    for (int e = 0; e < NH; e++) hs[e] = 0.f;
    for (int kk = 0; kk < P.w[2]; kk++)
        for (int jj = 0; jj < P.w[1]; jj++)
            for (int ii = 0; ii < P.w[0]; ii++) {
                const long long cell = cell_of(P, st.b[0], st.b[1], st.b[2], ii, jj, kk);
                const float* __restrict__ m = g + cell * 4 * NH;
                const float w = st.wx[ii] * st.wy[jj] * st.wz[kk];
#pragma unroll
                for (int e = 0; e < NH; e++) {
                    const float v = __ldg(m + e) - __ldg(m + NH + e) * vx - __ldg(m + 2 * NH + e) * vy -
                                    __ldg(m + 3 * NH + e) * vz;
                    hs[e] = fmaf(w, v, hs[e]);
                }
            }
}

template <int NF>
__global__ void __launch_bounds__(kBlock) k_rk4_stage_mixed(DevParams P, DevState S, int s,
                                                            const float* __restrict__ gmesh,
                                                            long long* __restrict__ qout, StepCtl* ctl)
{
    using H = Herm<NF>;
    constexpr int NH = NF * NF, NS = 2 * NH;
    if (ctl->done) return;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < S.n;
    const double dt = ctl->dt;
    const long long cap = S.cap;

    Stencil<float> st;
    float fN[NS];
    float vx = 0, vy = 0, vz = 0;
    if (active) {
        const double x = S.pos[0][p], y = S.pos[1][p], z = S.pos[2][p];
        vx = S.vhat32[0][p];
        vy = S.vhat32[1][p];
        vz = S.vhat32[2][p];
        double y0[NS], f[NS];
        load_state<NF>(S.f0, cap, p, y0);
        float kp[NS];
        if (s > 1) {
            const double aw = dt * kRK4A[s - 1];
#pragma unroll
            for (int c = 0; c < NS; c++) {
                kp[c] = S.k32[c * cap + p];
                f[c] = y0[c] + aw * (double)kp[c];
            }
        } else {
#pragma unroll
            for (int c = 0; c < NS; c++) f[c] = y0[c];
        }
        make_stencil<float>(P, x, y, z, st);
        // FP32 self-interaction part
        float hs[NH];
        potential_si32<NF>(P, gmesh, st, vx, vy, vz, hs);
        float tr = 0.f;
#pragma unroll
        for (int i = 0; i < NF; i++) tr += hs[H::re(i, i)];
        tr *= (1.0f / NF);
        float hsn[NS], f32[NS], k32v[NS];
#pragma unroll
        for (int e = 0; e < NH; e++) {
            float h = hs[e];
            if (H::is_diag(e)) h -= tr;
            hsn[e] = h;
            hsn[NH + e] = H::is_im(e) ? h : -h;
        }
#pragma unroll
        for (int c = 0; c < NS; c++) f32[c] = (float)f[c];
        const float ih = (float)P.inv_hbar;
        commutator<NF, float>(hsn, f32, k32v, ih);
        commutator<NF, float>(hsn + NH, f32 + NH, k32v + NH, ih);
        // FP64 vacuum + matter part
        double Hv[NS], Kv[NS];
        const double vs = S.vscale[p];
#pragma unroll
        for (int e = 0; e < NH; e++) {
            Hv[e] = P.M2[0][e] * vs;
            Hv[NH + e] = P.M2[1][e] * vs;
        }
        const double mat = P.sqrt2GF_inv_vol * P.matter;
        Hv[0] += mat;
        Hv[NH] -= mat;
        commutator<NF, double>(Hv, f, Kv, P.inv_hbar);
        commutator<NF, double>(Hv + NH, f + NH, Kv + NH, P.inv_hbar);
        double fn[NS];
        if (s < 4) {
            const double an = dt * kRK4A[s];
#pragma unroll
            for (int c = 0; c < NS; c++) {
                const float kc = (float)(Kv[c] + (double)k32v[c]);
                S.k32[c * cap + p] = kc;
                const float prev = (s == 1) ? 0.f : S.ksum32[c * cap + p];
                S.ksum32[c * cap + p] = (s == 1) ? kc : fmaf(2.f, kc, prev);
                fn[c] = y0[c] + an * (double)kc;
            }
        } else {
            const double w6 = dt * (1.0 / 6.0);
#pragma unroll
            for (int c = 0; c < NS; c++) {
                const double kc = Kv[c] + (double)k32v[c];
                fn[c] = y0[c] + w6 * ((double)S.ksum32[c * cap + p] + kc);
            }
            double xn[3] = {x, y, z};
            double tn = S.time[p];
            const double ipt = 1.0 / S.pup[3][p];
            const double kxv[3] = {S.pup[0][p] * ipt * kC, S.pup[1][p] * ipt * kC, S.pup[2][p] * ipt * kC};
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const double w = dt * kRK4B[i];
#pragma unroll
                for (int d = 0; d < 3; d++) xn[d] = __dadd_rn(__dmul_rn(w, kxv[d]), xn[d]);
                tn = __dadd_rn(w, tn);
            }
#pragma unroll
            for (int d = 0; d < 3; d++) {
                xn[d] = wrap_coord(xn[d], P.L[d]);
                S.pos[d][p] = xn[d];
            }
            S.time[p] = tn;
            int stt = renormalize<NF>(fn, S.Ll[0][p], P.maxError);
            stt |= renormalize<NF>(fn + NH, S.Ll[1][p], P.maxError);
            report_bad(ctl, stt, S.id[p]);
            store_state<NF>(S.f0, cap, p, fn);
            make_stencil<float>(P, xn[0], xn[1], xn[2], st);
        }
        const float N0 = S.N32[0][p], N1 = S.N32[1][p];
#pragma unroll
        for (int e = 0; e < NH; e++) {
            fN[e] = (float)fn[e] * N0;
            fN[NH + e] = (float)fn[NH + e] * N1;
        }
    }
    deposit_q<NF>(P, qout, active, st, fN, vx, vy, vz);
}

// ===========================================================================
// data movement
// ===========================================================================
// AoS records (rows of 3+nattribs) -> SoA, row perm[i] goes to slot i
template <int NF>
__global__ void k_pack(DevParams P, const double* __restrict__ aos, const unsigned* __restrict__ perm, long long n,
                       DevState S)
{
    constexpr int NH = NF * NF, NA = 8 + 2 * (2 + NH), NR = 3 + NA;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long row = perm ? (long long)perm[i] : i;
    const double* r = aos + row * NR;
    for (int d = 0; d < 3; d++) S.pos[d][i] = r[d];
    S.time[i] = r[3 + 0];
    for (int d = 0; d < 4; d++) S.pup[d][i] = r[3 + 4 + d];
    const double pupt = r[3 + 7];
    for (int d = 0; d < 3; d++) S.vhat[d][i] = r[3 + 4 + d] / pupt;
    S.vscale[i] = P.c4 / (2. * pupt);
    for (int sp = 0; sp < 2; sp++) {
        const int base = 3 + 8 + sp * (2 + NH);
        S.Nn[sp][i] = r[base];
        S.Ll[sp][i] = r[base + 1];
        for (int e = 0; e < NH; e++) S.f0[(sp * NH + e) * S.cap + i] = r[base + 2 + e];
    }
    S.id[i] = row;
}

template <int NF>
__global__ void k_unpack(DevState S, double* __restrict__ aos)
{
    constexpr int NH = NF * NF, NA = 8 + 2 * (2 + NH), NR = 3 + NA;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.n) return;
    double* r = aos + S.id[i] * NR;
    for (int d = 0; d < 3; d++) {
        r[d] = S.pos[d][i];
        r[3 + 1 + d] = S.pos[d][i];
    }
    r[3] = S.time[i];
    for (int d = 0; d < 4; d++) r[3 + 4 + d] = S.pup[d][i];
    for (int sp = 0; sp < 2; sp++) {
        const int base = 3 + 8 + sp * (2 + NH);
        r[base] = S.Nn[sp][i];
        r[base + 1] = S.Ll[sp][i];
        for (int e = 0; e < NH; e++) r[base + 2 + e] = S.f0[(sp * NH + e) * S.cap + i];
    }
}

// derivative records (interpolate_rhs_from_mesh output, Evolve.cpp:195-210)
template <int NF>
__global__ void k_unpack_rhs(DevState S, const double* __restrict__ K, double* __restrict__ aos)
{
    constexpr int NH = NF * NF, NA = 8 + 2 * (2 + NH), NR = 3 + NA;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.n) return;
    double* r = aos + S.id[i] * NR;
    for (int d = 0; d < 3; d++) r[d] = S.pos[d][i];
    for (int a = 0; a < NA; a++) r[3 + a] = 0.0;
    r[3 + 0] = 1.0;
    for (int d = 0; d < 3; d++) r[3 + 1 + d] = S.pup[d][i] / S.pup[3][i] * kC;
    for (int sp = 0; sp < 2; sp++) {
        const int base = 3 + 8 + sp * (2 + NH);
        for (int e = 0; e < NH; e++) r[base + 2 + e] = K[(sp * NH + e) * S.cap + i];
    }
}

__global__ void k_cell_keys_aos(DevParams P, const double* __restrict__ aos, int nreal, long long n,
                                unsigned* keys, unsigned* idx)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Stencil<double> st;
    make_stencil<double>(P, aos[i * nreal + 0], aos[i * nreal + 1], aos[i * nreal + 2], st);
    keys[i] = (unsigned)stencil_key(P, st.b);
    idx[i] = (unsigned)i;
}

__global__ void k_cell_keys_soa(DevParams P, DevState S, unsigned* keys, unsigned* idx)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.n) return;
    Stencil<double> st;
    make_stencil<double>(P, S.pos[0][i], S.pos[1][i], S.pos[2][i], st);
    keys[i] = (unsigned)stencil_key(P, st.b);
    idx[i] = (unsigned)i;
}

template <int NF>
__global__ void k_gather_state(DevState src, DevState dst, const unsigned* __restrict__ perm, int mixed)
{
    constexpr int NS = 2 * NF * NF;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= src.n) return;
    const long long j = perm[i];
    for (int d = 0; d < 3; d++) { dst.pos[d][i] = src.pos[d][j]; dst.vhat[d][i] = src.vhat[d][j]; }
    dst.time[i] = src.time[j];
    for (int d = 0; d < 4; d++) dst.pup[d][i] = src.pup[d][j];
    for (int sp = 0; sp < 2; sp++) { dst.Nn[sp][i] = src.Nn[sp][j]; dst.Ll[sp][i] = src.Ll[sp][j]; }
    dst.vscale[i] = src.vscale[j];
    dst.id[i] = src.id[j];
    for (int c = 0; c < NS; c++) dst.f0[c * dst.cap + i] = src.f0[c * src.cap + j];
    if (mixed) {
        for (int d = 0; d < 3; d++) dst.vhat32[d][i] = src.vhat32[d][j];
        for (int sp = 0; sp < 2; sp++) dst.N32[sp][i] = src.N32[sp][j];
    }
}

__global__ void k_mixed_shadow(DevState S)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.n) return;
    for (int d = 0; d < 3; d++) S.vhat32[d][i] = (float)S.vhat[d][i];
    for (int sp = 0; sp < 2; sp++) S.N32[sp][i] = (float)S.Nn[sp][i];
}

template <int NF>
__global__ void k_mesh_out(DevParams P, const double* __restrict__ mesh, double* __restrict__ out)
{
    constexpr int ND = 8 * NF * NF;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.ncells * ND) return;
    const long long c = i / ND;
    const int q = (int)(i % ND);
    out[(3 + q) * P.ncells + c] = mesh[i];
}

template <int NF>
__global__ void k_mesh_out_q(DevParams P, const long long* __restrict__ mesh, double* __restrict__ out)
{
    constexpr int NH = NF * NF, ND = 8 * NH;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.ncells * ND) return;
    const long long c = i / ND;
    const int q = (int)(i % ND);
    out[(3 + q) * P.ncells + c] = (double)mesh[i] * P.q_unscale[(q / NH) & 1];
}

template <int NF>
__global__ void k_q_to_f64(DevParams P, const long long* __restrict__ mesh, double* __restrict__ out)
{
    constexpr int NH = NF * NF, ND = 8 * NH;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.ncells * ND) return;
    out[i] = (double)mesh[i] * P.q_unscale[((int)(i % ND) / NH) & 1];
}

__global__ void k_ctl_set(StepCtl* ctl, double dt, double t, double end_time, int max_step, int reset_status)
{
    ctl->dt = dt;
    ctl->t = t;
    ctl->end_time = end_time;
    ctl->done = max_step <= 0 ? 1 : 0;
    ctl->step = 0;
    ctl->max_step = max_step;
    ctl->last = 0;
    ctl->blocks_done = 0u;
    ctl->vmax_bits[0] = ctl->vmax_bits[1] = 0ull;
    if (reset_status) {
        ctl->status = 0;
        ctl->bad = LLONG_MAX;
    }
}

__global__ void k_flush(double* buf, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) buf[i] = buf[i] * 0.5 + 1.0;
}

}  // namespace

// ===========================================================================
// launchers
// ===========================================================================
#define EMU_NF_DISPATCH(nf, KERNEL_CALL) \
    do {                                 \
        if ((nf) == 2) {                 \
            constexpr int NFv = 2;       \
            KERNEL_CALL;                 \
        } else {                         \
            constexpr int NFv = 3;       \
            KERNEL_CALL;                 \
        }                                \
    } while (0)

void launch_pack(int nf, const DevParams& P, const double* aos, const unsigned* perm, long long n, DevState S,
                 cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_pack<NFv><<<grid_for(n), kBlock, 0, st>>>(P, aos, perm, n, S)));
}

void launch_unpack(int nf, const DevState& S, double* aos, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_unpack<NFv><<<grid_for(S.n), kBlock, 0, st>>>(S, aos)));
}

void launch_unpack_rhs(int nf, const DevState& S, const double* K, double* aos, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_unpack_rhs<NFv><<<grid_for(S.n), kBlock, 0, st>>>(S, K, aos)));
}

void launch_cell_keys(const DevParams& P, const double* aos, int nreal, long long n, unsigned* keys, unsigned* idx,
                      cudaStream_t st)
{
    k_cell_keys_aos<<<grid_for(n), kBlock, 0, st>>>(P, aos, nreal, n, keys, idx);
}

void launch_state_keys(const DevParams& P, const DevState& S, unsigned* keys, unsigned* idx, cudaStream_t st)
{
    k_cell_keys_soa<<<grid_for(S.n), kBlock, 0, st>>>(P, S, keys, idx);
}

void launch_gather_state(int nf, bool mixed, const DevState& src, const DevState& dst, const unsigned* perm,
                         cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_gather_state<NFv><<<grid_for(src.n), kBlock, 0, st>>>(src, dst, perm, mixed ? 1 : 0)));
}

void launch_deposit(int nf, const DevParams& P, const DevState& S, const double* f, double* mesh, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_deposit<NFv><<<grid_for(S.n), kBlock, 0, st>>>(P, S, f, mesh)));
}

void launch_deposit_q(int nf, const DevParams& P, const DevState& S, const double* f, long long* mesh,
                      cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_deposit_q<NFv><<<grid_for(S.n), kBlock, 0, st>>>(P, S, f, mesh)));
}

void launch_rhs(int nf, const DevParams& P, const DevState& S, const double* f, const double* mesh, double* K,
                cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_rhs<NFv><<<grid_for(S.n), kBlock, 0, st>>>(P, S, f, mesh, K)));
}

void launch_stage_state(int nf, const DevState& S, const double* K, int nterms, const double* coef, double* out,
                        cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_stage_state<NFv><<<grid_for(S.n), kBlock, 0, st>>>(
                            S, K, nterms, coef[0], nterms > 1 ? coef[1] : 0.0, nterms > 2 ? coef[2] : 0.0, out)));
}

void launch_combine(int nf, const DevParams& P, const DevState& S, const double* K, int ns, const double* b,
                    StepCtl* ctl, cudaStream_t st)
{
    double w[4] = {0, 0, 0, 0};
    for (int i = 0; i < ns && i < 4; i++) w[i] = b[i];
    EMU_NF_DISPATCH(nf, (k_combine<NFv><<<grid_for(S.n), kBlock, 0, st>>>(P, S, K, ns, w[0], w[1], w[2], w[3], ctl)));
}

void launch_rk4_stage(int nf, const DevParams& P, const DevState& S, int s, const double* mesh_in, double* mesh_out,
                      double* mesh_zero, long long nzero, StepCtl* ctl, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_rk4_stage<NFv><<<grid_for(S.n), kBlock, 0, st>>>(P, S, s, mesh_in, mesh_out, mesh_zero,
                                                                            nzero, ctl)));
}

void launch_rk4_stage_mixed(int nf, const DevParams& P, const DevState& S, int s, const float* gmesh,
                            long long* qmesh_out, StepCtl* ctl, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_rk4_stage_mixed<NFv><<<grid_for(S.n), kBlock, 0, st>>>(P, S, s, gmesh, qmesh_out, ctl)));
}

static unsigned reduce_grid(long long ncells)
{
    long long g = (ncells + kBlock - 1) / kBlock;
    if (g > 148 * 4) g = 148 * 4;
    if (g < 1) g = 1;
    return (unsigned)g;
}

void launch_finalize_mixed(int nf, const DevParams& P, const long long* qread, long long* qzero, float* gmesh,
                           StepCtl* ctl, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_finalize_mixed<NFv><<<reduce_grid(P.ncells), kBlock, 0, st>>>(P, qread, qzero, gmesh,
                                                                                        ctl)));
}

void launch_dt(int nf, const DevParams& P, const double* mesh, StepCtl* ctl, int mode, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_dt<NFv, double><<<reduce_grid(P.ncells), kBlock, 0, st>>>(P, mesh, ctl, mode)));
}

void launch_dt_q(int nf, const DevParams& P, const long long* mesh, StepCtl* ctl, int mode, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_dt<NFv, long long><<<reduce_grid(P.ncells), kBlock, 0, st>>>(P, mesh, ctl, mode)));
}

void launch_renorm(int nf, const DevParams& P, const DevState& S, StepCtl* ctl, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_renorm<NFv><<<grid_for(S.n), kBlock, 0, st>>>(P, S, ctl)));
}

void launch_mesh_out(int nf, const DevParams& P, const double* mesh, double* out, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_mesh_out<NFv><<<grid_for(P.ncells * 8 * NFv * NFv), kBlock, 0, st>>>(P, mesh, out)));
}

void launch_mesh_out_q(int nf, const DevParams& P, const long long* mesh, double* out, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_mesh_out_q<NFv><<<grid_for(P.ncells * 8 * NFv * NFv), kBlock, 0, st>>>(P, mesh, out)));
}

void launch_q_to_f64(int nf, const DevParams& P, const long long* mesh, double* out, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_q_to_f64<NFv><<<grid_for(P.ncells * 8 * NFv * NFv), kBlock, 0, st>>>(P, mesh, out)));
}

void launch_ctl_set(StepCtl* ctl, double dt, double t, double end_time, int max_step, int reset_status,
                    cudaStream_t st)
{
    k_ctl_set<<<1, 1, 0, st>>>(ctl, dt, t, end_time, max_step, reset_status);
}

void launch_mixed_shadow(int nf, const DevState& S, cudaStream_t st)
{
    (void)nf;
    k_mixed_shadow<<<grid_for(S.n), kBlock, 0, st>>>(S);
}

void launch_flush(double* buf, long long n, cudaStream_t st)
{
    k_flush<<<148 * 8, kBlock, 0, st>>>(buf, n);
}

}  // namespace emu
