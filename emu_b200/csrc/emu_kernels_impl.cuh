// emu_kernels_impl.cuh -- CUDA kernels (sm_100a) for Emu's per-step evolution
// path (instantiated per flavor count in emu_k_fp64_<nf>.cu,
// emu_k_mixed_<nf>.cu and emu_k_misc.cu).
//
// One thread per particle (two for the species-split kernels); particles are
// cell-sorted so that a CTA's particles share stencils and their deposits are
// summed per run in registers (the tile deposit, emu_device.cuh).
//   k_rk4_stage<NF,W>        fused RK4 stage (FP64): interpolate the stage
//                            mesh, -i[H,rho], RK bookkeeping, deposit of the
//                            next stage state.  Stage 4 also combines, wraps,
//                            renormalises, deposits the new state for the
//                            next step and (device-resident loop) reduces
//                            compute_dt over the stage-4 mesh.
//   k_rk4_stage_split<2,W>   the same, 2 threads per particle (nu, nubar)
//   k_rk4_step_coop*         a whole step in one cooperative launch
//   k_gather_deposit         re-sort gather + deposit of the new state
//   k_rk4_stage_mixed<NF,W>  the same with FP32 interpolation and
//                            commutator (self-interaction + vacuum + matter),
//                            FP64 state, int64 fixed-point deposit
//   k_finalize_mixed<NF>     int64 mesh -> FP32 potential mesh
//   k_dt<NF>                 compute_dt reduction (host-driven calls)
//   k_deposit / k_rhs / k_stage_state / k_combine: unfused building blocks
//                            for the C ABI calls and FE/trapezoid/SSPRK3
// W = stencil widths (WX,WY,WZ): (1,1,3) for 1D runs along z, (3,3,3) for 3D
// TSC, (0,0,0) generic runtime widths.
#pragma once
#include "emu_kernels.cuh"

#include <cub/block/block_radix_sort.cuh>

#include <climits>
#include <cstdio>
#include <type_traits>

#include <utility>

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

#define STENCIL_LOOP(SWt, BODY)                                  \
    _Pragma("unroll") for (int kk = 0; kk < SWt::MZ; kk++)       \
        _Pragma("unroll") for (int jj = 0; jj < SWt::MY; jj++)   \
            _Pragma("unroll") for (int ii = 0; ii < SWt::MX; ii++) { \
        if (!SWt::on(P, ii, jj, kk)) continue;                   \
        BODY                                                     \
    }

// ---------------------------------------------------------------------------
// FP64 potential of one particle (Evolve.cpp:128-158 with the Vvac and
// interpolate fills): V starts at the vacuum term and accumulates
// coef*inside per stencil cell, nubar with the reference's sign rule.
template <int NF, class SWt>
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
    STENCIL_LOOP(SWt, {
        const long long cell = cell_of(P, st.b[0], st.b[1], st.b[2], ii, jj, kk);
        const double* __restrict__ m = mesh + cell * ND;
        const double coef = ((P.sqrt2GF_inv_vol * st.wx[ii]) * st.wy[jj]) * st.wz[kk];
#pragma unroll
        for (int e = 0; e < NH; e++) {
            const double SI = __ldg(m + e) - __ldg(m + 2 * NH + e) * vx - __ldg(m + 4 * NH + e) * vy -
                              __ldg(m + 6 * NH + e) * vz;
            const double Sb = __ldg(m + NH + e) - __ldg(m + 3 * NH + e) * vx - __ldg(m + 5 * NH + e) * vy -
                              __ldg(m + 7 * NH + e) * vz;
            double inside = H::is_im(e) ? SI + Sb : SI - Sb;
            if (e == 0) inside = inside + P.matter;
            const double t = coef * inside;
            V[e] += t;
            if (H::is_im(e)) V[NH + e] += t; else V[NH + e] -= t;
        }
    })
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

// the stage-4 particle push: x += sum_i dt b_i c p/p^t, t += sum_i dt b_i,
// then the periodic wrap (one definition for the mixed stage 4 and for the
// keys of the re-sort computed before it, so that both give the same bits)
__device__ __forceinline__ void rk4_push(const DevParams& P, double dt, const double* pq, double* xn, double& tn)
{
    const double ipt = 1.0 / pq[3];
    const double kxv[3] = {pq[0] * ipt * kC, pq[1] * ipt * kC, pq[2] * ipt * kC};
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const double w = dt * kRK4B[i];
#pragma unroll
        for (int d = 0; d < 3; d++) xn[d] = __dadd_rn(__dmul_rn(w, kxv[d]), xn[d]);
        tn = __dadd_rn(w, tn);
    }
#pragma unroll
    for (int d = 0; d < 3; d++) xn[d] = wrap_coord(xn[d], P.L[d]);
}

__device__ __forceinline__ void report_bad(StepCtl* ctl, int st, long long id)
{
    if (st) {
        atomicOr(&ctl->status, st);
        atomicMin(&ctl->bad, id);
    }
}

// recorded runs: the dt of the step in progress goes to dt_hist[step]
__device__ __forceinline__ void record_dt(StepCtl* ctl, double dt)
{
    if (blockIdx.x == 0 && threadIdx.x == 0 && ctl->dt_hist) ctl->dt_hist[ctl->step] = dt;
}

// grid-stride zeroing fused into a kernel
template <class T>
__device__ __forceinline__ void zero_slice(T* buf, long long n)
{
    if (!buf) return;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) buf[i] = (T)0;
}

// Programmatic dependent launch (sm_90+).  The stage kernels are launched
// with programmatic stream serialization: a stage may start while the
// previous kernel of the stream drains.  Before grid_dep_wait it only loads
// fields that no kernel of the same step writes (positions, velocities,
// weights, the state at the start of the step: written by the previous
// step's last stage or a re-sort, which completed before the previous
// kernel passed its own wait), through L2 (ld.global.cg, no stale L1 lines);
// after it, everything the previous kernel wrote is complete and visible.
// grid_dep_launch lets the next kernel start its own prologue; it comes after
// the wait, so that a prologue never overlaps a kernel two launches back.
// Without the launch attribute both are no-ops.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Bulk copies global -> shared on the TMA engine (cp.async.bulk, no
// multicast) completing on an mbarrier: a CTA stages its particles' state
// arrays (one contiguous 128-particle slice per component) while its threads
// do other work.  Addresses and sizes are multiples of 16 bytes (particle
// capacities are multiples of 128).
__device__ __forceinline__ unsigned smem_u32(const void* ptr) { return (unsigned)__cvta_generic_to_shared(ptr); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// wait for phase `parity` of the barrier, at most kMbarPolls polls (each
// try_wait may suspend the thread for a while); false when it gave up
constexpr int kMbarPolls = 1 << 22;
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity)
{
    const unsigned a = smem_u32(bar);
    for (int i = 0; i < kMbarPolls; i++) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// ===========================================================================
// compute_dt pieces (Evolve.cpp:22-89 + compute_dt fill)
// ===========================================================================
__device__ __forceinline__ void block_max2(double& a, double& b)
{
    __shared__ double sa[32], sb[32];
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

// the step in progress deposits the full stage-4 mesh (DevParams::m4_reduced)
__device__ __forceinline__ bool m4_full_step(const StepCtl* ctl)
{
    return ctl->step >= ctl->m4_full_from || ctl->last || ctl->step + 1 >= ctl->max_step;
}

// V_stupid of a cell from its diagonal slots (the operations of
// cell_potentials on the same values)
template <int NF>
__device__ __forceinline__ void cell_vstupid(const DevParams& P, const long long* d, double& Vs)
{
    double vs = 0.0;
#pragma unroll
    for (int i = 0; i < NF; i++) {
        vs = fmax(vs, (double)d[i] * P.q_unscale[0]);
        vs = fmax(vs, (double)d[NF + i] * P.q_unscale[1]);
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

// Reduce compute_dt over cells [this block's grid-stride share) and, in the
// last block to arrive, finish the step control.  Every block of the grid
// must call it exactly once (all threads).  ncb = number of blocks that take
// part in the cell reduction.
template <int NF, class T>
__device__ __forceinline__ void dt_reduce_and_finish(const DevParams& P, const T* __restrict__ mesh, StepCtl* ctl,
                                                     int mode, unsigned ncb,
                                                     const long long* __restrict__ diag = nullptr)
{
    constexpr int NH = NF * NF, ND = 8 * NH;
    double va = 0.0, vs = 0.0;
    if (P.flavor_cfl_factor > 0.0 && blockIdx.x < ncb) {
        // cell c goes to block c % ncb: every block takes a few cells
        const long long stride = (long long)ncb * blockDim.x;
        for (long long c = blockIdx.x + (long long)ncb * threadIdx.x; c < P.ncells; c += stride) {
            double a = 0.0, b;
            if (diag) {
                // V_stupid from the diagonal slots (V_adaptive is not used)
                cell_vstupid<NF>(P, diag + c * kDiagSlots, b);
            } else {
                const T* m = mesh + c * ND;
                cell_potentials<NF>(P, [&](int q) { return mesh_value<T>(P, m, q, NH); }, a, b);
            }
            va = fmax(va, a);
            vs = fmax(vs, b);
        }
    }
    // (the barrier: every thread of the block has read this step's dt)
    if (blockIdx.x < ncb) block_max2(va, vs);
    else __syncthreads();
    if (threadIdx.x == 0) {
        if (blockIdx.x < ncb) {
            atomicMax(&ctl->vmax_bits[0], (unsigned long long)__double_as_longlong(va));
            atomicMax(&ctl->vmax_bits[1], (unsigned long long)__double_as_longlong(vs));
            __threadfence();   // the maxima before the count
        }
        // the last block to count finishes, in its thread 0 alone
        if (atomicAdd(&ctl->blocks_done, 1u) == gridDim.x - 1) {
            __threadfence();
            dt_finish(P, ctl, mode);
        }
    }
}

// blocks of a stage grid that take part in the compute_dt cell reduction:
// 32 cells per block (one per thread of a warp's worth), at most 1184 blocks
// (each adds its maxima with two atomics on the same words)
__device__ __forceinline__ unsigned reduce_blocks(const DevParams& P)
{
    long long g = (P.ncells + 31) / 32;
    if (g > 1184) g = 1184;
    if (g > gridDim.x) g = gridDim.x;
    return (unsigned)(g < 1 ? 1 : g);
}

// ===========================================================================
// block-level deposit: every thread writes its particle's record to shared
// memory, then the CTA reduces the records (tile_deposit in emu_device.cuh)
// ===========================================================================
template <int NF, class SWt, class R>
__host__ __device__ constexpr int tile_smem_bytes()
{
    return kBlock * 8 + kBlock * TileRec<NF, SWt, R>::RW * (int)sizeof(R);
}

// int64 fixed-point conversion of a run total (mixed path)
struct QuantConv {
    const DevParams& P;
    __device__ long long operator()(float a, int sp) const
    {
        return __float2ll_rn(a * (float)P.q_scale[sp]);
    }
};
// (the combined self-interaction mesh: one scale for both species)
struct QuantConvG {
    const DevParams& P;
    __device__ long long operator()(float a, int) const { return __float2ll_rn(a * (float)P.g_scale); }
};
// the Comb<NF> values of a particle's f N: the NF^2 self-interaction
// combinations (nu minus nubar, nu plus nubar for imaginary components: the
// potential's sign rule), traceless for three flavors
template <int NF>
__device__ __forceinline__ void combine_species(const float* fN, float* v)
{
    constexpr int NH = NF * NF;
    float c[NH];
#pragma unroll
    for (int e = 0; e < NH; e++) c[e] = Herm<NF>::is_im(e) ? fN[e] + fN[NH + e] : fN[e] - fN[NH + e];
    Comb<NF>::values(c, v);
}

// Stable rank of the stencil keys held by the first NW warps of the block
// (key -1 = inactive, ranked last): the permutation a stable sort of the
// keys gives, by a counting sort over the distinct keys when the warps hold
// at most 32 (warp, key) groups (cell-sorted particles that moved a few
// cells: the usual case).  Group leaders list their keys, one warp sorts the
// list (bitonic, shuffles) and drops repeats, every thread finds its key's
// bucket by binary search, and one warp scans the (bucket, warp) counts.
// Every thread of the block calls it; the result is uniform over the block:
// false (nothing ranked, the caller sorts; the scratch is free again) when
// there are more groups.  scratch: 66 + 32 NW ints; on success it is read
// after the last barrier here, so the caller waits at a barrier before it
// writes there.
template <int NW>
__device__ __forceinline__ bool distinct_key_rank(int key, int* scratch, int& slot)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const bool part = w < NW;
    const unsigned lt = (1u << lane) - 1u;
    int* ngroups = scratch;                                      // (warp, key) groups listed
    int* nkeys = scratch + 1;                                    // distinct keys
    unsigned* list = reinterpret_cast<unsigned*>(scratch + 2);   // [32] group keys
    unsigned* ukey = list + 32;                                  // [32] sorted distinct keys
    int* cnt = scratch + 66;                                     // [NW][32] counts, then bases
    if (threadIdx.x == 0) *ngroups = 0;
    if (part) cnt[w * 32 + lane] = 0;
    __syncthreads();
    const unsigned k = key >= 0 ? (unsigned)key : 0xffffffffu;   // inactive last
    unsigned peers = 0u;
    if (part) {
        peers = __match_any_sync(kFull, k);
        if ((peers & lt) == 0u) {
            const int i = atomicAdd(ngroups, 1);
            if (i < 32) list[i] = k;
        }
    }
    __syncthreads();
    const int ng = *ngroups;
    if (ng > 32) {
        __syncthreads();   // every thread has read the count before the caller's sort reuses the scratch
        return false;
    }
    if (w == 0) {
        unsigned v = lane < ng ? list[lane] : 0xffffffffu;
#pragma unroll
        for (int size = 2; size <= 32; size <<= 1)
#pragma unroll
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                const unsigned o = __shfl_xor_sync(kFull, v, stride);
                const bool up = (lane & size) == 0, lower = (lane & stride) == 0;
                v = (lower == up) ? min(v, o) : max(v, o);
            }
        const unsigned prev = __shfl_up_sync(kFull, v, 1);
        const bool first = lane == 0 || prev != v;
        const unsigned fm = __ballot_sync(kFull, first);
        if (first) ukey[__popc(fm & lt)] = v;
        if (lane == 0) *nkeys = __popc(fm);
    }
    __syncthreads();
    int b = 0, rank = 0;
    if (part) {
        int lo = 0, hi = *nkeys - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (ukey[mid] < k) lo = mid + 1;
            else hi = mid;
        }
        b = lo;
        rank = __popc(peers & lt);
        if ((peers & lt) == 0u) cnt[w * 32 + b] = __popc(peers);
    }
    __syncthreads();
    if (w == 0) {
        // lane = bucket: base of each (bucket, warp) in bucket-major order
        int c[NW], tot = 0;
#pragma unroll
        for (int i = 0; i < NW; i++) {
            c[i] = cnt[i * 32 + lane];
            tot += c[i];
        }
        int inc = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(kFull, inc, o);
            if (lane >= o) inc += t;
        }
        int base = inc - tot;
#pragma unroll
        for (int i = 0; i < NW; i++) {
            cnt[i * 32 + lane] = base;
            base += c[i];
        }
    }
    __syncthreads();
    if (part) slot = cnt[w * 32 + b] + rank;
    return true;
}

// sort_keys: the CTA's particles may not be in stencil order (particles
// that moved since the last re-sort; the deposit of moved particles at the
// end of a step): the 128 keys are ranked first (stable, so cell-sorted
// particles keep their order), so that each stencil forms one run
// COMB: the mixed path's combined deposit (fN holds the Comb<NF> values;
// NREC > NV: further values the records carry for a later pass)
// given_slot >= 0 (in every thread, or in none): the record slots are given
// (a rank made earlier for the same keys) and no ranking is done.
// dg (COMB): the diagonal slots summed in the same walk (tile_deposit_comb).
// Returns the thread's slot.
template <int NF, class SWt, class R, class T, class Conv, bool COMB = false, int NREC = Comb<NF>::NV,
          class DG = NoDiag>
__device__ __forceinline__ int tile_deposit_block(const DevParams& P, T* mesh, bool active, const Stencil<R>& st,
                                                  const R* fN, R vx, R vy, R vz, Conv conv, bool sort_keys = false,
                                                  int given_slot = -1, DG dg = {})
{
    using Sort = cub::BlockRadixSort<unsigned, kBlock, 1, int>;
    static_assert(sizeof(typename Sort::TempStorage) <= kBlock * TileRec<NF, SWt, R>::RW * sizeof(R),
                  "sort scratch aliases the record area");
    static_assert((66 + kBlock) * sizeof(int) <= kBlock * TileRec<NF, SWt, R>::RW * sizeof(R),
                  "rank scratch aliases the record area");
    extern __shared__ __align__(16) unsigned char tile_smem[];
    int* skey = reinterpret_cast<int*>(tile_smem);
    int* srank = skey + kBlock;
    R* srec = reinterpret_cast<R*>(tile_smem + kBlock * 8);
    const int key = active ? stencil_key(P, st.b) : -1;
    int slot = threadIdx.x;
    if (given_slot >= 0) {
        slot = given_slot;
    } else if (sort_keys) {
        // rank the keys (scratch in the record area, not yet written), then
        // every thread writes its record at its key's rank
        if (distinct_key_rank<kBlock / 32>(key, reinterpret_cast<int*>(srec), slot)) {
            __syncthreads();   // (the record area held the ranking scratch)
        } else {
            auto& tmp = *reinterpret_cast<typename Sort::TempStorage*>(srec);
            unsigned k[1] = {key >= 0 ? (unsigned)key : (unsigned)P.ncells};   // inactive slots last
            int v[1] = {(int)threadIdx.x};
            Sort(tmp).Sort(k, v, 0, P.key_bits);
            srank[v[0]] = threadIdx.x;
            __syncthreads();
            slot = srank[threadIdx.x];
        }
    }
    if constexpr (COMB) {
        tile_record<NF, SWt, R, NREC>(srec, skey, slot, key, fN, vx, vy, vz, st);
        __syncthreads();
        tile_deposit_comb<NF, kBlock, kBlock, SWt, T>(P, mesh, skey, srec, kBlock, conv, dg);
    } else {
        tile_record<NF, SWt, R>(srec, skey, slot, key, fN, vx, vy, vz, st);
        __syncthreads();
        tile_deposit<NF, kBlock, kBlock, SWt, R, T>(P, mesh, skey, srec, kBlock, conv);
    }
    return slot;
}

// The same for a species-split CTA (kBlock particles, 2 kBlock threads:
// thread t works on species t / kBlock of particle t % kBlock).  Both threads
// of a particle write their species' f N into its record; the species-0
// thread writes the key, weights and velocity.
template <int NF, class SWt, class R, class T, class Conv>
__device__ __forceinline__ int tile_deposit_block_split(const DevParams& P, T* mesh, bool active,
                                                        const Stencil<R>& st, int sp, const R* fNs, R vx, R vy, R vz,
                                                        Conv conv, bool sort_keys, int given_slot = -1)
{
    using TR = TileRec<NF, SWt, R>;
    constexpr int NT = 2 * kBlock, NH = NF * NF, RW = TR::RW, SP = TR::SP;
    using Sort = cub::BlockRadixSort<unsigned, NT, 1, int>;
    static_assert(sizeof(typename Sort::TempStorage) <= kBlock * RW * sizeof(R), "sort scratch aliases the records");
    static_assert((66 + kBlock) * sizeof(int) <= kBlock * RW * sizeof(R), "rank scratch aliases the records");
    extern __shared__ __align__(16) unsigned char tile_smem[];
    int* skey = reinterpret_cast<int*>(tile_smem);
    int* srank = skey + kBlock;
    R* srec = reinterpret_cast<R*>(tile_smem + kBlock * 8);
    const int pl = threadIdx.x % kBlock;
    const int key = active ? stencil_key(P, st.b) : -1;
    int slot = pl;
    if (given_slot >= 0) {
        slot = given_slot;
    } else if (sort_keys) {
        int sl = pl;
        if (distinct_key_rank<kBlock / 32>(key, reinterpret_cast<int*>(srec), sl)) {
            // the species-0 threads (the first kBlock) hold the ranks
            if (sp == 0) srank[pl] = sl;
        } else {
            // species-1 threads sort behind every real key (ncells + 1)
            auto& tmp = *reinterpret_cast<typename Sort::TempStorage*>(srec);
            unsigned k[1] = {sp ? (unsigned)P.ncells + 1u : (key >= 0 ? (unsigned)key : (unsigned)P.ncells)};
            int v[1] = {(int)threadIdx.x};
            Sort(tmp).Sort(k, v, 0, P.key_bits + 1);
            if (threadIdx.x < kBlock) srank[v[0]] = threadIdx.x;
        }
        __syncthreads();
        slot = srank[pl];
    }
    R* r = srec + slot * RW;
    if (sp == 0) {
        skey[slot] = key;
#pragma unroll
        for (int kk = 0; kk < SWt::MZ; kk++)
#pragma unroll
            for (int jj = 0; jj < SWt::MY; jj++)
#pragma unroll
                for (int ii = 0; ii < SWt::MX; ii++)
                    r[(kk * SWt::MY + jj) * SWt::MX + ii] = (st.wx[ii] * st.wy[jj]) * st.wz[kk];
#pragma unroll
        for (int k = TR::S; k < SP; k++) r[k] = (R)0;
        r[SP + TR::NS + 0] = vx;
        r[SP + TR::NS + 1] = vy;
        r[SP + TR::NS + 2] = vz;
    }
#pragma unroll
    for (int e = 0; e < NH; e++) r[SP + sp * NH + e] = fNs[e];
    __syncthreads();
    tile_deposit<NF, NT, kBlock, SWt, R, T>(P, mesh, skey, srec, kBlock, conv);
    return slot;
}

// ===========================================================================
// fused FP64 RK4 stage
// ===========================================================================
template <int NF, class SWt>
__device__ __forceinline__ void rk4_stage_body(const DevParams& P, const DevState& S, int s,
                                               const double* __restrict__ mesh_in, double* __restrict__ mesh_out,
                                               double* mesh_zero, long long nzero, StepCtl* ctl, double dt,
                                               int dt_mode = -1)
{
    constexpr int NH = NF * NF, NS = 2 * NH;
    // whole-state preload where it fits the register budget (two flavors,
    // one-dimensional stencil)
    constexpr bool PRELOAD = NF == 2 && SWt::MX * SWt::MY * SWt::MZ <= 3;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < S.n;
    const long long cap = S.cap;

    // prologue: fields that no kernel of this step writes
    Stencil<double> st{};
    double fN[NS] = {};
    double vx = 0, vy = 0, vz = 0, x = 0, y = 0, z = 0, vsc = 0;
    double Nsp[2] = {0, 0}, Lsp[2] = {0, 0}, t_in = 0;
    constexpr int PRE = PRELOAD ? NS : 1;
    double fc[PRE], yv[PRE], av[PRE];
    const bool hoist = PRELOAD && s == 4;
    if (active) {
        x = __ldcg(S.pos[0] + p);
        y = __ldcg(S.pos[1] + p);
        z = __ldcg(S.pos[2] + p);
        vx = __ldcg(S.vhat[0] + p);
        vy = __ldcg(S.vhat[1] + p);
        vz = __ldcg(S.vhat[2] + p);
        vsc = __ldcg(S.vscale + p);
        Nsp[0] = __ldcg(S.Nn[0] + p);
        Nsp[1] = __ldcg(S.Nn[1] + p);
        if (hoist) {
            Lsp[0] = __ldcg(S.Ll[0] + p);
            Lsp[1] = __ldcg(S.Ll[1] + p);
            t_in = __ldcg(S.time + p);
        }
        if constexpr (PRELOAD) {
            if (s > 1) {
#pragma unroll
                for (int c = 0; c < NS; c++) yv[c] = __ldcg(S.f0 + c * cap + p);
            }
        }
        make_stencil<double>(P, x, y, z, st);
    }
    grid_dep_wait();
    grid_dep_launch();
    // stage 4 of the device-resident loop: compute_dt on the stage-4 mesh
    // (main.cpp:193-198), which this kernel only reads; every block has read
    // this step's dt before it takes part
    if (dt_mode == DT_ADVANCE) dt_reduce_and_finish<NF, double>(P, mesh_in, ctl, DT_ADVANCE, reduce_blocks(P));
    zero_slice(mesh_zero, nzero);
    if (active) {
        // the stage's remaining per-particle loads are issued together (one
        // memory round trip); the state arrays never alias
        const double* __restrict__ fin = s == 1 ? S.f0 : S.fs;
        const double* __restrict__ f0p = S.f0;
        const double* __restrict__ accp = S.acc;
        if constexpr (PRELOAD) {
#pragma unroll
            for (int c = 0; c < NS; c++) fc[c] = fin[c * cap + p];
            if (s > 1) {
#pragma unroll
                for (int c = 0; c < NS; c++) av[c] = accp[c * cap + p];
            }
        }
        double V[NS];
        potential_fp64<NF, SWt>(P, mesh_in, st, vx, vy, vz, vsc, V);
        const double bw = dt * kRK4B[s - 1];
        const double aw = s < 4 ? dt * kRK4A[s] : 0.0;
        int stt = 0;
        // one species at a time keeps the live state small
#pragma unroll
        for (int sp = 0; sp < 2; sp++) {
            double fl[NH], K[NH];
            double* f = fl;
            if constexpr (PRELOAD) f = fc + sp * NH;
            else {
#pragma unroll
                for (int e = 0; e < NH; e++) fl[e] = fin[(sp * NH + e) * cap + p];
            }
            commutator<NF, double>(V + sp * NH, f, K, P.inv_hbar);
            double* fn = f;   // reuse as the next state
            if (s < 4) {
#pragma unroll
                for (int e = 0; e < NH; e++) {
                    const long long o = (sp * NH + e) * cap + p;
                    double y0, a0;
                    if constexpr (PRELOAD) {
                        y0 = (s == 1) ? f[e] : yv[sp * NH + e];
                        a0 = (s == 1) ? y0 : av[sp * NH + e];
                    } else {
                        y0 = (s == 1) ? f[e] : f0p[o];
                        a0 = (s == 1) ? y0 : accp[o];
                    }
                    S.acc[o] = __dadd_rn(__dmul_rn(bw, K[e]), a0);
                    fn[e] = __dadd_rn(__dmul_rn(aw, K[e]), y0);
                    S.fs[o] = fn[e];
                }
            } else {
#pragma unroll
                for (int e = 0; e < NH; e++) {
                    double a0;
                    if constexpr (PRELOAD) a0 = av[sp * NH + e];
                    else a0 = accp[(sp * NH + e) * cap + p];
                    fn[e] = __dadd_rn(__dmul_rn(bw, K[e]), a0);
                }
                stt |= renormalize<NF>(fn, PRELOAD ? Lsp[sp] : S.Ll[sp][p], P.maxError);
#pragma unroll
                for (int e = 0; e < NH; e++) S.f0[(sp * NH + e) * cap + p] = fn[e];
            }
            const double Ns = Nsp[sp];
#pragma unroll
            for (int e = 0; e < NH; e++) fN[sp * NH + e] = fn[e] * Ns;
        }
        if (s == 4) {
            // x, time: the integrator applies the same derivative at every
            // stage: x += (dt*b_i) * (pup/pupt*c), time += (dt*b_i) * 1
            double xn[3] = {x, y, z};
            const double kxv[3] = {vx * kC, vy * kC, vz * kC};
            double tn = PRELOAD ? t_in : S.time[p];
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
            report_bad(ctl, stt, S.id[p]);
            make_stencil<double>(P, xn[0], xn[1], xn[2], st);
        }
    }
    if (mesh_out) {   // (null: the stage-4 deposit is made by the re-sort gather)
        // stages 1-3 deposit at the step-start positions: the rank stage 4
        // stored for them (identity after a load or re-sort)
        const int given = (s < 4 && P.rank_stages) ? (active ? S.rslot[p] : (int)threadIdx.x) : -1;
        const int sl = tile_deposit_block<NF, SWt, double>(P, mesh_out, active, st, fN, vx, vy, vz,
                                                           [](double a, int) -> double { return a; }, s == 4, given);
        if (s == 4 && active) S.rslot[p] = sl;
    }
}

// FP64 potential of one species (potential_fp64 restricted to species sp)
template <int NF, class SWt>
__device__ __forceinline__ void potential_fp64_sp(const DevParams& P, const double* __restrict__ mesh,
                                                  const Stencil<double>& st, double vx, double vy, double vz,
                                                  double vscale, int sp, double* V)
{
    using H = Herm<NF>;
    constexpr int NH = NF * NF, ND = 8 * NH;
#pragma unroll
    for (int e = 0; e < NH; e++) V[e] = P.M2[sp][e] * vscale;
    STENCIL_LOOP(SWt, {
        const long long cell = cell_of(P, st.b[0], st.b[1], st.b[2], ii, jj, kk);
        const double* __restrict__ m = mesh + cell * ND;
        const double coef = ((P.sqrt2GF_inv_vol * st.wx[ii]) * st.wy[jj]) * st.wz[kk];
        // the cell's 8 NH values (two flavors: 16-byte vector loads, every
        // group of NH = 4 starts on a 32-byte boundary)
        double c[ND];
        if constexpr (NH % 2 == 0) {
#pragma unroll
            for (int k = 0; k < ND / 2; k++) {
                const double2 v = __ldg(reinterpret_cast<const double2*>(m) + k);
                c[2 * k] = v.x;
                c[2 * k + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int k = 0; k < ND; k++) c[k] = __ldg(m + k);
        }
#pragma unroll
        for (int e = 0; e < NH; e++) {
            const double SI = c[e] - c[2 * NH + e] * vx - c[4 * NH + e] * vy - c[6 * NH + e] * vz;
            const double Sb = c[NH + e] - c[3 * NH + e] * vx - c[5 * NH + e] * vy - c[7 * NH + e] * vz;
            double inside = H::is_im(e) ? SI + Sb : SI - Sb;
            if (e == 0) inside = inside + P.matter;
            const double t = coef * inside;
            if (sp == 0 || H::is_im(e)) V[e] += t; else V[e] -= t;
        }
    })
}

// Species-split FP64 RK4 stage (1D stencils): thread t advances species
// t / kBlock of particle t % kBlock; same arithmetic as rk4_stage_body.
template <int NF, class SWt>
__device__ __forceinline__ void rk4_stage_body_split(const DevParams& P, const DevState& S, int s,
                                                     const double* __restrict__ mesh_in, double* __restrict__ mesh_out,
                                                     double* mesh_zero, long long nzero, StepCtl* ctl, double dt,
                                                     int dt_mode = -1)
{
    constexpr int NH = NF * NF;
    const int sp = threadIdx.x / kBlock;
    const long long p = (long long)blockIdx.x * kBlock + threadIdx.x % kBlock;
    const bool active = p < S.n;
    const long long cap = S.cap;
    // prologue: fields that no kernel of this step writes
    Stencil<double> st{};
    double fN[NH] = {};
    double vx = 0, vy = 0, vz = 0, x = 0, y = 0, z = 0, vsc = 0, Ns = 0, Ls = 0, t_in = 0;
    double y0[NH];
    if (active) {
        x = __ldcg(S.pos[0] + p);
        y = __ldcg(S.pos[1] + p);
        z = __ldcg(S.pos[2] + p);
        vx = __ldcg(S.vhat[0] + p);
        vy = __ldcg(S.vhat[1] + p);
        vz = __ldcg(S.vhat[2] + p);
        vsc = __ldcg(S.vscale + p);
        Ns = __ldcg(S.Nn[sp] + p);
        if (s == 4) Ls = __ldcg(S.Ll[sp] + p);
        if (s == 4 && sp == 0) t_in = __ldcg(S.time + p);
#pragma unroll
        for (int e = 0; e < NH; e++) y0[e] = s > 1 ? __ldcg(S.f0 + (sp * NH + e) * cap + p) : 0.0;
        make_stencil<double>(P, x, y, z, st);
    }
    grid_dep_wait();
    grid_dep_launch();
    if (dt_mode == DT_ADVANCE) dt_reduce_and_finish<NF, double>(P, mesh_in, ctl, DT_ADVANCE, reduce_blocks(P));
    zero_slice(mesh_zero, nzero);
    if (active) {
        const double* __restrict__ fin = s == 1 ? S.f0 : S.fs;
        double f[NH], a0[NH];
#pragma unroll
        for (int e = 0; e < NH; e++) {
            const long long o = (sp * NH + e) * cap + p;
            f[e] = fin[o];
            a0[e] = s > 1 ? S.acc[o] : 0.0;
        }
        double V[NH], K[NH];
        potential_fp64_sp<NF, SWt>(P, mesh_in, st, vx, vy, vz, vsc, sp, V);
        commutator<NF, double>(V, f, K, P.inv_hbar);
        const double bw = dt * kRK4B[s - 1];
        const double aw = s < 4 ? dt * kRK4A[s] : 0.0;
        double* fn = f;
        int stt = 0;
        if (s < 4) {
#pragma unroll
            for (int e = 0; e < NH; e++) {
                const long long o = (sp * NH + e) * cap + p;
                const double yy = (s == 1) ? f[e] : y0[e];
                const double aa = (s == 1) ? yy : a0[e];
                S.acc[o] = __dadd_rn(__dmul_rn(bw, K[e]), aa);
                fn[e] = __dadd_rn(__dmul_rn(aw, K[e]), yy);
                S.fs[o] = fn[e];
            }
        } else {
#pragma unroll
            for (int e = 0; e < NH; e++) fn[e] = __dadd_rn(__dmul_rn(bw, K[e]), a0[e]);
            stt = renormalize<NF>(fn, Ls, P.maxError);
#pragma unroll
            for (int e = 0; e < NH; e++) S.f0[(sp * NH + e) * cap + p] = fn[e];
        }
#pragma unroll
        for (int e = 0; e < NH; e++) fN[e] = fn[e] * Ns;
        if (s == 4) {
            double xn[3] = {x, y, z};
            const double kxv[3] = {vx * kC, vy * kC, vz * kC};
            double tn = t_in;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const double w = dt * kRK4B[i];
#pragma unroll
                for (int d = 0; d < 3; d++) xn[d] = __dadd_rn(__dmul_rn(w, kxv[d]), xn[d]);
                tn = __dadd_rn(w, tn);
            }
#pragma unroll
            for (int d = 0; d < 3; d++) xn[d] = wrap_coord(xn[d], P.L[d]);
            if (sp == 0) {
#pragma unroll
                for (int d = 0; d < 3; d++) S.pos[d][p] = xn[d];
                S.time[p] = tn;
            }
            report_bad(ctl, stt, S.id[p]);
            make_stencil<double>(P, xn[0], xn[1], xn[2], st);
        }
    }
    if (mesh_out) {
        // (stages 1-3: the rank the last stage 4 stored, see rk4_stage_body)
        const int given = (s < 4 && P.rank_stages) ? (active ? S.rslot[p] : (int)(threadIdx.x % kBlock)) : -1;
        const int sl = tile_deposit_block_split<NF, SWt, double>(P, mesh_out, active, st, sp, fN, vx, vy, vz,
                                                                 [](double a, int) -> double { return a; }, s == 4,
                                                                 given);
        if (s == 4 && active && sp == 0) S.rslot[p] = sl;
    }
}

// Two flavors, 1D stencils: species-split kernels (2 kBlock threads per
// CTA).  Three flavors keep one thread per particle: the split duplicates a
// 72-component mesh gather per thread and exceeds the register budget.
template <int NF, int WX, int WY>
constexpr bool kSplit = NF == 2 && WX == 1 && WY == 1;

template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(2 * kBlock, 2) k_rk4_stage_split(DevParams P, DevState S, int s,
                                                                  const double* __restrict__ mesh_in,
                                                                  double* __restrict__ mesh_out, double* mesh_zero,
                                                                  long long nzero, StepCtl* ctl, int dt_mode)
{
    // stage 1 follows the previous step's last stage (or a re-sort), which
    // writes the control block: it waits first
    if (s == 1) grid_dep_wait();
    const int done = __ldcg(&ctl->done);
    const double dt = __ldcg(&ctl->dt);
    if (done) return;
    if (s == 1) record_dt(ctl, dt);
    rk4_stage_body_split<NF, SW<WX, WY, WZ>>(P, S, s, mesh_in, mesh_out, mesh_zero, nzero, ctl, dt, dt_mode);
}

template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock, 4) k_rk4_stage(DevParams P, DevState S, int s, const double* __restrict__ mesh_in,
                                                      double* __restrict__ mesh_out, double* mesh_zero, long long nzero,
                                                      StepCtl* ctl, int dt_mode)
{
    if (s == 1) grid_dep_wait();   // (see k_rk4_stage_split)
    const int done = __ldcg(&ctl->done);
    const double dt = __ldcg(&ctl->dt);   // both control loads in one round trip
    if (done) return;
    if (s == 1) record_dt(ctl, dt);
    rk4_stage_body<NF, SW<WX, WY, WZ>>(P, S, s, mesh_in, mesh_out, mesh_zero, nzero, ctl, dt, dt_mode);
}

// Grid-wide barrier of the cooperative step kernel (its CTAs are co-resident
// by cooperative launch).  The wait is bounded: after `polls` polls (64 ns
// sleeps; DevParams::wait_polls, kBarrierSpins unless a caller set another
// limit) the CTA records ST_TIMEOUT in the step status and continues, so a
// failure can never hang the GPU.  The results of a step that timed out are
// invalid; every memory index of the step is computed from wrapped
// positions and CTA-local ranks, so they stay in bounds whatever the data.
__device__ __forceinline__ void grid_barrier(StepCtl* ctl, long long polls)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* genp = &ctl->bar_gen;
        const unsigned g = *genp;
        __threadfence();
        if (atomicAdd(&ctl->bar_count, 1u) == gridDim.x - 1) {
            ctl->bar_count = 0u;
            __threadfence();
            atomicAdd(&ctl->bar_gen, 1u);
        } else {
            long long it = 0;
            while (*genp == g) {
                if (++it > polls) {
                    atomicOr(&ctl->status, ST_TIMEOUT);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// Whole RK4 step in one cooperative launch (small problems whose grid fits
// on the GPU at once): the four stage bodies separated by grid barriers, then
// compute_dt on the stage-4 mesh.  Saves three kernel boundaries per step.
template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock, 4) k_rk4_step_coop(DevParams P, DevState S, double* m0, double* m1,
                                                            double* m2, double* m3, long long nmesh, StepCtl* ctl,
                                                            int dt_mode)
{
    using SWt = SW<WX, WY, WZ>;
    const int done = ctl->done;
    const double dt = ctl->dt;
    if (done) return;
    record_dt(ctl, dt);
    double* const m[4] = {m0, m1, m2, m3};
#pragma unroll 1
    for (int s = 1; s <= 4; s++) {
        rk4_stage_body<NF, SWt>(P, S, s, m[s - 1], m[s % 4], m[(s + 1) % 4], nmesh, ctl, dt);
        if (s < 4) grid_barrier(ctl, P.wait_polls);
    }
    if (dt_mode == DT_ADVANCE) dt_reduce_and_finish<NF, double>(P, m3, ctl, DT_ADVANCE, reduce_blocks(P));
}

template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(2 * kBlock, 2) k_rk4_step_coop_split(DevParams P, DevState S, double* m0, double* m1,
                                                                      double* m2, double* m3, long long nmesh,
                                                                      StepCtl* ctl, int dt_mode)
{
    using SWt = SW<WX, WY, WZ>;
    const int done = ctl->done;
    const double dt = ctl->dt;
    if (done) return;
    record_dt(ctl, dt);
    // one copy of the stage body (a runtime stage loop): every instruction
    // of the step runs only a few times, so code size costs fetch stalls
    double* const m[4] = {m0, m1, m2, m3};
#pragma unroll 1
    for (int s = 1; s <= 4; s++) {
        rk4_stage_body_split<NF, SWt>(P, S, s, m[s - 1], m[s % 4], m[(s + 1) % 4], nmesh, ctl, dt);
        if (s < 4) grid_barrier(ctl, P.wait_polls);
    }
    if (dt_mode == DT_ADVANCE) dt_reduce_and_finish<NF, double>(P, m3, ctl, DT_ADVANCE, reduce_blocks(P));
}

// ===========================================================================
// unfused building blocks (FP64)
// ===========================================================================
template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock) k_deposit(DevParams P, DevState S, const double* __restrict__ f,
                                                    double* __restrict__ mesh)
{
    using SWt = SW<WX, WY, WZ>;
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
        const double N0 = S.Nn[0][p], N1 = S.Nn[1][p];
#pragma unroll
        for (int e = 0; e < NH; e++) {
            fN[e] = f[e * S.cap + p] * N0;
            fN[NH + e] = f[(NH + e) * S.cap + p] * N1;
        }
    }
    tile_deposit_block<NF, SWt, double>(P, mesh, active, st, fN, vx, vy, vz,
                                        [](double a, int) -> double { return a; }, true);
}

template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock) k_rhs(DevParams P, DevState S, const double* __restrict__ f,
                                                const double* __restrict__ mesh, double* __restrict__ K)
{
    using SWt = SW<WX, WY, WZ>;
    constexpr int NH = NF * NF, NS = 2 * NH;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= S.n) return;
    Stencil<double> st;
    double fl[NS], V[NS], k[NS];
    load_state<NF>(f, S.cap, p, fl);
    make_stencil<double>(P, S.pos[0][p], S.pos[1][p], S.pos[2][p], st);
    potential_fp64<NF, SWt>(P, mesh, st, S.vhat[0][p], S.vhat[1][p], S.vhat[2][p], S.vscale[p], V);
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
    if (S.f032)
        for (int c = 0; c < NS; c++) S.f032[c * S.cap + p] = (float)f[c];
}

// compute_dt for host-driven calls and the initial dt of a run
template <int NF, class T>
__global__ void __launch_bounds__(kBlock) k_dt(DevParams P, const T* __restrict__ mesh, StepCtl* ctl, int mode,
                                               const long long* __restrict__ diag)
{
    if (mode == DT_ADVANCE && ctl->done) return;
    dt_reduce_and_finish<NF, T>(P, mesh, ctl, mode, gridDim.x, diag);
}

// ===========================================================================
// mixed precision
// ===========================================================================
// finalize an int64 mesh into FP32 potentials G[cell][d][e] =
// sqrt(2)GF/dV * (M_d,nu,e + sgn_e M_d,nubar,e) and zero the other int64
// mesh (the one the next stage deposits into).  One thread per output value
// (cell-major, coalesced): a cell per thread left a 1024-cell mesh on 8 SMs.
template <int NF>
__global__ void __launch_bounds__(kBlock) k_finalize_mixed(DevParams P, const long long* __restrict__ q,
                                                           long long* __restrict__ qzero, float* __restrict__ g,
                                                           StepCtl* ctl, int comb, long long* __restrict__ qzero_m4)
{
    using H = Herm<NF>;
    using C = Comb<NF>;
    constexpr int NH = NF * NF, ND = 8 * NH, NV = C::NV, NG = C::NG;
    grid_dep_wait();   // the previous stage's deposit is complete
    grid_dep_launch();
    if (ctl->done) return;
    zero_slice(qzero, qzero ? P.ncells * (ND + kDiagSlots) : 0);
    // (before stage 3: the full stage-4 mesh's target, on the steps that
    // deposit it)
    if (qzero_m4 && m4_full_step(ctl)) zero_slice(qzero_m4, P.ncells * ND);
    const long long stride = (long long)gridDim.x * blockDim.x;
    if (comb) {
        // a combined mesh holds the values of G itself
        const long long total = P.ncells * NG;
        const double f = P.sqrt2GF_inv_vol * P.g_unscale;
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride)
            g[i] = (float)((double)q[i] * f);
        return;
    }
    // a full mesh (8 NF^2 per cell, a scale per species): one thread per
    // (cell, d)
    const long long total = P.ncells * 4;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const long long cidx = i / 4;
        const int d = (int)(i - cidx * 4);
        const long long* m = q + cidx * ND;
        double c[NH], v[NV];
#pragma unroll
        for (int e = 0; e < NH; e++) {
            const double a = (double)m[2 * d * NH + e] * P.q_unscale[0];
            const double b = (double)m[(2 * d + 1) * NH + e] * P.q_unscale[1];
            c[e] = P.sqrt2GF_inv_vol * (H::is_im(e) ? a + b : a - b);
        }
        C::values(c, v);
#pragma unroll
        for (int j = 0; j < NV; j++) g[cidx * NG + d * NV + j] = (float)v[j];
    }
}

// full int64 mesh (8 NF^2 per cell, a scale per species) -> the combined
// layout of the step meshes (Comb<NF>: 4 NV per cell, one scale)
template <int NF>
__global__ void __launch_bounds__(kBlock) k_full_to_comb(DevParams P, const long long* __restrict__ q,
                                                         long long* __restrict__ out)
{
    using H = Herm<NF>;
    using C = Comb<NF>;
    constexpr int NH = NF * NF, ND = 8 * NH, NV = C::NV, NG = C::NG;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long total = P.ncells * 4;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const long long cidx = i / 4;
        const int d = (int)(i - cidx * 4);
        const long long* m = q + cidx * ND;
        double c[NH], v[NV];
#pragma unroll
        for (int e = 0; e < NH; e++) {
            const double a = (double)m[2 * d * NH + e] * P.q_unscale[0];
            const double b = (double)m[(2 * d + 1) * NH + e] * P.q_unscale[1];
            c[e] = H::is_im(e) ? a + b : a - b;
        }
        C::values(c, v);
#pragma unroll
        for (int j = 0; j < NV; j++) out[cidx * NG + d * NV + j] = __double2ll_rn(v[j] * P.g_scale);
    }
}

template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock) k_deposit_q(DevParams P, DevState S, const double* __restrict__ f,
                                                      long long* __restrict__ mesh)
{
    using SWt = SW<WX, WY, WZ>;
    constexpr int NH = NF * NF, NS = 2 * NH;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < S.n;
    Stencil<float> st{};
    float fN[NS] = {};
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
    tile_deposit_block<NF, SWt, float>(P, mesh, active, st, fN, vx, vy, vz, QuantConv{P}, true);
}

// FP32 self-interaction potential from the finalized mesh: H_SI,e (nu; the
// traceless part for three flavors); the nubar potential is sgn_e * H_SI,e
// (generate_code.py:317-355).  Per stencil cell the values come from 16-byte
// loads as pairs (j, j+1) of Blackwell's packed FP32 FMA:
// u = G_0 - vx G_x - vy G_y - vz G_z, then H += w u (per component the same
// FMAs, in the same order, as one component at a time).  cell4(ii, jj, kk, k)
// returns the k-th 16-byte vector of stencil cell (ii, jj, kk): from the
// mesh in global memory, or from the CTA's staged neighbourhood.
template <int NF, class SWt, class Cell4>
__device__ __forceinline__ void potential_si32_from(const DevParams& P, Cell4 cell4, const Stencil<float>& st,
                                                    float vx, float vy, float vz, float* hs)
{
    using C = Comb<NF>;
    constexpr int NV = C::NV, NG = C::NG, NP = NV / 2;
    static_assert(NV % 4 == 0, "a block of values is whole 16-byte loads");
    float2 h2[NP];
#pragma unroll
    for (int k = 0; k < NP; k++) h2[k] = f2(0.f, 0.f);
    const float2 nvx = f2(-vx, -vx), nvy = f2(-vy, -vy), nvz = f2(-vz, -vz);
    STENCIL_LOOP(SWt, {
        float2 m[NG / 2];
#pragma unroll
        for (int k = 0; k < NG / 4; k++) {
            const float4 v = cell4(ii, jj, kk, k);
            m[2 * k] = f2(v.x, v.y);
            m[2 * k + 1] = f2(v.z, v.w);
        }
        const float w = st.wx[ii] * st.wy[jj] * st.wz[kk];
        const float2 ww = f2(w, w);
#pragma unroll
        for (int k = 0; k < NP; k++) {
            float2 u = __ffma2_rn(m[NP + k], nvx, m[k]);
            u = __ffma2_rn(m[2 * NP + k], nvy, u);
            u = __ffma2_rn(m[3 * NP + k], nvz, u);
            h2[k] = __ffma2_rn(u, ww, h2[k]);
        }
    })
    float v[NV];
#pragma unroll
    for (int j = 0; j < NV; j++) v[j] = (j & 1) ? h2[j / 2].y : h2[j / 2].x;
    C::hermitian(v, hs);
}

template <int NF, class SWt>
__device__ __forceinline__ void potential_si32(const DevParams& P, const float* __restrict__ g, const Stencil<float>& st,
                                               float vx, float vy, float vz, float* hs)
{
    constexpr int NG = Comb<NF>::NG;
    potential_si32_from<NF, SWt>(
        P,
        [&](int ii, int jj, int kk, int k) {
            const long long cell = cell_of(P, st.b[0], st.b[1], st.b[2], ii, jj, kk);
            return __ldg(reinterpret_cast<const float4*>(g + cell * NG) + k);
        },
        st, vx, vy, vz, hs);
}

// The neighbourhood of a CTA's particles for 27-cell stencils: the box of
// cells their stencils touch, staged in shared memory by bulk copies (the TMA
// engine, no multicast) of the potential mesh's rows when it holds at most
// kMeshTileCells cells.  Built from the smallest and largest stencil key of
// the CTA: every key between them lies in one z plane and in one or two
// consecutive y rows, so the box is x from the smallest key's x to the
// largest's (+ nx when the rows differ), y over one or two rows, z one
// plane, each grown by the stencil's two further cells.  Otherwise (keys
// spread wider, a mesh smaller than a box) the interpolation reads the mesh
// in global memory.
constexpr int kMeshTileCells = 80;

struct MeshBox {
    int x0, y0, z0;   // first cell of the box (wrapped)
    int nx, ny, nz;   // its extent; nx = 0: not staged
};

__device__ __forceinline__ MeshBox mesh_box(const DevParams& P, unsigned kmin, unsigned kmax)
{
    MeshBox b{0, 0, 0, 0, 0, 0};
    if (kmin > kmax) return b;   // no particle
    const int n0 = P.n[0], n1 = P.n[1];
    const int xa = (int)(kmin % n0), ya = (int)((kmin / n0) % n1), za = (int)(kmin / (n0 * n1));
    const int xb = (int)(kmax % n0), yb = (int)((kmax / n0) % n1), zb = (int)(kmax / (n0 * n1));
    if (za != zb || (yb != ya && yb != ya + 1)) return b;
    const int lx = (yb == ya ? xb - xa : xb + n0 - xa) + 3;
    const int ly = yb - ya + 3;
    if (lx > n0 || ly > n1 || 3 > P.n[2] || lx * ly * 3 > kMeshTileCells) return b;
    b.x0 = xa; b.y0 = ya; b.z0 = za;
    b.nx = lx; b.ny = ly; b.nz = 3;
    return b;
}

// dynamic shared memory of a mixed stage: the deposit tile, or the staged
// state slices (f0 FP64, k32 and ksum32 FP32) when those are larger
template <int NF, int WX, int WY, int WZ>
__host__ __device__ constexpr bool mixed_mesh_tile()
{
    return WX == 3 && WY == 3 && WZ == 3;
}

template <int NF, int WX, int WY, int WZ>
__host__ __device__ constexpr int mixed_stage_smem_bytes()
{
    constexpr int tile = tile_smem_bytes<NF, SW<WX, WY, WZ>, float>();
    using SWt = SW<WX, WY, WZ>;
    constexpr bool preload = NF == 2 && SWt::MX * SWt::MY * SWt::MZ <= 3;
    constexpr int staged = preload ? 0 : 2 * NF * NF * kBlock * 16 + 7 * kBlock * 8;
    constexpr int area = tile > staged ? tile : staged;
    // (after the area: the staged mesh neighbourhood of 27-cell stencils)
    return area + (mixed_mesh_tile<NF, WX, WY, WZ>() ? kMeshTileCells * Comb<NF>::NG * 4 : 0);
}
template <int NF, int WX, int WY, int WZ>
__host__ __device__ constexpr int mixed_mesh_tile_offset()
{
    return mixed_stage_smem_bytes<NF, WX, WY, WZ>() -
           (mixed_mesh_tile<NF, WX, WY, WZ>() ? kMeshTileCells * Comb<NF>::NG * 4 : 0);
}

// Key of the cell re-sort that the next stage 4 scatters into, stored by
// stage 3 of a step followed by a re-sort: particle p's stencil key after
// the step (the stage-4 push of its momentum with the step's dt; the key of
// the unchanged position once the run has ended), with the identity index,
// for the radix sort.
__device__ __forceinline__ void sc_key(const DevParams& P, const DevState& S, long long p, double dt, bool push,
                                       unsigned* keys, unsigned* idx)
{
    double xn[3] = {__ldcg(S.pos[0] + p), __ldcg(S.pos[1] + p), __ldcg(S.pos[2] + p)};
    if (push) {
        const double pq[4] = {__ldcg(S.pup[0] + p), __ldcg(S.pup[1] + p), __ldcg(S.pup[2] + p), __ldcg(S.pup[3] + p)};
        double tn = 0.0;
        rk4_push(P, dt, pq, xn, tn);
    }
    Stencil<double> st;
    make_stencil<double>(P, xn[0], xn[1], xn[2], st);
    keys[p] = (unsigned)stencil_key(P, st.b);
    idx[p] = (unsigned)p;
}

// the same keys before the sort, when stage 3 does not store them
__global__ void k_sc_keys(DevParams P, DevState S, const StepCtl* __restrict__ ctl, unsigned* __restrict__ keys,
                          unsigned* __restrict__ idx)
{
    const int done = __ldcg(&ctl->done);
    const double dt = __ldcg(&ctl->dt);
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < S.n) sc_key(P, S, p, dt, !done, keys, idx);
}

// inverse of the sort's permutation: particle perm[i] goes to slot i
__global__ void k_sc_invert(const unsigned* __restrict__ perm, unsigned* __restrict__ inv, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) inv[perm[i]] = (unsigned)i;
}

// the fields of particle p that no stage changes, into slot q of D
__device__ __forceinline__ void sc_static_fields(const DevParams& P, const DevState& S, const DevState& D, long long p,
                                                 long long q, const double* pq, const double* L2)
{
    D.rslot[q] = (int)(q % kBlock);   // in cell order: the identity rank
    D.id[q] = S.id[p];
#pragma unroll
    for (int sp = 0; sp < 2; sp++) {
        const double nn = S.Nn[sp][p];
        D.Nn[sp][q] = nn;
        D.N32[sp][q] = (float)nn;
        D.Ll[sp][q] = L2[sp];
    }
#pragma unroll
    for (int d = 0; d < 4; d++) D.pup[d][q] = pq[d];
    D.vscale[q] = P.c4 / (2. * pq[3]);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double v = pq[d] / pq[3];
        D.vhat[d][q] = v;
        D.vhat32[d][q] = (float)v;
    }
}

// One kernel per RK stage SG (1-4): each holds only its stage's paths.
// SC (stage 4 before a re-sort): the new state and every unchanged field of
// particle p go to slot inv[p] of D, the other particle buffer, in the new
// cell order (the re-sort's gather, made by the stores of this stage; its
// keys, stored by stage 3 into kout/iout, and their sort ran before it,
// from the same push); D's deposit follows.
template <int NF, int WX, int WY, int WZ, int SG, bool SC = false>
// (1D: 5 CTAs per SM at 96 registers beat 4 at 128 despite the spills)
__global__ void __launch_bounds__(kBlock, WX == 1 ? 5 : 4) k_rk4_stage_mixed(DevParams P, DevState S,
                                                            const float* __restrict__ gmesh,
                                                            long long* __restrict__ qout,
                                                            const long long* __restrict__ qdt,
                                                            long long* __restrict__ qm4, StepCtl* ctl,
                                                            int dt_mode, DevState D,
                                                            const unsigned* __restrict__ inv,
                                                            unsigned* __restrict__ kout,
                                                            unsigned* __restrict__ iout)
{
    using H = Herm<NF>;
    using SWt = SW<WX, WY, WZ>;
    constexpr int NH = NF * NF, NS = 2 * NH;
    constexpr int s = SG;
    constexpr bool PRELOAD = NF == 2 && SWt::MX * SWt::MY * SWt::MZ <= 3;
    // stages 1-3 read the FP32 copy of the step-start state (mixed_f0_copy)
    constexpr bool F32C = mixed_f0_copy_w<WX, WY, WZ>() && s < 4;
    // without the register preload, the CTA's slices of f0, k32 and ksum32
    // are staged in shared memory by bulk copies (the record area of the
    // deposit, written only after the state is consumed)
    constexpr bool STAGE = !PRELOAD;
    // (programmatic dependent launch: see grid_dep_wait; the finalize
    // kernel before this stage has waited for the previous stage)
    static_assert(!SC || SG == 4, "the re-sort scatter is stage 4's");
    const int done = __ldcg(&ctl->done);
    const double dt = __ldcg(&ctl->dt);   // both control loads in one round trip
    if (done) {
        if constexpr (SG == 3 && sc_keys_in_stage3_w<WX, WY, WZ>()) {
            const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
            if (kout && p < S.n) sc_key(P, S, p, dt, false, kout, iout);
        }
        if constexpr (SC) {
            // after the run's end the re-sort still moves the unchanged
            // state (its keys were those of the unchanged positions)
            grid_dep_wait();
            const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
            if (p < S.n) {
                const long long q = inv[p];
                double pq[4], L2[2];
                for (int d = 0; d < 4; d++) pq[d] = S.pup[d][p];
                for (int sp = 0; sp < 2; sp++) L2[sp] = S.Ll[sp][p];
                sc_static_fields(P, S, D, p, q, pq, L2);
                for (int d = 0; d < 3; d++) D.pos[d][q] = S.pos[d][p];
                D.time[q] = S.time[p];
                for (int c = 0; c < 2 * NF * NF; c++) {
                    D.f0[c * D.cap + q] = S.f0[c * S.cap + p];
                    if (D.f032) D.f032[c * D.cap + q] = S.f032[c * S.cap + p];
                }
            }
        }
        return;
    }
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < S.n;
    const long long cap = S.cap;
    const int t = threadIdx.x;
    extern __shared__ __align__(16) unsigned char tile_smem[];
    __shared__ __align__(8) unsigned long long stage_bar;
    // 27-cell stencils: the staged mesh neighbourhood (see mesh_box)
    constexpr bool MTILE = STAGE && mixed_mesh_tile<NF, WX, WY, WZ>();
    constexpr int NGC = Comb<NF>::NG;
    __shared__ __align__(8) unsigned long long mesh_bar;
    __shared__ unsigned key_ext[2][kBlock / 32];
    __shared__ MeshBox mbox;
    float* const mtile = reinterpret_cast<float*>(tile_smem + mixed_mesh_tile_offset<NF, WX, WY, WZ>());
    double* const sf0 = reinterpret_cast<double*>(tile_smem);        // [NS][kBlock]
    float* const sf32 = reinterpret_cast<float*>(tile_smem);         // [NS][kBlock] (F32C)
    float* const sk = reinterpret_cast<float*>(sf0 + NS * kBlock);   // [NS][kBlock]
    float* const sks = sk + NS * kBlock;                             // [NS][kBlock]
    double* const s4 = reinterpret_cast<double*>(sks + NS * kBlock); // stage 4: time, pup[4], L[2] x kBlock
    const long long p0 = (long long)blockIdx.x * kBlock;
    // slices of k32 and ksum32 staged: none in stage 1; K_1 alone in stage
    // 2 (after stage 1 the running sum K_1 + 2 K_2 + ... is K_1 itself, so
    // stage 1 stores no ksum32); both in stages 3 and 4
    constexpr int NKS = s == 1 ? 0 : (s == 2 ? NS : 2 * NS);
    if constexpr (STAGE) {
        // f0 is written only by the previous step: its copies start before
        // the dependency wait, k32 and ksum32 (the previous stage's) after it
        if (t < 32) {
            if (t == 0) {
                mbar_init(&stage_bar, 1);
                mbar_expect_tx(&stage_bar, NS * kBlock * (F32C ? 4 : 8) + NKS * kBlock * 4 + (s == 4 ? 7 * kBlock * 8 : 0));
                if constexpr (MTILE) mbar_init(&mesh_bar, 1);
            }
            __syncwarp();
            // (F32C: the FP32 copy, in the first half of the FP64 slices' area)
            for (int c = t; c < NS; c += 32) {
                if (F32C) bulk_g2s(sf32 + c * kBlock, S.f032 + c * cap + p0, kBlock * 4, &stage_bar);
                else bulk_g2s(sf0 + c * kBlock, S.f0 + c * cap + p0, kBlock * 8, &stage_bar);
            }
            // stage 4's time, momentum and SU(n) lengths (written only by
            // the previous step too)
            if (s == 4 && t < 7) {
                const double* src = t == 0 ? S.time : t < 5 ? S.pup[t - 1] : S.Ll[t - 5];
                bulk_g2s(s4 + t * kBlock, src + p0, kBlock * 8, &stage_bar);
            }
        }
        __syncthreads();   // the barrier is initialised before anyone waits on it
    }

    // prologue: fields that no kernel of this step writes (one memory round
    // trip with the control loads; all of the state at the step start for
    // two flavors in 1D, the per-species scalars otherwise)
    Stencil<float> st{};
    float fN[NS] = {};
    float vx = 0, vy = 0, vz = 0;
    double x = 0, y = 0, z = 0, vs = 0, t_in = 0;
    float Nsp[2] = {0.f, 0.f};
    double Lsp[2] = {0, 0}, pu[4] = {0, 0, 0, 1};
    const bool hoist = PRELOAD && s == 4;
    constexpr int PRE = PRELOAD ? NS : 1;
    double y0a[PRE];
    float ka[PRE], ksa[PRE];
    if (active) {
        x = __ldcg(S.pos[0] + p);
        y = __ldcg(S.pos[1] + p);
        z = __ldcg(S.pos[2] + p);
        vx = __ldcg(S.vhat32[0] + p);
        vy = __ldcg(S.vhat32[1] + p);
        vz = __ldcg(S.vhat32[2] + p);
        vs = __ldcg(S.vscale + p);
        Nsp[0] = __ldcg(S.N32[0] + p);
        Nsp[1] = __ldcg(S.N32[1] + p);
        if (hoist) {
            Lsp[0] = __ldcg(S.Ll[0] + p);
            Lsp[1] = __ldcg(S.Ll[1] + p);
            t_in = __ldcg(S.time + p);
#pragma unroll
            for (int d = 0; d < 4; d++) pu[d] = __ldcg(S.pup[d] + p);
        }
        if constexpr (PRELOAD) {
#pragma unroll
            for (int c = 0; c < NS; c++) y0a[c] = F32C ? (double)__ldcg(S.f032 + c * cap + p) : __ldcg(S.f0 + c * cap + p);
        }
        make_stencil<float>(P, x, y, z, st);
        // (a re-sort follows the step: its keys, from fields no kernel of
        // the step writes)
        if constexpr (SG == 3 && sc_keys_in_stage3_w<WX, WY, WZ>())
            if (kout) sc_key(P, S, p, dt, true, kout, iout);
    }
    if constexpr (MTILE) {
        // the CTA's smallest and largest stencil key
        const unsigned key = active ? (unsigned)stencil_key(P, st.b) : 0u;
        const unsigned kmin = __reduce_min_sync(kFull, active ? key : 0xffffffffu);
        const unsigned kmax = __reduce_max_sync(kFull, key);
        if ((t & 31) == 0) {
            key_ext[0][t >> 5] = kmin;
            key_ext[1][t >> 5] = kmax;
        }
        __syncthreads();
    }
    grid_dep_wait();
    grid_dep_launch();
    bool live = active;   // false: this particle's staged state never arrived
    long long qsc = 0;    // SC: the particle's slot in D (the inverse, written before this stage)
    if constexpr (SC) qsc = active ? (long long)inv[p] : 0;
    if constexpr (STAGE) {
        if (s > 1 && t < 32)
            for (int c = t; c < NKS; c += 32) {
                const float* src = c < NS ? S.k32 + c * cap + p0 : S.ksum32 + (c - NS) * cap + p0;
                bulk_g2s(sk + c * kBlock, src, kBlock * 4, &stage_bar);
            }
    }
    if constexpr (MTILE) {
        // the neighbourhood's rows of the potential mesh (written by the
        // finalize kernel this stage waited for): one or two contiguous x
        // segments per (y, z) row, one lane per row
        if (t < 32) {
            if (t == 0) {
                unsigned kmin = key_ext[0][0], kmax = key_ext[1][0];
#pragma unroll
                for (int w = 1; w < kBlock / 32; w++) {
                    kmin = min(kmin, key_ext[0][w]);
                    kmax = max(kmax, key_ext[1][w]);
                }
                const MeshBox b = mesh_box(P, kmin, kmax);
                mbox = b;
                mbar_expect_tx(&mesh_bar, (unsigned)(b.nx * b.ny * b.nz * NGC * 4));
            }
            __syncwarp();
            const MeshBox b = mbox;
            const int nrow = b.ny * b.nz;
            for (int row = t; row < nrow; row += 32) {
                const int yy = row % b.ny, zz = row / b.ny;
                const int gy = (b.y0 + yy) % P.n[1], gz = (b.z0 + zz) % P.n[2];
                const long long grow = ((long long)gz * P.n[1] + gy) * P.n[0];
                float* dst = mtile + (long long)row * b.nx * NGC;
                // x from b.x0 over b.nx cells, split where it wraps
                const int first = min(b.nx, P.n[0] - b.x0);
                bulk_g2s(dst, gmesh + (grow + b.x0) * NGC, (unsigned)(first * NGC * 4), &mesh_bar);
                if (first < b.nx)
                    bulk_g2s(dst + first * NGC, gmesh + grow * NGC, (unsigned)((b.nx - first) * NGC * 4), &mesh_bar);
            }
        }
    }
    // compute_dt on the stage-4 mesh (every block has read this step's dt)
    if (dt_mode == DT_ADVANCE)
        dt_reduce_and_finish<NF, long long>(P, qdt, ctl, DT_ADVANCE, reduce_blocks(P),
                                            P.m4_reduced ? qdt + P.ncells * (8 * NH) : nullptr);
    if (active) {
        // the state arrays never alias
        const float* __restrict__ k32p = S.k32;
        const float* __restrict__ ks32p = S.ksum32;
        if constexpr (PRELOAD) {
#pragma unroll
            for (int c = 0; c < NS; c++) {
                ka[c] = s > 1 ? k32p[c * cap + p] : 0.f;
                ksa[c] = s > 2 ? ks32p[c * cap + p] : ka[c];   // (stage 2: the sum is K_1)
            }
        }
        // FP32 self-interaction part, trace removed (it commutes; three
        // flavors: the combined mesh holds only the traceless part)
        float hs[NH];
        bool tiled = false;
        if constexpr (MTILE) {
            // (the wait also orders mbox, written before the arrival)
            if (!mbar_wait(&mesh_bar, 0)) {
                atomicOr(&ctl->status, ST_TIMEOUT);
                live = false;
            } else {
                const MeshBox b = mbox;
                const int lx = wrapi(st.b[0] - b.x0, P.n[0]), ly = wrapi(st.b[1] - b.y0, P.n[1]),
                          lz = wrapi(st.b[2] - b.z0, P.n[2]);
                if (b.nx > 0 && lx + 2 < b.nx && ly + 2 < b.ny && lz + 2 < b.nz) {
                    tiled = true;
                    const float4* base =
                        reinterpret_cast<const float4*>(mtile + ((lz * b.ny + ly) * b.nx + lx) * NGC);
                    const int sy = b.nx * NGC / 4, sz = b.ny * b.nx * NGC / 4;
                    potential_si32_from<NF, SWt>(
                        P, [&](int ii, int jj, int kk, int k) { return base[kk * sz + jj * sy + ii * (NGC / 4) + k]; },
                        st, vx, vy, vz, hs);
                }
            }
        }
        if (!tiled) potential_si32<NF, SWt>(P, gmesh, st, vx, vy, vz, hs);
        if constexpr (!Comb<NF>::TRACELESS) {
            float tr = 0.f;
#pragma unroll
            for (int i = 0; i < NF; i++) tr += hs[H::re(i, i)];
            tr *= (1.0f / NF);
#pragma unroll
            for (int e = 0; e < NH; e++)
                if (H::is_diag(e)) hs[e] -= tr;
        }
        const float ih = (float)P.inv_hbar;
        const double mat = P.sqrt2GF_inv_vol * P.matter;
        const float awf = (float)(s > 1 ? dt * kRK4A[s - 1] : 0.0);
        const float anf = (float)(s < 4 ? dt * kRK4A[s] : 0.0);
        const double w6 = dt * (1.0 / 6.0);
        int stt = 0;
        if constexpr (STAGE) {
            // a thread whose wait gives up reads none of the staged state
            // and writes nothing of its particle (the step is invalid)
            if (!mbar_wait(&stage_bar, 0)) {
                atomicOr(&ctl->status, ST_TIMEOUT);
                live = false;
            }
        }
        // one species at a time keeps the live state small
#pragma unroll
        for (int sp = 0; sp < 2; sp++) {
            if (!live) break;
            // the stage state Y_s = y0 + aw K_{s-1} only enters the FP32
            // commutator and (stages 1-3) the FP32 deposit: formed in FP32
            // from the step-start state rounded to FP32 (with 1D stencils
            // stages 1-3 read only its FP32 copy); stage 4's update below is
            // FP64
            double y0[NH];
            float y0f[NH], f32[NH];
#pragma unroll
            for (int e = 0; e < NH; e++) {
                float k;
                if constexpr (PRELOAD) {
                    y0[e] = y0a[sp * NH + e];
                    k = ka[sp * NH + e];
                } else {
                    y0[e] = F32C ? (double)sf32[(sp * NH + e) * kBlock + t] : sf0[(sp * NH + e) * kBlock + t];
                    k = s > 1 ? sk[(sp * NH + e) * kBlock + t] : 0.f;
                }
                y0f[e] = (float)y0[e];
                f32[e] = s > 1 ? fmaf(awf, k, y0f[e]) : y0f[e];
            }
            // nubar: H_SI conjugated and negated (generate_code.py:317-355)
            float hsn[NH], ksi[NH];
#pragma unroll
            for (int e = 0; e < NH; e++) hsn[e] = (sp == 0 || H::is_im(e)) ? hs[e] : -hs[e];
            {
                // the vacuum + matter Hamiltonian, formed in FP64 with its
                // trace removed (the commutator does not see the trace, and
                // the diagonal differences keep their precision when
                // rounded), joins the self-interaction part: one FP32
                // commutator per species gives the RHS, which is FP32 (k32,
                // ksum32) while the state and its accumulation stay FP64
                double hv[NH];
#pragma unroll
                for (int e = 0; e < NH; e++) hv[e] = P.M2[sp][e] * vs;
                hv[0] += sp == 0 ? mat : -mat;
                double tr = 0.0;
#pragma unroll
                for (int i = 0; i < NF; i++) tr += hv[H::re(i, i)];
                tr *= 1.0 / NF;
#pragma unroll
                for (int i = 0; i < NF; i++) hv[H::re(i, i)] -= tr;
#pragma unroll
                for (int e = 0; e < NH; e++) hsn[e] += (float)hv[e];
            }
            commutator<NF, float>(hsn, f32, ksi, ih);
            const float Ns = Nsp[sp];
            if (s < 4) {
#pragma unroll
                for (int e = 0; e < NH; e++) {
                    const long long o = (sp * NH + e) * cap + p;
                    const float kc = ksi[e];
                    float ks;
                    if constexpr (PRELOAD) ks = ksa[sp * NH + e];
                    else ks = s > 2 ? sks[(sp * NH + e) * kBlock + t] : (s == 2 ? sk[(sp * NH + e) * kBlock + t] : 0.f);
                    S.k32[o] = kc;
                    // (after stage 1 the running sum is K_1 = k32)
                    if (s > 1) S.ksum32[o] = fmaf(2.f, kc, ks);
                    // the next stage's state, for the deposit only
                    fN[sp * NH + e] = fmaf(anf, kc, y0f[e]) * Ns;
                }
            } else {
                double fn[NH];
#pragma unroll
                for (int e = 0; e < NH; e++) {
                    float ks;
                    if constexpr (PRELOAD) ks = ksa[sp * NH + e];
                    else ks = sks[(sp * NH + e) * kBlock + t];
                    fn[e] = y0[e] + w6 * ((double)ks + (double)ksi[e]);
                }
                stt |= renormalize<NF>(fn, PRELOAD ? Lsp[sp] : s4[(5 + sp) * kBlock + t], P.maxError);
#pragma unroll
                for (int e = 0; e < NH; e++) {
                    const float f32n = (float)fn[e];
                    constexpr bool C32 = mixed_f0_copy_w<WX, WY, WZ>();
                    if constexpr (SC) {
                        D.f0[(sp * NH + e) * cap + qsc] = fn[e];
                        if constexpr (C32) D.f032[(sp * NH + e) * cap + qsc] = f32n;
                    } else {
                        S.f0[(sp * NH + e) * cap + p] = fn[e];
                        if constexpr (C32) S.f032[(sp * NH + e) * cap + p] = f32n;
                    }
                    fN[sp * NH + e] = f32n * Ns;
                }
            }
        }
        if (s == 4 && live) {
            double xn[3] = {x, y, z};
            double tn = PRELOAD ? t_in : s4[t];
            const double pq[4] = {PRELOAD ? pu[0] : s4[kBlock + t], PRELOAD ? pu[1] : s4[2 * kBlock + t],
                                  PRELOAD ? pu[2] : s4[3 * kBlock + t], PRELOAD ? pu[3] : s4[4 * kBlock + t]};
            rk4_push(P, dt, pq, xn, tn);
            if constexpr (SC) {
#pragma unroll
                for (int d = 0; d < 3; d++) D.pos[d][qsc] = xn[d];
                D.time[qsc] = tn;
                const double L2[2] = {PRELOAD ? Lsp[0] : s4[5 * kBlock + t], PRELOAD ? Lsp[1] : s4[6 * kBlock + t]};
                sc_static_fields(P, S, D, p, qsc, pq, L2);
            } else {
#pragma unroll
                for (int d = 0; d < 3; d++) S.pos[d][p] = xn[d];
                S.time[p] = tn;
            }
            report_bad(ctl, stt, S.id[p]);
            make_stencil<float>(P, xn[0], xn[1], xn[2], st);
        }
    }
    if constexpr (STAGE) {
        // the staged state is consumed (and the copies complete) before the
        // deposit records reuse the area; when the copies do not complete
        // within the bounded wait the CTA deposits nothing
        const bool drained =
            __syncthreads_and(t != 0 || (mbar_wait(&stage_bar, 0) && (!MTILE || mbar_wait(&mesh_bar, 0))));
        if (!drained) {
            if (t == 0) atomicOr(&ctl->status, ST_TIMEOUT);
            return;
        }
    }
    if (qout) {
        // (stages 1-3: the rank the last stage 4 stored, see rk4_stage_body)
        const int given = (s < 4 && P.rank_stages) ? (active ? S.rslot[p] : t) : -1;
        if (s == 3 && !P.m4_reduced) {
            // M_4 in the full layout (N, Nbar and the fluxes apart): compute_dt
            // reads more of it than the diagonal
            tile_deposit_block<NF, SWt, float>(P, qout, live, st, fN, vx, vy, vz, QuantConv{P}, false, given);
        } else if (s == 3) {
            // M_4: the combined layout stage 4 interpolates, the diagonal N_ii
            // compute_dt reads apart, and the full layout (into qm4) only on
            // the steps after which it can be read
            constexpr int NV = Comb<NF>::NV;
            float cN[NV + 2 * NF];
            combine_species<NF>(fN, cN);
#pragma unroll
            for (int i = 0; i < NF; i++) {
                cN[NV + i] = fN[H::re(i, i)];
                cN[NV + NF + i] = fN[NH + H::re(i, i)];
            }
            long long* const qdiag = qout + P.ncells * (8 * NH);
            int sl;
            if constexpr (NF == 3 && SWt::MX * SWt::MY * SWt::MZ == 27) {
                // (27-cell stencils: the diagonal slots in the same walk)
                sl = tile_deposit_block<NF, SWt, float, long long, QuantConvG, true, NV + 2 * NF>(
                    P, qout, live, st, cN, vx, vy, vz, QuantConvG{P}, false, given,
                    DiagOut<long long, QuantConv>{qdiag, QuantConv{P}});
            } else {
                sl = tile_deposit_block<NF, SWt, float, long long, QuantConvG, true, NV + 2 * NF>(
                    P, qout, live, st, cN, vx, vy, vz, QuantConvG{P}, false, given);
                // (the records the deposit above has read, still in place)
                tile_deposit_diag<NF, kBlock, kBlock, SWt, long long>(
                    P, qdiag, reinterpret_cast<const int*>(tile_smem),
                    reinterpret_cast<const float*>(tile_smem + kBlock * 8), kBlock, true, QuantConv{P});
            }
            const bool full = m4_full_step(ctl);   // uniform over the grid
            if (full) {
                __syncthreads();   // every record has been read
                tile_deposit_block<NF, SWt, float>(P, qm4, live, st, fN, vx, vy, vz, QuantConv{P}, false, sl);
            }
            if (blockIdx.x == 0 && t == 0) ctl->m4_full = full ? 1 : 0;
        } else {
            // M_2, M_3 and the next step's M_1: only the combinations the
            // stages interpolate
            float cN[Comb<NF>::NV];
            combine_species<NF>(fN, cN);
            const int sl = tile_deposit_block<NF, SWt, float, long long, QuantConvG, true>(
                P, qout, live, st, cN, vx, vy, vz, QuantConvG{P}, s == 4, given);
            if (s == 4 && active) S.rslot[p] = sl;
        }
    }
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
    S.rslot[i] = (int)(i % kBlock);   // cell-sorted: the identity rank
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

// derivative records (interpolate_rhs_from_mesh output, Evolve.cpp:160-174)
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
// (a plain copy of every field: recomputing the derived ones from the
// momentum instead measured no faster, and slower in isolation)
__global__ void k_gather_state(DevState src, DevState dst, const unsigned* __restrict__ perm, int mixed)
{
    constexpr int NS = 2 * NF * NF;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= src.n) return;
    const long long j = perm[i];
    dst.rslot[i] = (int)(i % kBlock);   // re-sorted: the identity rank
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
        if (dst.f032)
            for (int c = 0; c < NS; c++) dst.f032[c * dst.cap + i] = src.f032[c * src.cap + j];
    }
}

// Re-sort gather fused with the deposit of the gathered (new, cell-sorted)
// state: the deposit the last RK stage makes otherwise at the moved
// positions, where the particles are out of stencil order.  Same values as
// that deposit (f N and v in the path's precision).
template <int NF, int WX, int WY, int WZ, bool MIXED>
__global__ void __launch_bounds__(kBlock) k_gather_deposit(DevParams P, DevState src, DevState dst,
                                                           const unsigned* __restrict__ perm,
                                                           double* __restrict__ mesh, long long* __restrict__ qmesh)
{
    using SWt = SW<WX, WY, WZ>;
    using R = typename std::conditional<MIXED, float, double>::type;
    constexpr int NH = NF * NF, NS = 2 * NH;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < src.n;
    Stencil<R> st{};
    R fN[NS] = {};
    R vx = 0, vy = 0, vz = 0;
    if (active) {
        const long long j = perm[i];
        dst.rslot[i] = (int)(i % kBlock);   // re-sorted: the identity rank
        double x[3];
        for (int d = 0; d < 3; d++) {
            x[d] = src.pos[d][j];
            dst.pos[d][i] = x[d];
            dst.vhat[d][i] = src.vhat[d][j];
        }
        dst.time[i] = src.time[j];
        for (int d = 0; d < 4; d++) dst.pup[d][i] = src.pup[d][j];
        double Nn[2];
        for (int sp = 0; sp < 2; sp++) {
            Nn[sp] = src.Nn[sp][j];
            dst.Nn[sp][i] = Nn[sp];
            dst.Ll[sp][i] = src.Ll[sp][j];
        }
        dst.vscale[i] = src.vscale[j];
        dst.id[i] = src.id[j];
        float N32[2] = {0.f, 0.f};
        if constexpr (MIXED) {
            for (int d = 0; d < 3; d++) dst.vhat32[d][i] = src.vhat32[d][j];
            for (int sp = 0; sp < 2; sp++) {
                N32[sp] = src.N32[sp][j];
                dst.N32[sp][i] = N32[sp];
            }
            vx = src.vhat32[0][j];
            vy = src.vhat32[1][j];
            vz = src.vhat32[2][j];
        } else {
            vx = src.vhat[0][j];
            vy = src.vhat[1][j];
            vz = src.vhat[2][j];
        }
#pragma unroll
        for (int c = 0; c < NS; c++) {
            const double f = src.f0[c * src.cap + j];
            dst.f0[c * dst.cap + i] = f;
            if constexpr (MIXED) {
                if (dst.f032) dst.f032[c * dst.cap + i] = (float)f;
                fN[c] = (float)f * N32[c / NH];
            } else {
                fN[c] = f * Nn[c / NH];
            }
        }
        make_stencil<R>(P, x[0], x[1], x[2], st);
    }
    if constexpr (MIXED) {
        // the next step's first mesh: the combined layout
        float cN[Comb<NF>::NV];
        combine_species<NF>(fN, cN);
        tile_deposit_block<NF, SWt, float, long long, QuantConvG, true>(P, qmesh, active, st, cN, vx, vy, vz,
                                                                        QuantConvG{P});
    } else
        tile_deposit_block<NF, SWt, double>(P, mesh, active, st, fN, vx, vy, vz,
                                            [](double a, int) -> double { return a; });
}

// The combined deposit (Comb<NF>) of a cell-sorted mixed state, one particle
// per thread: the next step's first mesh after a re-sort.  Kept apart from
// the gather (a lean kernel of many loads in flight) so that each runs at
// its own occupancy.
template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock) k_deposit_comb(DevParams P, DevState S, long long* __restrict__ qmesh)
{
    using SWt = SW<WX, WY, WZ>;
    constexpr int NH = NF * NF, NS = 2 * NH;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < S.n;
    Stencil<float> st{};
    float fN[NS] = {};
    float vx = 0, vy = 0, vz = 0;
    if (active) {
        make_stencil<float>(P, S.pos[0][p], S.pos[1][p], S.pos[2][p], st);
        vx = S.vhat32[0][p];
        vy = S.vhat32[1][p];
        vz = S.vhat32[2][p];
        const float N0 = S.N32[0][p], N1 = S.N32[1][p];
#pragma unroll
        for (int e = 0; e < NH; e++) {
            fN[e] = (float)S.f0[e * S.cap + p] * N0;
            fN[NH + e] = (float)S.f0[(NH + e) * S.cap + p] * N1;
        }
    }
    float cN[Comb<NF>::NV];
    combine_species<NF>(fN, cN);
    tile_deposit_block<NF, SWt, float, long long, QuantConvG, true>(P, qmesh, active, st, cN, vx, vy, vz,
                                                                    QuantConvG{P});
}

__global__ void k_mixed_shadow(DevState S, int ns)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.n) return;
    for (int d = 0; d < 3; d++) S.vhat32[d][i] = (float)S.vhat[d][i];
    for (int sp = 0; sp < 2; sp++) S.N32[sp][i] = (float)S.Nn[sp][i];
    if (S.f032)
        for (int c = 0; c < ns; c++) S.f032[c * S.cap + i] = (float)S.f0[c * S.cap + i];
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

__global__ void k_ctl_hist(StepCtl* ctl, double* hist) { ctl->dt_hist = hist; }

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
    ctl->bar_count = 0u;
    ctl->bar_gen = 0u;
    ctl->dt_hist = nullptr;
    ctl->m4_full_from = 0;
    if (reset_status) {
        ctl->status = 0;
        ctl->bad = LLONG_MAX;
    }
}

__global__ void k_ctl_m4(StepCtl* ctl, int nsteps)
{
    ctl->m4_full_from = ctl->step + nsteps - 1;
}

__global__ void k_flush(double* buf, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) buf[i] = buf[i] * 0.5 + 1.0;
}

}  // namespace

// ===========================================================================
// launcher templates (explicitly instantiated per flavor count in
// emu_k_fp64_<nf>.cu / emu_k_mixed_<nf>.cu, dispatched in emu_kernels.cu)
// ===========================================================================
inline unsigned launch_grid(long long n) { return grid_for(n); }

// stencil-width specialisations: 1D along z with TSC, 3D TSC, generic
#define EMU_W_DISPATCH(P, ...)                                                    \
    do {                                                                          \
        if ((P).w[0] == 1 && (P).w[1] == 1 && (P).w[2] == 3) {                    \
            constexpr int WXv = 1, WYv = 1, WZv = 3;                              \
            __VA_ARGS__;                                                          \
        } else if ((P).w[0] == 3 && (P).w[1] == 3 && (P).w[2] == 3) {             \
            constexpr int WXv = 3, WYv = 3, WZv = 3;                              \
            __VA_ARGS__;                                                          \
        } else {                                                                  \
            constexpr int WXv = 0, WYv = 0, WZv = 0;                              \
            __VA_ARGS__;                                                          \
        }                                                                         \
    } while (0)

// tiles above the 48 KB default need the opt-in attribute (FP64, 3 flavors,
// 27-cell stencils: 51 KB)
template <class K>
void smem_optin(K kernel, int bytes)
{
    if (bytes > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

// launch with programmatic stream serialization: the kernel may start while
// the previous kernel of the stream drains (the kernels launched this way
// call grid_dep_wait before they read anything the previous kernel writes).
// A launch error is left for cudaGetLastError, like a <<<>>> launch.
template <class... KArgs, class... Args>
void launch_pdl(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t st,
                Args&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

template <int NF>
void launch_rk4_stage_t(const DevParams& P, const DevState& S, int s, const double* mesh_in, double* mesh_out,
                        double* mesh_zero, long long nzero, StepCtl* ctl, int dt_mode, cudaStream_t st)
{
    EMU_W_DISPATCH(P, {
        constexpr int bytes = tile_smem_bytes<NF, SW<WXv, WYv, WZv>, double>();
        if constexpr (kSplit<NF, WXv, WYv>) {
            smem_optin(k_rk4_stage_split<NF, WXv, WYv, WZv>, bytes);
            launch_pdl(k_rk4_stage_split<NF, WXv, WYv, WZv>, grid_for(S.n), 2 * kBlock, bytes, st, P, S, s, mesh_in,
                       mesh_out, mesh_zero, nzero, ctl, dt_mode);
        } else {
            smem_optin(k_rk4_stage<NF, WXv, WYv, WZv>, bytes);
            launch_pdl(k_rk4_stage<NF, WXv, WYv, WZv>, grid_for(S.n), kBlock, bytes, st, P, S, s, mesh_in, mesh_out,
                       mesh_zero, nzero, ctl, dt_mode);
        }
    });
}

template <int NF>
bool coop_step_fits_t(const DevParams& P, long long n)
{
    bool ok = false;
    EMU_W_DISPATCH(P, {
        constexpr int bytes = tile_smem_bytes<NF, SW<WXv, WYv, WZv>, double>();
        constexpr bool split = kSplit<NF, WXv, WYv>;
        auto kern = split ? k_rk4_step_coop_split<NF, WXv, WYv, WZv> : k_rk4_step_coop<NF, WXv, WYv, WZv>;
        smem_optin(kern, bytes);
        int per_sm = 0, dev = 0, nsm = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, split ? 2 * kBlock : kBlock, bytes) ==
                cudaSuccess)
            ok = (long long)per_sm * nsm >= (long long)grid_for(n);
    });
    cudaGetLastError();
    return ok;
}

template <int NF>
cudaError_t launch_rk4_step_coop_t(const DevParams& P, const DevState& S, double* const mesh[4], long long nmesh,
                                   StepCtl* ctl, int dt_mode, cudaStream_t st)
{
    cudaError_t err = cudaSuccess;
    EMU_W_DISPATCH(P, {
        constexpr int bytes = tile_smem_bytes<NF, SW<WXv, WYv, WZv>, double>();
        constexpr bool split = kSplit<NF, WXv, WYv>;
        auto kern = split ? k_rk4_step_coop_split<NF, WXv, WYv, WZv> : k_rk4_step_coop<NF, WXv, WYv, WZv>;
        smem_optin(kern, bytes);
        DevParams Pc = P;
        DevState Sc = S;
        double *m0 = mesh[0], *m1 = mesh[1], *m2 = mesh[2], *m3 = mesh[3];
        long long nm = nmesh;
        StepCtl* c = ctl;
        int mode = dt_mode;
        void* args[] = {&Pc, &Sc, &m0, &m1, &m2, &m3, &nm, &c, &mode};
        err = cudaLaunchCooperativeKernel((const void*)kern, dim3(grid_for(S.n)), dim3(split ? 2 * kBlock : kBlock),
                                          args, bytes, st);
    });
    return err;
}

template <int NF>
void launch_gather_deposit_t(bool mixed, const DevParams& P, const DevState& src, const DevState& dst,
                             const unsigned* perm, double* mesh, long long* qmesh, cudaStream_t st)
{
    EMU_W_DISPATCH(P, {
        if (mixed) {
            // (mixed: the gather and the deposit as two kernels, each at its
            // own occupancy)
            k_gather_state<NF><<<grid_for(src.n), kBlock, 0, st>>>(src, dst, perm, 1);
            constexpr int bytes = tile_smem_bytes<NF, SW<WXv, WYv, WZv>, float>();
            smem_optin(k_deposit_comb<NF, WXv, WYv, WZv>, bytes);
            k_deposit_comb<NF, WXv, WYv, WZv><<<grid_for(src.n), kBlock, bytes, st>>>(P, dst, qmesh);
        } else {
            constexpr int bytes = tile_smem_bytes<NF, SW<WXv, WYv, WZv>, double>();
            smem_optin(k_gather_deposit<NF, WXv, WYv, WZv, false>, bytes);
            k_gather_deposit<NF, WXv, WYv, WZv, false><<<grid_for(src.n), kBlock, bytes, st>>>(P, src, dst, perm,
                                                                                              mesh, qmesh);
        }
    });
}

template <int NF>
void launch_deposit_t(const DevParams& P, const DevState& S, const double* f, double* mesh, cudaStream_t st)
{
    EMU_W_DISPATCH(P, {
        constexpr int bytes = tile_smem_bytes<NF, SW<WXv, WYv, WZv>, double>();
        smem_optin(k_deposit<NF, WXv, WYv, WZv>, bytes);
        k_deposit<NF, WXv, WYv, WZv><<<grid_for(S.n), kBlock, bytes, st>>>(P, S, f, mesh);
    });
}

template <int NF>
void launch_rhs_t(const DevParams& P, const DevState& S, const double* f, const double* mesh, double* K,
                  cudaStream_t st)
{
    EMU_W_DISPATCH(P, (k_rhs<NF, WXv, WYv, WZv><<<grid_for(S.n), kBlock, 0, st>>>(P, S, f, mesh, K)));
}

template <int NF>
void launch_rk4_stage_mixed_t(const DevParams& P, const DevState& S, int s, const float* gmesh, long long* qout,
                              const long long* qdt, long long* qm4, StepCtl* ctl, int dt_mode, cudaStream_t st,
                              const DevState* D, const unsigned* inv, unsigned* kout, unsigned* iout)
{
    EMU_W_DISPATCH(P, {
        constexpr int bytes = mixed_stage_smem_bytes<NF, WXv, WYv, WZv>();
        const DevState& Dv = D ? *D : S;
        auto go = [&](auto kern) {
            smem_optin(kern, bytes);
            launch_pdl(kern, grid_for(S.n), kBlock, bytes, st, P, S, gmesh, qout, qdt, qm4, ctl, dt_mode, Dv, inv,
                       kout, iout);
        };
        if (s == 1) go(k_rk4_stage_mixed<NF, WXv, WYv, WZv, 1>);
        else if (s == 2) go(k_rk4_stage_mixed<NF, WXv, WYv, WZv, 2>);
        else if (s == 3) go(k_rk4_stage_mixed<NF, WXv, WYv, WZv, 3>);
        else if (D) go(k_rk4_stage_mixed<NF, WXv, WYv, WZv, 4, true>);
        else go(k_rk4_stage_mixed<NF, WXv, WYv, WZv, 4>);
    });
}

template <int NF>
void launch_deposit_comb_t(const DevParams& P, const DevState& S, long long* qmesh, cudaStream_t st)
{
    EMU_W_DISPATCH(P, {
        constexpr int bytes = tile_smem_bytes<NF, SW<WXv, WYv, WZv>, float>();
        smem_optin(k_deposit_comb<NF, WXv, WYv, WZv>, bytes);
        k_deposit_comb<NF, WXv, WYv, WZv><<<grid_for(S.n), kBlock, bytes, st>>>(P, S, qmesh);
    });
}

template <int NF>
void launch_deposit_q_t(const DevParams& P, const DevState& S, const double* f, long long* mesh, cudaStream_t st)
{
    EMU_W_DISPATCH(P, (k_deposit_q<NF, WXv, WYv, WZv><<<grid_for(S.n), kBlock, tile_smem_bytes<NF, SW<WXv, WYv, WZv>, float>(), st>>>(P, S, f, mesh)));
}

}  // namespace emu
