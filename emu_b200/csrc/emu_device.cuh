// emu_device.cuh -- device-side building blocks of the Emu evolution path on
// sm_100a: Hermitian component layout, shape factors, the interpolated
// potential, the commutator right-hand side, renormalisation and the
// shared-memory tile deposit.
//
// Reference semantics (paths relative to the Emu tree):
//   shape factors        Source/ParticleInterpolator.H:34-131
//   deposit              Source/Evolve.cpp:91-126, generate_code.py:150-169
//   potentials           Source/Evolve.cpp:128-158, generate_code.py:239-357
//   commutator RHS       Source/Evolve.cpp:160-174, generate_code.py:359-389
//   Renormalize          Source/FlavoredNeutrinoContainer.cpp:89-113,
//                        generate_code.py:391-445
#pragma once

#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

namespace emu {

// Source/Constants.H:6-26
constexpr double kC = 2.99792458e10;
constexpr double kHbar = 1.05457266e-27;
constexpr double kMp = 1.6726219e-24;
constexpr double kEV = 1.60218e-12;

constexpr unsigned kFull = 0xffffffffu;

// status bits shared with include/emu_b200.h
enum : int { ST_TRACE = 1, ST_NEGDIAG = 2, ST_LENGTH = 4, ST_DT = 8, ST_TIMEOUT = 2048 };

// ---------------------------------------------------------------------------
// Hermitian component layout: upper triangle, row-major, Re before Im
// (Scripts/symbolic_hermitians/HermitianUtils.py:170-178).
template <int NF>
struct Herm {
    static constexpr int NH = NF * NF;
    // row i starts at sum_{r<i} (1 + 2(NF-1-r)) = i(2NF - i)
    __host__ __device__ static constexpr int re(int i, int j)
    {
        return i * (2 * NF - i) + (j == i ? 0 : 2 * (j - i) - 1);
    }
    __host__ __device__ static constexpr int im(int i, int j) { return re(i, j) + 1; }
    __host__ __device__ static constexpr bool is_diag(int e)
    {
        return NF == 2 ? (e == 0 || e == 3) : (e == 0 || e == 5 || e == 8);
    }
    __host__ __device__ static constexpr bool is_im(int e)
    {
        return NF == 2 ? (e == 2) : (e == 2 || e == 4 || e == 7);
    }
};

// ---------------------------------------------------------------------------
// Geometry and physics constants handed to every kernel by value.
struct DevParams {
    int nf;
    int n[3];          // cells per dimension
    int w[3];          // stencil width per dimension (order+1, order 0 for 1-cell dims)
    int ord[3];        // shape order per dimension
    long long ncells;
    int key_bits;      // bits of a stencil key in [0, ncells]
    int rank_stages;   // particles may have moved since the last re-sort: every deposit ranks its keys
    double g_scale, g_unscale;   // fixed point of the mixed path's self-interaction mesh (both species)
    double L[3];       // domain length (periodic, [0,L))
    double dxi[3];     // inverse cell size
    double sqrt2GF_inv_vol;   // sqrt(2)*GF*inv_cell_volume (Evolve.cpp:132 + fill)
    double matter;            // rho*Ye/Mp/inv_cell_volume (uniform background)
    double M2[2][9];          // vacuum mass-squared matrix, nu and nubar (conjugated)
    double c4;                // c^4
    double inv_hbar;
    double maxError;
    double cell_volume;
    double sqrt2GF;
    double GF;
    double rho, Ye;
    double cfl_factor, flavor_cfl_factor, max_adaptive_speedup;
    double dt_translation;
    double vvac_max;
    // mixed path: int64 fixed point scales per species and the factor that
    // turns an integer mesh sum back into sqrt(2) GF n (erg)
    double q_scale[2];        // contribution * q_scale -> integer
    double q_unscale[2];      // integer * q_unscale -> number (same units as FP64 mesh)
    long long wait_polls;     // polls of a grid-barrier wait before it gives up (ST_TIMEOUT)
    // mixed path, compute_dt without the adaptive branch (max_adaptive_speedup
    // <= 1, Evolve.cpp:64-71): the only stage-4 mesh values compute_dt reads
    // are the diagonal N_ii, Nbar_ii (V_stupid, generate_code.py:287-293).  They are deposited apart (kDiagSlots per
    // cell after the mesh), and the stage-4 mesh is deposited in full only
    // where it can be read (see StepCtl::m4_full_from)
    int m4_reduced;
};

// the diagonal number densities of a cell apart from its mesh: N_ii
// (i < NF) then Nbar_ii, padded to eight int64 slots
constexpr int kDiagSlots = 8;

// ---------------------------------------------------------------------------
// ParticleInterpolator (Source/ParticleInterpolator.H:34-131).  The nearest
// index uses C truncation (static_cast<int>), reproduced exactly.
template <class R>
__device__ __forceinline__ void shape(double delta, int order, int& first, R w[3])
{
    double dstar = (delta - 0.5 < 0.0) ? delta - 1.0 : delta;
    int nearest = (int)dstar;
    double fraction = delta - (double)(int)delta;
    double offset = (delta <= 0.0) ? fraction + 0.5 : fraction - 0.5;
    if (order >= 2) {
        first = nearest - 1;
        w[0] = (R)(0.5 * (0.5 - offset) * (0.5 - offset));
        w[1] = (R)(0.75 - offset * offset);
        w[2] = (R)(0.5 * (0.5 + offset) * (0.5 + offset));
    } else if (order == 1) {
        if (offset >= 0) {
            first = nearest;
            w[0] = (R)(1.0 - offset);
            w[1] = (R)offset;
        } else {
            first = nearest - 1;
            w[0] = (R)(-offset);
            w[1] = (R)(1.0 + offset);
        }
        w[2] = (R)0;
    } else {
        first = nearest;
        w[0] = (R)1;
        w[1] = w[2] = (R)0;
    }
}

__device__ __forceinline__ int wrapi(int a, int n)
{
    int r = a % n;
    return r < 0 ? r + n : r;
}

// Stencil of one particle: first cell per dimension (wrapped) and weights.
template <class R>
struct Stencil {
    int b[3];      // first cell, already wrapped into [0,n)
    R wx[3], wy[3], wz[3];
};

template <class R>
__device__ __forceinline__ void make_stencil(const DevParams& P, double x, double y, double z, Stencil<R>& s)
{
    int f;
    shape<R>(x * P.dxi[0], P.ord[0], f, s.wx); s.b[0] = wrapi(f, P.n[0]);
    shape<R>(y * P.dxi[1], P.ord[1], f, s.wy); s.b[1] = wrapi(f, P.n[1]);
    shape<R>(z * P.dxi[2], P.ord[2], f, s.wz); s.b[2] = wrapi(f, P.n[2]);
}

__device__ __forceinline__ int stencil_key(const DevParams& P, const int b[3])
{
    return (b[2] * P.n[1] + b[1]) * P.n[0] + b[0];
}

__device__ __forceinline__ long long cell_of(const DevParams& P, int bx, int by, int bz, int ii, int jj, int kk)
{
    int i = bx + ii; if (i >= P.n[0]) i -= P.n[0];
    int j = by + jj; if (j >= P.n[1]) j -= P.n[1];
    int k = bz + kk; if (k >= P.n[2]) k -= P.n[2];
    return ((long long)k * P.n[1] + j) * P.n[0] + i;
}

// ---------------------------------------------------------------------------
// -i/hbar [H, F] in real components (generate_code.py:359-389), both given as
// Hermitian component arrays.  Fully unrolled; the index algebra folds at
// compile time.
template <int NF, class R>
__device__ __forceinline__ void commutator(const R* h, const R* f, R* out, R inv_hbar)
{
    using H = Herm<NF>;
    R HR[NF][NF], HI[NF][NF], FR[NF][NF], FI[NF][NF];
#pragma unroll
    for (int i = 0; i < NF; i++)
#pragma unroll
        for (int j = i; j < NF; j++) {
            HR[i][j] = h[H::re(i, j)];
            FR[i][j] = f[H::re(i, j)];
            if (j > i) {
                HI[i][j] = h[H::im(i, j)];
                FI[i][j] = f[H::im(i, j)];
                HR[j][i] = HR[i][j]; HI[j][i] = -HI[i][j];
                FR[j][i] = FR[i][j]; FI[j][i] = -FI[i][j];
            } else {
                HI[i][i] = (R)0;
                FI[i][i] = (R)0;
            }
        }
#pragma unroll
    for (int i = 0; i < NF; i++)
#pragma unroll
        for (int j = i; j < NF; j++) {
            R cr = (R)0, ci = (R)0;
#pragma unroll
            for (int k = 0; k < NF; k++) {
                cr += HR[i][k] * FR[k][j] - HI[i][k] * FI[k][j];
                ci += HR[i][k] * FI[k][j] + HI[i][k] * FR[k][j];
                cr -= FR[i][k] * HR[k][j] - FI[i][k] * HI[k][j];
                ci -= FR[i][k] * HI[k][j] + FI[i][k] * HR[k][j];
            }
            out[H::re(i, j)] = ci * inv_hbar;
            if (j > i) out[H::im(i, j)] = -cr * inv_hbar;
        }
}

// SU(n) flavour-vector length (HermitianUtils.py:102-123), summation in the
// order of the generated expression: Im^2 then Re^2 per off-diagonal pair,
// then the Cartan terms.
template <int NF>
__device__ __forceinline__ double su_length(const double* f)
{
    using H = Herm<NF>;
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < NF; i++)
#pragma unroll
        for (int j = i + 1; j < NF; j++) {
            double a = f[H::im(i, j)], b = f[H::re(i, j)];
            s = __dadd_rn(s, __dmul_rn(a, a));
            s = __dadd_rn(s, __dmul_rn(b, b));
        }
#pragma unroll
    for (int l = 1; l < NF; l++) {
        const double cl = (l == 1) ? 0.5 : 0.28867513459481287;   // sqrt(2/(l(l+1)))/2
        double t = 0.0;
#pragma unroll
        for (int i = 0; i < l; i++) t = __dadd_rn(t, __dmul_rn(cl, f[H::re(i, i)]));
        t = __dsub_rn(t, __dmul_rn(cl * l, f[H::re(l, l)]));
        s = __dadd_rn(s, __dmul_rn(t, t));
    }
    return sqrt(s);
}

// Renormalize one species (generate_code.py:391-445).  Returns status bits
// instead of aborting.
template <int NF>
__device__ __forceinline__ int renormalize(double* f, double L, double maxError)
{
    using H = Herm<NF>;
    int st = 0;
    double sumP = 0.0;
#pragma unroll
    for (int i = 0; i < NF; i++) sumP = __dadd_rn(sumP, f[H::re(i, i)]);
    double error = sumP - 1.0;
    if (fabs(error) > 100. * maxError) st |= ST_TRACE;
    if (fabs(error) > maxError) {
#pragma unroll
        for (int i = 0; i < NF; i++) f[H::re(i, i)] = __dsub_rn(f[H::re(i, i)], __ddiv_rn(error, (double)NF));
    }
#pragma unroll
    for (int i = 0; i < NF; i++) {
        if (f[H::re(i, i)] < -100. * maxError) st |= ST_NEGDIAG;
        if (f[H::re(i, i)] < -maxError) f[H::re(i, i)] = 0;
    }
    double length = su_length<NF>(f);
    error = length - L;
    if (fabs(error) > 100. * maxError) st |= ST_LENGTH;
    if (fabs(error) > maxError) {
        double r = __ddiv_rn(length, L);
#pragma unroll
        for (int e = 0; e < H::NH; e++) f[e] = __ddiv_rn(f[e], r);
    }
    return st;
}

// ---------------------------------------------------------------------------
// Stencil widths as template parameters: WX/WY/WZ in {1,2,3} are fixed
// widths, 0 means "runtime width up to 3".  Loops over the stencil are fully
// unrolled so that the weights and per-cell values stay in registers.
template <int WX, int WY, int WZ>
struct SW {
    static constexpr int MX = WX ? WX : 3, MY = WY ? WY : 3, MZ = WZ ? WZ : 3;
    __device__ __forceinline__ static bool on(const DevParams& P, int ii, int jj, int kk)
    {
        return (WX || ii < P.w[0]) && (WY || jj < P.w[1]) && (WZ || kk < P.w[2]);
    }
};


// mesh sums: global-memory reductions without a returned value (the mesh is
// always global memory: context, adjoint and static meshes)
__device__ __forceinline__ void atomic_add_mesh(double* p, double v)
{
    asm volatile("red.global.add.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void atomic_add_mesh(long long* p, long long v)
{
    asm volatile("red.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// ---------------------------------------------------------------------------
// Tile deposit.  The CTA's particles (consecutive in cell-sorted order) have
// written one record each to shared memory:
//   skey[i]             stencil key (first cell), -1 for no particle
//   srec[i*RW + ...]    fN[2NF^2] = f*N per species, v[3], wx[3], wy[3], wz[3]
// Threads then own deposit components q (GIdx order minus 3); each
// accumulates w*f*N*v over a run of particles with the same key in
// registers (27 accumulators in 3D, 3 in 1D) and adds the run total to the
// mesh with one atomic per (cell, component) when the key changes.  With
// ND = 32 (2 flavors) the CTA runs kBlock/32 independent particle streams.
// Record layout (R = float or double): w[SP] stencil-weight products in
// stencil order (kk, jj, ii), then fN[2NF^2], then v[3]; SP and the record
// width RW are padded to 16 bytes so the weights load as 16-byte vectors.
template <int NF, class SWt, class R>
struct TileRec {
    static constexpr int NS = 2 * NF * NF;
    static constexpr int S = SWt::MX * SWt::MY * SWt::MZ;
    static constexpr int VEC = 16 / (int)sizeof(R);
    static constexpr int SP = (S + VEC - 1) / VEC * VEC;
    static constexpr int RW = (SP + NS + 3 + VEC - 1) / VEC * VEC;
};

template <class R, int SP>
__device__ __forceinline__ void load_weights(const R* r, R (&w)[SP])
{
    if constexpr (sizeof(R) == 4) {
#pragma unroll
        for (int k = 0; k < SP; k += 4) {
            const float4 v = *reinterpret_cast<const float4*>(r + k);
            w[k] = v.x; w[k + 1] = v.y; w[k + 2] = v.z; w[k + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < SP; k += 2) {
            const double2 v = *reinterpret_cast<const double2*>(r + k);
            w[k] = v.x; w[k + 1] = v.y;
        }
    }
}

// Run accumulators of the tile deposit: S stencil-cell sums of one mesh
// component.  FP32 sums use Blackwell's packed FP32x2 FMA (two cells per
// instruction; SP pads S to an even count with zero weights).
// (two stencil cells per instruction: Blackwell's packed FP32 FMA through
// the __ffma2_rn builtin, so that the compiler allocates the register pairs)
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// Combined self-interaction layout of the mixed path's step meshes and of its
// FP32 potential mesh: per cell four blocks d (weights 1, v_x, v_y, v_z) of
// NV values each, q = d * NV + j.  Two flavors: the NF^2 combinations c_e =
// fN_nu,e - s_e fN_nubar,e (s_e = -1 for imaginary components: the
// potential's sign rule), NV = 4.  Three flavors: only the traceless part,
// which is all the commutator sees (the trace commutes with rho): NV = 8,
// j = (c_00 - tr/3, c_11 - tr/3, c_01 re, im, c_02 re, im, c_12 re, im) with
// tr = c_00 + c_11 + c_22; c_22 - tr/3 = -(j0 + j1).  32 values per cell: a
// deposit record stream is exactly one warp, and a cell is eight 16-byte
// loads.
template <int NF>
struct Comb {
    static constexpr bool TRACELESS = NF == 3;
    static constexpr int NV = TRACELESS ? 8 : NF * NF;
    static constexpr int NG = 4 * NV;
    // values of one particle (or one cell) from its NF^2 combinations c
    template <class R>
    __host__ __device__ static void values(const R* c, R* v)
    {
        if constexpr (TRACELESS) {
            const R t3 = (c[0] + c[5] + c[8]) * (R)(1.0 / 3.0);
            v[0] = c[0] - t3;
            v[1] = c[5] - t3;
            v[2] = c[1]; v[3] = c[2]; v[4] = c[3]; v[5] = c[4]; v[6] = c[6]; v[7] = c[7];
        } else {
            for (int e = 0; e < NV; e++) v[e] = c[e];
        }
    }
    // the Hermitian components (upper triangle, Re/Im) from the values
    template <class R>
    __host__ __device__ static void hermitian(const R* v, R* h)
    {
        if constexpr (TRACELESS) {
            h[0] = v[0]; h[5] = v[1]; h[8] = -(v[0] + v[1]);
            h[1] = v[2]; h[2] = v[3]; h[3] = v[4]; h[4] = v[5]; h[6] = v[6]; h[7] = v[7];
        } else {
            for (int e = 0; e < NV; e++) h[e] = v[e];
        }
    }
};

template <class R, int S, int SP>
struct RunAcc {
    R a[S];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int k = 0; k < S; k++) a[k] = (R)0;
    }
    __device__ __forceinline__ void add(const R (&w)[SP], R q)
    {
#pragma unroll
        for (int k = 0; k < S; k++) a[k] += w[k] * q;
    }
    __device__ __forceinline__ R get(int k) const { return a[k]; }
};

template <int S, int SP>
struct RunAcc<float, S, SP> {
    static constexpr int NP = (S + 1) / 2;
    static_assert(2 * NP <= SP, "padded weights");
    float2 a[NP];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int k = 0; k < NP; k++) a[k] = f2(0.f, 0.f);
    }
    __device__ __forceinline__ void add(const float (&w)[SP], float q)
    {
        const float2 qq = f2(q, q);
#pragma unroll
        for (int k = 0; k < NP; k++) a[k] = __ffma2_rn(f2(w[2 * k], w[2 * k + 1]), qq, a[k]);
    }
    // the same with the record's weights (16-byte aligned, zero padded to
    // SP) read as 16-byte vectors
    __device__ __forceinline__ void add_rec(const float* r, float q)
    {
        const float2 qq = f2(q, q);
        const float4* w4 = reinterpret_cast<const float4*>(r);
#pragma unroll
        for (int k = 0; k < NP; k += 2) {
            const float4 w = w4[k / 2];
            a[k] = __ffma2_rn(f2(w.x, w.y), qq, a[k]);
            if (k + 1 < NP) a[k + 1] = __ffma2_rn(f2(w.z, w.w), qq, a[k + 1]);
        }
    }
    // two accumulators fed by one read of the weights
    __device__ __forceinline__ static void add_rec2(RunAcc& x, RunAcc& y, const float* r, float qx, float qy)
    {
        const float2 qqx = f2(qx, qx), qqy = f2(qy, qy);
        const float4* w4 = reinterpret_cast<const float4*>(r);
#pragma unroll
        for (int k = 0; k < NP; k += 2) {
            const float4 w = w4[k / 2];
            x.a[k] = __ffma2_rn(f2(w.x, w.y), qqx, x.a[k]);
            y.a[k] = __ffma2_rn(f2(w.x, w.y), qqy, y.a[k]);
            if (k + 1 < NP) {
                x.a[k + 1] = __ffma2_rn(f2(w.z, w.w), qqx, x.a[k + 1]);
                y.a[k + 1] = __ffma2_rn(f2(w.z, w.w), qqy, y.a[k + 1]);
            }
        }
    }
    __device__ __forceinline__ float get(int k) const { return (k & 1) ? a[k / 2].y : a[k / 2].x; }
};

// Phase B of the tile deposit: thread q owns mesh component q of every
// stencil cell; it walks its stream of records (contiguous), sums each run
// of equal stencil keys in registers and adds the run total with one atomic
// per (cell, component).  Inside a run, aligned groups of four records with
// the run's key are summed without per-record key tests.
// FP32, three flavors: a thread owns the component pair (q, q + 36) (same
// f N, velocity factors d and d + 2), so that one load of a record's stencil
// weights and f N serves two run sums per cell; 36 pairs per stream, three
// streams of records per 128-thread CTA (a component per thread leaves one
// stream of 72 threads).  (Warp-aligned streams with a second pass for the
// components beyond 64 measured slower: 12.1 against 10.5 ms per C5 launch.)
template <int BLOCK, int NTILE, class SWt, class T, class Conv>
__device__ __forceinline__ void tile_deposit_pairs(const DevParams& P, T* mesh, const int* skey, const float* srec,
                                                   int ntile, Conv conv)
{
    using TR = TileRec<3, SWt, float>;
    constexpr int NH = 9, NS = 18, ND = 72, NQ = ND / 2, RW = TR::RW, SP = TR::SP, S = TR::S;
    constexpr int NSTREAM = BLOCK / NQ;
    constexpr int CH = (NTILE + NSTREAM - 1) / NSTREAM;
    const int q0 = threadIdx.x % NQ;
    const int stream = threadIdx.x / NQ;
    if (stream >= NSTREAM) return;   // no block-wide barrier follows inside
    const int q1 = q0 + NQ;
    const int dir0 = q0 / (2 * NH), sp = (q0 / NH) & 1, e = q0 % NH;   // dir1 = dir0 + 2
    const int boff = SP + sp * NH + e;
    const int voff0 = SP + NS + (dir0 > 0 ? dir0 - 1 : 0);
    const int voff1 = SP + NS + dir0 + 1;
    RunAcc<float, S, SP> acc0, acc1;
    auto flush = [&](int key) {
        const int bx = key % P.n[0];
        const int by = (key / P.n[0]) % P.n[1];
        const int bz = key / (P.n[0] * P.n[1]);
#pragma unroll
        for (int kk = 0; kk < SWt::MZ; kk++)
#pragma unroll
            for (int jj = 0; jj < SWt::MY; jj++)
#pragma unroll
                for (int ii = 0; ii < SWt::MX; ii++) {
                    if (!SWt::on(P, ii, jj, kk)) continue;
                    const int k = (kk * SWt::MY + jj) * SWt::MX + ii;
                    T* m = &mesh[cell_of(P, bx, by, bz, ii, jj, kk) * ND];
                    const T v0 = conv(acc0.get(k), sp), v1 = conv(acc1.get(k), sp);
                    if (v0 != (T)0) atomic_add_mesh(m + q0, v0);
                    if (v1 != (T)0) atomic_add_mesh(m + q1, v1);
                }
    };
    const int i1 = min((stream + 1) * CH, ntile);
    int cur = -1;
    acc0.zero();
    acc1.zero();
    for (int i = stream * CH; i < i1; i++) {
        const int key = skey[i];
        if (key != cur) {
            if (cur >= 0) flush(cur);
            acc0.zero();
            acc1.zero();
            cur = key;
        }
        if (key < 0) continue;
        const float* r = srec + i * RW;
        const float b = r[boff];
        const float qv0 = dir0 == 0 ? b : b * r[voff0];
        const float qv1 = b * r[voff1];
        RunAcc<float, S, SP>::add_rec2(acc0, acc1, r, qv0, qv1);
    }
    if (cur >= 0) flush(cur);
}

// The diagonal slots a combined deposit may sum in the same walk over its
// records (DiagOut), or none (NoDiag).
struct NoDiag {};
template <class T, class Conv>
struct DiagOut {
    T* diag;     // diag[cell * kDiagSlots + c]
    Conv conv;   // per-species fixed-point conversion
};

// Combined deposit of the mixed path (FP32 records): per cell the Comb<NF>
// values G[d][j] = sum w v_d c_j (v_0 = 1), which is all a stage's
// interpolation reads.  Records hold the particle's NV values c_j; thread
// q = (d, j) of NSTREAM = BLOCK / NG record streams sums its runs and adds
// them to mesh[cell * NG + q].  Three flavors: NG = 32, each stream is one
// warp (no divergence between streams).  The weights are read as 16-byte
// vectors, two pairs of the packed FMA each.
// With a DiagOut (27-cell stencils, three flavors): lane k < 27 of each
// stream also sums the 2 NF diagonal values of the records (at SP + NV,
// combined layout) with stencil weight k, as tile_deposit_diag's lane per
// stencil cell does (the same record ranges, runs and FP32 operations, so
// the same int64 sums), sharing this walk's key tests and flushes.
template <int NF, int BLOCK, int NTILE, class SWt, class T, class Conv, class DG = NoDiag>
__device__ __forceinline__ void tile_deposit_comb(const DevParams& P, T* mesh, const int* skey, const float* srec,
                                                  int ntile, Conv conv, DG dg = {})
{
    constexpr bool WITH_DIAG = !std::is_same<DG, NoDiag>::value;
    using TR = TileRec<NF, SWt, float>;
    using C = Comb<NF>;
    constexpr int NS = 2 * NF * NF, NV = C::NV, NG = C::NG, RW = TR::RW, SP = TR::SP, S = TR::S;
    constexpr int NP = (S + 1) / 2;   // weight pairs
    constexpr int NSTREAM = BLOCK / NG;
    static_assert(NSTREAM >= 1, "one stream of components");
    static_assert(2 * NP <= SP, "padded weights");
    constexpr int CH = (NTILE + NSTREAM - 1) / NSTREAM;
    const int q = threadIdx.x % NG;
    const int stream = threadIdx.x / NG;
    if (stream >= NSTREAM) return;   // no block-wide barrier follows inside
    const int d = q / NV, j = q % NV;
    const int coff = SP + j;
    const int voff = SP + NS + (d > 0 ? d - 1 : 0);
    static_assert(!WITH_DIAG || (S == 27 && NG == 32 && NF == 3), "diagonal slots: a lane per stencil cell");
    // (WITH_DIAG: this lane's stencil cell)
    const int dk = q / 9, dj = (q / 3) % 3, di = q % 3;
    const bool don = WITH_DIAG && q < S && SWt::on(P, di, dj, dk);
    float2 acc[NP];
    float2 dacc[WITH_DIAG ? NF : 1];
    auto flush = [&](int key) {
        const int bx = key % P.n[0];
        const int by = (key / P.n[0]) % P.n[1];
        const int bz = key / (P.n[0] * P.n[1]);
#pragma unroll
        for (int kk = 0; kk < SWt::MZ; kk++)
#pragma unroll
            for (int jj = 0; jj < SWt::MY; jj++)
#pragma unroll
                for (int ii = 0; ii < SWt::MX; ii++) {
                    if (!SWt::on(P, ii, jj, kk)) continue;
                    const int k = (kk * SWt::MY + jj) * SWt::MX + ii;
                    const float a = (k & 1) ? acc[k / 2].y : acc[k / 2].x;
                    atomic_add_mesh(&mesh[cell_of(P, bx, by, bz, ii, jj, kk) * NG + q], conv(a, 0));
                }
        if constexpr (WITH_DIAG) {
            if (don) {
                T* g = dg.diag + cell_of(P, bx, by, bz, di, dj, dk) * kDiagSlots;
#pragma unroll
                for (int m = 0; m < NF; m++) {
                    atomic_add_mesh(g + 2 * m, dg.conv(dacc[m].x, (2 * m) / NF));
                    atomic_add_mesh(g + 2 * m + 1, dg.conv(dacc[m].y, (2 * m + 1) / NF));
                }
            }
        }
    };
    auto zero = [&]() {
#pragma unroll
        for (int k = 0; k < NP; k++) acc[k] = f2(0.f, 0.f);
        if constexpr (WITH_DIAG) {
#pragma unroll
            for (int m = 0; m < NF; m++) dacc[m] = f2(0.f, 0.f);
        }
    };
    auto add_one = [&](int i) {
        const float* r = srec + i * RW;
        const float b = r[coff];
        const float qv = d == 0 ? b : b * r[voff];
        const float2 qq = f2(qv, qv);
        const float4* w4 = reinterpret_cast<const float4*>(r);
#pragma unroll
        for (int k = 0; k < NP; k += 2) {
            const float4 w = w4[k / 2];
            acc[k] = __ffma2_rn(f2(w.x, w.y), qq, acc[k]);
            if (k + 1 < NP) acc[k + 1] = __ffma2_rn(f2(w.z, w.w), qq, acc[k + 1]);
        }
        if constexpr (WITH_DIAG) {
            const float wt = q < S ? r[q] : 0.f;
            const float2 ww = f2(wt, wt);
#pragma unroll
            for (int m = 0; m < NF; m++) {
                const float2 x = reinterpret_cast<const float2*>(r + SP + NV)[m];
                dacc[m] = __ffma2_rn(x, ww, dacc[m]);
            }
        }
    };
    // (four at a time: measured 2 % faster than two on C5's stage kernels)
    constexpr int BATCH = 4;
    const int i1 = min((stream + 1) * CH, ntile);
    int cur = -1;
    zero();
    for (int i = stream * CH; i < i1; i++) {
        // BATCH records of the current run in one go: their loads are
        // independent and issue together (the stream's keys are sorted,
        // so most records continue the run)
        if (cur >= 0 && i + BATCH <= i1) {
            bool same = true;
#pragma unroll
            for (int u = 0; u < BATCH; u++) same = same && skey[i + u] == cur;
            if (same) {
#pragma unroll
                for (int u = 0; u < BATCH; u++) add_one(i + u);
                i += BATCH - 1;
                continue;
            }
        }
        const int key = skey[i];
        if (key != cur) {
            if (cur >= 0) flush(cur);
            zero();
            cur = key;
        }
        if (key < 0) continue;
        add_one(i);
    }
    if (cur >= 0) flush(cur);
}

// Deposit of the diagonal number densities N_ii, Nbar_ii (weight 1) into
// diag[cell * kDiagSlots + c], c = sp * NF + i, from the CTA's FP32 records
// (written for a full or a combined deposit, which has just read them; no
// barrier is needed, the records are only read).  The record holds the
// value of slot c at SP + voff(c): the particle's f N in the full layout,
// the values after the NV combinations in the combined one.  Eight threads
// per record stream (BLOCK / 8 streams of NTILE / (BLOCK / 8) records), or
// for 27-cell stencils a warp per stream with a lane per stencil cell: the
// grouping of the FP32 run sums, and so the int64 results, do not depend on
// which layout the records have.
template <int NF, int BLOCK, int NTILE, class SWt, class T, class Conv>
__device__ __forceinline__ void tile_deposit_diag(const DevParams& P, T* diag, const int* skey, const float* srec,
                                                  int ntile, bool comb_layout, Conv conv)
{
    using TR = TileRec<NF, SWt, float>;
    using H = Herm<NF>;
    constexpr int NH = NF * NF, RW = TR::RW, SP = TR::SP, S = TR::S;
    constexpr int NSTREAM = BLOCK / kDiagSlots;
    constexpr int CH = (NTILE + NSTREAM - 1) / NSTREAM;
    static_assert(2 * NF <= kDiagSlots, "diagonal slots");
    if constexpr (S == 27) {
        // 27-cell stencils: lane k of a record stream (one warp) owns stencil
        // cell k and sums all 2 NF values there: one weight load per record
        // and lane, one cell index per flush
        constexpr int NW = BLOCK / 32, CW = (NTILE + NW - 1) / NW;
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (w >= NW || lane >= S) return;   // no block-wide barrier follows inside
        const int kk = lane / 9, jj = (lane / 3) % 3, ii = lane % 3;
        const bool on = SWt::on(P, ii, jj, kk);
        float2 acc[NF];
        auto flush = [&](int key) {
            if (!on) return;
            const int bx = key % P.n[0];
            const int by = (key / P.n[0]) % P.n[1];
            const int bz = key / (P.n[0] * P.n[1]);
            T* g = diag + cell_of(P, bx, by, bz, ii, jj, kk) * kDiagSlots;
#pragma unroll
            for (int m = 0; m < NF; m++) {
                atomic_add_mesh(g + 2 * m, conv(acc[m].x, (2 * m) / NF));
                atomic_add_mesh(g + 2 * m + 1, conv(acc[m].y, (2 * m + 1) / NF));
            }
        };
        const int r1 = min((w + 1) * CW, ntile);
        int cur = -1;
#pragma unroll
        for (int m = 0; m < NF; m++) acc[m] = f2(0.f, 0.f);
        for (int r = w * CW; r < r1; r++) {
            const int key = skey[r];
            if (key != cur) {
                if (cur >= 0) flush(cur);
#pragma unroll
                for (int m = 0; m < NF; m++) acc[m] = f2(0.f, 0.f);
                cur = key;
            }
            if (key < 0) continue;
            const float* rec = srec + r * RW;
            const float wt = rec[lane];
            const float2 ww = f2(wt, wt);
#pragma unroll
            for (int m = 0; m < NF; m++) {
                float2 x;
                if (comb_layout) {
                    x = reinterpret_cast<const float2*>(rec + SP + Comb<NF>::NV)[m];
                } else {
                    const int c0 = 2 * m, c1 = 2 * m + 1;
                    x = f2(rec[SP + (c0 / NF) * NH + H::re(c0 % NF, c0 % NF)],
                           rec[SP + (c1 / NF) * NH + H::re(c1 % NF, c1 % NF)]);
                }
                acc[m] = __ffma2_rn(x, ww, acc[m]);
            }
        }
        if (cur >= 0) flush(cur);
        return;
    }
    const int c = threadIdx.x % kDiagSlots;
    const int stream = threadIdx.x / kDiagSlots;
    if (stream >= NSTREAM || c >= 2 * NF) return;   // no block-wide barrier follows inside
    const int sp = c / NF, i = c % NF;
    const int voff = SP + (comb_layout ? Comb<NF>::NV + c : sp * NH + H::re(i, i));
    RunAcc<float, S, SP> acc;
    auto flush = [&](int key) {
        const int bx = key % P.n[0];
        const int by = (key / P.n[0]) % P.n[1];
        const int bz = key / (P.n[0] * P.n[1]);
#pragma unroll
        for (int kk = 0; kk < SWt::MZ; kk++)
#pragma unroll
            for (int jj = 0; jj < SWt::MY; jj++)
#pragma unroll
                for (int ii = 0; ii < SWt::MX; ii++) {
                    if (!SWt::on(P, ii, jj, kk)) continue;
                    const int k = (kk * SWt::MY + jj) * SWt::MX + ii;
                    const T v = conv(acc.get(k), sp);
                    if (v != (T)0) atomic_add_mesh(&diag[cell_of(P, bx, by, bz, ii, jj, kk) * kDiagSlots + c], v);
                }
    };
    const int i1 = min((stream + 1) * CH, ntile);
    int cur = -1;
    acc.zero();
    for (int r = stream * CH; r < i1; r++) {
        const int key = skey[r];
        if (key != cur) {
            if (cur >= 0) flush(cur);
            acc.zero();
            cur = key;
        }
        if (key < 0) continue;
        const float* rec = srec + r * RW;
        acc.add_rec(rec, rec[voff]);
    }
    if (cur >= 0) flush(cur);
}

template <int NF, int BLOCK, int NTILE, class SWt, class R, class T, class Conv>
__device__ __forceinline__ void tile_deposit(const DevParams& P, T* mesh, const int* skey, const R* srec, int ntile,
                                             Conv conv)
{
    if constexpr (NF == 3 && sizeof(R) == 4 && BLOCK >= 72) {
        tile_deposit_pairs<BLOCK, NTILE, SWt, T>(P, mesh, skey, reinterpret_cast<const float*>(srec), ntile, conv);
        return;
    }
    using TR = TileRec<NF, SWt, R>;
    constexpr int NH = NF * NF, NS = 2 * NH, ND = 8 * NH, RW = TR::RW, SP = TR::SP;
    constexpr int NDP = (ND + 31) / 32 * 32;
    constexpr int NSTREAM = BLOCK / NDP > 0 ? BLOCK / NDP : 1;
    constexpr int CH = NTILE / NSTREAM;   // records per stream (a multiple of 4)
    static_assert(CH % 4 == 0, "stream chunks hold whole groups of four records");
    constexpr int SX = SWt::MX, SY = SWt::MY, SZ = SWt::MZ;
    const int q = threadIdx.x % NDP;
    const int stream = threadIdx.x / NDP;
    if (stream >= NSTREAM || q >= ND) return;   // no block-wide barrier follows inside
    const int dir = q / (2 * NH), sp = (q / NH) & 1, e = q % NH;
    const int boff = SP + sp * NH + e;               // f N of this component
    const int voff = SP + NS + (dir > 0 ? dir - 1 : 0);
    RunAcc<R, SZ * SY * SX, SP> acc;
    auto flush = [&](int key) {
        const int bx = key % P.n[0];
        const int by = (key / P.n[0]) % P.n[1];
        const int bz = key / (P.n[0] * P.n[1]);
#pragma unroll
        for (int kk = 0; kk < SZ; kk++)
#pragma unroll
            for (int jj = 0; jj < SY; jj++)
#pragma unroll
                for (int ii = 0; ii < SX; ii++) {
                    if (!SWt::on(P, ii, jj, kk)) continue;
                    const T v = conv(acc.get((kk * SY + jj) * SX + ii), sp);
                    if (v != (T)0) atomic_add_mesh(&mesh[cell_of(P, bx, by, bz, ii, jj, kk) * ND + q], v);
                }
    };
    auto add_one = [&](int i) {
        const R* r = srec + i * RW;
        const R b = r[boff];
        const R qv = dir == 0 ? b : b * r[voff];
        if constexpr (sizeof(R) == 4) {
            acc.add_rec(r, qv);
        } else {
            R w[SP];
            load_weights<R, SP>(r, w);
            acc.add(w, qv);
        }
    };
    const int i1 = min((stream + 1) * CH, ntile);
    int cur = -1;
    acc.zero();
    // FP64 27-cell runs keep the plain loop (their accumulators and weights
    // already fill the registers)
    constexpr bool QUAD = sizeof(R) == 4 || SX * SY * SZ <= 4;
    for (int i = stream * CH; i < i1;) {
        if (QUAD && (i & 3) == 0 && i + 4 <= i1 && cur >= 0) {
            const int4 k4 = *reinterpret_cast<const int4*>(skey + i);
            if (k4.x == cur && k4.y == cur && k4.z == cur && k4.w == cur) {
                // the compiler hoists the four records' loads as far as the
                // registers allow (all four for 1D stencils)
#pragma unroll
                for (int u = 0; u < 4; u++) add_one(i + u);
                i += 4;
                continue;
            }
        }
        const int key = skey[i];
        if (key != cur) {
            if (cur >= 0) flush(cur);
            acc.zero();
            cur = key;
        }
        if (key >= 0) add_one(i);
        i++;
    }
    if (cur >= 0) flush(cur);
}

// write one particle's deposit record (phase A of the tile deposit)
// (NV values per particle: f N of both species, or the NF^2 self-interaction
// combinations of the combined deposit; v always sits after 2 NF^2 slots)
template <int NF, class SWt, class R, int NV = 2 * NF * NF>
__device__ __forceinline__ void tile_record(R* srec, int* skey, int i, int key, const R* fN, R vx, R vy, R vz,
                                            const Stencil<R>& st)
{
    using TR = TileRec<NF, SWt, R>;
    constexpr int NS = TR::NS, RW = TR::RW, SP = TR::SP;
    static_assert(NV <= NS, "record values");
    skey[i] = key;
    R* r = srec + i * RW;
#pragma unroll
    for (int kk = 0; kk < SWt::MZ; kk++)
#pragma unroll
        for (int jj = 0; jj < SWt::MY; jj++)
#pragma unroll
            for (int ii = 0; ii < SWt::MX; ii++)
                r[(kk * SWt::MY + jj) * SWt::MX + ii] = (st.wx[ii] * st.wy[jj]) * st.wz[kk];
#pragma unroll
    for (int k = TR::S; k < SP; k++) r[k] = (R)0;
#pragma unroll
    for (int c = 0; c < NV; c++) r[SP + c] = fN[c];
    r[SP + NS + 0] = vx;
    r[SP + NS + 1] = vy;
    r[SP + NS + 2] = vz;
}


}  // namespace emu
