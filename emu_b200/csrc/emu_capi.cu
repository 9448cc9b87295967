// emu_capi.cu -- the C ABI (include/emu_b200.h): device context, particle
// upload/download with on-device cell sorting, the step drivers (fused RK4,
// unfused Butcher tableau, mixed precision) and the CUDA-graph step loop.
#include "emu_context.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

thread_local std::string g_host_err;

int widths(int ord) { return ord >= 2 ? 3 : (ord == 1 ? 2 : 1); }

}  // namespace

std::recursive_mutex& emu_ctx::device_lock()
{
    static std::recursive_mutex m;
    return m;
}

int emu_ctx::fail(emu_context* c, int code, const std::string& msg)
{
    if (c) c->err = msg; else g_host_err = msg;
    return code;
}

int emu_ctx::check_launch(emu_context* ctx, const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ctx, EMU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return EMU_OK;
}

using emu_ctx::check_launch;
using emu_ctx::fail;

void emu_host::set_error(const std::string& msg) { g_host_err = msg; }

// DevParams from the run parameters (geometry as AMReX computes it:
// CellSize = L/n, InvCellSize = 1/CellSize)
void emu::make_devparams(const emu_params& p, DevParams& P)
{
    std::memset(&P, 0, sizeof(P));
    P.nf = p.nflavors;
    P.wait_polls = kBarrierSpins;
    double L[3] = {p.Lx, p.Ly, p.Lz};
    double dx[3];
    for (int d = 0; d < 3; d++) {
        P.n[d] = p.ncell[d];
        P.ord[d] = p.ncell[d] > 1 ? p.shape_order : 0;
        P.w[d] = widths(P.ord[d]);
        P.L[d] = L[d];
        dx[d] = L[d] / (double)p.ncell[d];
        P.dxi[d] = 1.0 / dx[d];
    }
    P.ncells = (long long)p.ncell[0] * p.ncell[1] * p.ncell[2];
    P.key_bits = 1;
    while ((1ll << P.key_bits) <= P.ncells) P.key_bits++;
    const double inv_cell_volume = P.dxi[0] * P.dxi[1] * P.dxi[2];
    P.cell_volume = dx[0] * dx[1] * dx[2];
    P.GF = emu_host::gf();
    P.sqrt2GF = std::sqrt(2.) * P.GF;
    P.sqrt2GF_inv_vol = P.sqrt2GF * inv_cell_volume;
    P.matter = p.rho_in * p.Ye_in / emu::kMp / inv_cell_volume;
    P.rho = p.rho_in;
    P.Ye = p.Ye_in;
    P.c4 = emu_host::c4();
    P.inv_hbar = 1.0 / emu::kHbar;
    P.maxError = p.maxError;
    P.cfl_factor = p.cfl_factor;
    P.flavor_cfl_factor = p.flavor_cfl_factor;
    P.max_adaptive_speedup = p.max_adaptive_speedup;
    P.m4_reduced = p.precision == EMU_PREC_MIXED && !(p.max_adaptive_speedup > 1.0);
    P.dt_translation = 0.0;
    if (p.cfl_factor > 0.0) P.dt_translation = std::min(std::min(dx[0], dx[1]), dx[2]) / emu::kC * p.cfl_factor;
    double m2[2][9];
    emu_host::vacuum_m2(p, m2);
    for (int s = 0; s < 2; s++)
        for (int e = 0; e < 9; e++) P.M2[s][e] = m2[s][e];
    P.q_scale[0] = P.q_scale[1] = 1.0;
    P.q_unscale[0] = P.q_unscale[1] = 1.0;
}

namespace {

template <class T>
T* carve(char*& ptr, long long count)
{
    T* r = reinterpret_cast<T*>(ptr);
    size_t bytes = ((size_t)count * sizeof(T) + 255) & ~(size_t)255;
    ptr += bytes;
    return r;
}

size_t persistent_bytes(int NS, bool mixed, bool f0copy, long long cap)
{
    size_t per = (size_t)(16 + NS) * 8 + 8;
    if (mixed) per += (size_t)(5 + (f0copy ? NS : 0)) * 4;
    return per * cap + 64 * 256;
}

size_t transient_bytes(int NS, bool mixed, long long cap)
{
    if (mixed) return (size_t)2 * NS * 4 * cap + (size_t)4 * cap + 4 * 256;
    return (size_t)2 * NS * 8 * cap + (size_t)4 * cap + 4 * 256;
}

void assign_persistent(DevState& S, void* block, int NS, bool mixed, bool f0copy, long long cap)
{
    char* p = static_cast<char*>(block);
    for (int d = 0; d < 3; d++) S.pos[d] = carve<double>(p, cap);
    S.time = carve<double>(p, cap);
    for (int d = 0; d < 4; d++) S.pup[d] = carve<double>(p, cap);
    for (int s = 0; s < 2; s++) S.Nn[s] = carve<double>(p, cap);
    for (int s = 0; s < 2; s++) S.Ll[s] = carve<double>(p, cap);
    for (int d = 0; d < 3; d++) S.vhat[d] = carve<double>(p, cap);
    S.vscale = carve<double>(p, cap);
    S.f0 = carve<double>(p, (long long)NS * cap);
    S.id = carve<long long>(p, cap);
    if (mixed) {
        for (int d = 0; d < 3; d++) S.vhat32[d] = carve<float>(p, cap);
        for (int s = 0; s < 2; s++) S.N32[s] = carve<float>(p, cap);
        if (f0copy) S.f032 = carve<float>(p, (long long)NS * cap);
    }
    S.cap = cap;
}

void assign_transient(DevState& S, void* block, int NS, bool mixed, long long cap)
{
    char* p = static_cast<char*>(block);
    if (mixed) {
        S.k32 = carve<float>(p, (long long)NS * cap);
        S.ksum32 = carve<float>(p, (long long)NS * cap);
        S.fs = S.acc = nullptr;
    } else {
        S.fs = carve<double>(p, (long long)NS * cap);
        S.acc = carve<double>(p, (long long)NS * cap);
        S.k32 = S.ksum32 = nullptr;
    }
    S.rslot = carve<int>(p, cap);
}

void free_graphs(emu_context* c)
{
    for (int i = 0; i < 2; i++)
        for (int v = 0; v < 2; v++)
            if (c->graph[i][v]) {
                cudaGraphExecDestroy(c->graph[i][v]);
                c->graph[i][v] = nullptr;
            }
}

int ensure_capacity(emu_context* ctx, long long n)
{
    if (n <= ctx->cap && ctx->pblock[0]) return EMU_OK;
    free_graphs(ctx);
    for (int i = 0; i < 2; i++)
        if (ctx->pblock[i]) emu_ctx::dev_free(ctx->pblock[i]);
    if (ctx->tblock) emu_ctx::dev_free(ctx->tblock);
    if (ctx->S[0].kgen) emu_ctx::dev_free(ctx->S[0].kgen);
    for (void* a : {(void*)ctx->keys, (void*)ctx->keys2, (void*)ctx->idx, (void*)ctx->idx2})
        if (a) emu_ctx::dev_free(a);
    if (ctx->sort_tmp) emu_ctx::dev_free(ctx->sort_tmp);
    ctx->pblock[0] = ctx->pblock[1] = ctx->tblock = nullptr;
    ctx->keys = ctx->keys2 = ctx->idx = ctx->idx2 = nullptr;
    ctx->sort_tmp = nullptr;
    ctx->S[0].kgen = ctx->S[1].kgen = nullptr;
    // whole 128-particle tiles: every CTA's slice of a state array is a
    // 16-byte aligned block that bulk copies may read in full
    const long long cap = (std::max<long long>(n, 1) + 127) / 128 * 128;
    for (int i = 0; i < 2; i++) {
        CU(emu_ctx::dev_malloc(&ctx->pblock[i],
                               persistent_bytes(ctx->NS, ctx->mixed, emu::mixed_f0_copy(ctx->P), cap)));
        ctx->S[i] = DevState();
        assign_persistent(ctx->S[i], ctx->pblock[i], ctx->NS, ctx->mixed, emu::mixed_f0_copy(ctx->P), cap);
    }
    CU(emu_ctx::dev_malloc(&ctx->tblock, transient_bytes(ctx->NS, ctx->mixed, cap)));
    for (int i = 0; i < 2; i++) assign_transient(ctx->S[i], ctx->tblock, ctx->NS, ctx->mixed, cap);
    CU(emu_ctx::dev_malloc(&ctx->keys, sizeof(unsigned) * cap));
    CU(emu_ctx::dev_malloc(&ctx->keys2, sizeof(unsigned) * cap));
    CU(emu_ctx::dev_malloc(&ctx->idx, sizeof(unsigned) * cap));
    CU(emu_ctx::dev_malloc(&ctx->idx2, sizeof(unsigned) * cap));
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, ctx->keys, ctx->keys2, ctx->idx, ctx->idx2, (int)cap);
    ctx->sort_tmp_bytes = tb + 256;
    CU(emu_ctx::dev_malloc(&ctx->sort_tmp, ctx->sort_tmp_bytes));
    ctx->cap = cap;
    return EMU_OK;
}

int ensure_aos(emu_context* ctx, long long n)
{
    if (n <= ctx->aos_cap && ctx->aos) return EMU_OK;
    if (ctx->aos) emu_ctx::dev_free(ctx->aos);
    ctx->aos = nullptr;
    CU(emu_ctx::dev_malloc(&ctx->aos, sizeof(double) * (size_t)std::max<long long>(n, 1) * ctx->nreal));
    ctx->aos_cap = std::max<long long>(n, 1);
    return EMU_OK;
}

int key_bits(long long ncells)
{
    int b = 1;
    while ((1ll << b) < ncells) b++;
    return b;
}

// device radix sort of (keys, idx) -> idx2 holds the permutation
int sort_perm(emu_context* ctx, long long n, cudaStream_t st)
{
    size_t tb = ctx->sort_tmp_bytes;
    CU(cub::DeviceRadixSort::SortPairs(ctx->sort_tmp, tb, ctx->keys, ctx->keys2, ctx->idx, ctx->idx2, (int)n, 0,
                                       key_bits(ctx->P.ncells), st));
    return EMU_OK;
}
int sort_perm(emu_context* ctx, long long n) { return sort_perm(ctx, n, ctx->stream); }

// The mixed path's re-sort after a step, around stage 4: the keys of the
// positions after the step (stored by stage 3 into keys and idx, or here
// when !sc_keys_in_stage3) and their sort before it (the inverse permutation in idx), the deposit of the
// re-sorted state after it.  The next step's first mesh is zeroed here too:
// once the run has ended the finalize kernel does not, and the unchanged
// state is deposited again.
int enqueue_sc_before(emu_context* ctx, cudaStream_t st)
{
    const DevState& S = ctx->S[ctx->cur];
    CU(cudaMemsetAsync(ctx->qmesh[0], 0, sizeof(long long) * ctx->P.ncells * ctx->ND, st));
    if (!emu::sc_keys_in_stage3(ctx->P)) emu::launch_sc_keys(ctx->P, S, ctx->ctl, ctx->keys, ctx->idx, st);
    int r;
    if ((r = sort_perm(ctx, S.n, st))) return r;
    emu::launch_sc_invert(ctx->idx2, ctx->idx, S.n, st);
    return EMU_OK;
}

int sync_ctl(emu_context* ctx)
{
    CU(cudaMemcpyAsync(ctx->ctl_host, ctx->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return EMU_OK;
}

// the mixed path's stage-4 mesh of the latest step in the full layout (a
// step inside a longer run keeps only the combined layout there)
int require_full_m4(emu_context* ctx, const char* what)
{
    if (!ctx->mixed || !ctx->P.m4_reduced || ctx->cur_mesh != 1) return EMU_OK;
    int r;
    if ((r = sync_ctl(ctx))) return r;
    if (!ctx->ctl_host->m4_full)
        return fail(ctx, EMU_ERR_STATE,
                    std::string(what) + ": the latest step kept only the combined layout of its stage-4 mesh (a "
                                        "step timed by emu_profile_step, or a run stopped by an error); take a step "
                                        "with emu_evolve_steps or emu_step first");
    return EMU_OK;
}

int status_of(emu_context* ctx, int64_t* bad)
{
    const StepCtl& h = *ctx->ctl_host;
    if (bad) *bad = (h.bad == LLONG_MAX) ? -1 : (int64_t)h.bad;
    if (h.status) {
        char buf[256];
        std::snprintf(buf, sizeof buf, "device status 0x%x (first particle %lld): %s%s%s%s", h.status,
                      h.bad == LLONG_MAX ? -1ll : (long long)h.bad,
                      (h.status & EMU_ERR_TRACE) ? "trace error exceeds 100*maxError; " : "",
                      (h.status & EMU_ERR_NEGDIAG) ? "negative diagonal below -100*maxError; " : "",
                      (h.status & EMU_ERR_LENGTH) ? "flavor vector length error exceeds 100*maxError; " : "",
                      (h.status & EMU_ERR_DT) ? "timestep selection failed (no limiter); " : "");
        ctx->err = buf;
    }
    return h.status;
}

// ---- mesh helpers ----------------------------------------------------------
long long mesh_elems(const emu_context* c) { return c->P.ncells * c->ND; }
// an int64 mesh of the mixed path with its diagonal slots
long long qmesh_elems(const emu_context* c) { return c->P.ncells * (c->ND + emu::kDiagSlots); }

int zero_mesh(emu_context* ctx, int i)
{
    if (ctx->mixed) CU(cudaMemsetAsync(ctx->qmesh[i], 0, sizeof(long long) * mesh_elems(ctx), ctx->stream));
    else CU(cudaMemsetAsync(ctx->mesh[i], 0, sizeof(double) * mesh_elems(ctx), ctx->stream));
    return EMU_OK;
}

// mixed path: full deposit of the current state into qfull (summed over the
// ranks)
int deposit_full_q(emu_context* ctx)
{
    const DevState& S = ctx->S[ctx->cur];
    CU(cudaMemsetAsync(ctx->qfull, 0, sizeof(long long) * mesh_elems(ctx), ctx->stream));
    emu::launch_deposit_q(ctx->nf, ctx->P, S, S.f0, ctx->qfull, ctx->stream);
    int r;
    if ((r = check_launch(ctx, "full deposit"))) return r;
    return emu_ctx::reduce_mesh(ctx, ctx->qfull, true, ctx->stream);
}

// the full mesh of the mixed path that the API reads: the last deposit's
// (after a load or emu_deposit) or the stage-4 mesh M_4 (after steps: in
// qfull with DevParams::m4_reduced, else in q[1])
// stage 3's target for the full stage-4 mesh (DevParams::m4_reduced): qfull,
// or this rank's part of it when sharded
long long* m4_target(emu_context* ctx) { return ctx->qfull_part ? ctx->qfull_part : ctx->qfull; }

// sharded: the ranks' parts of the latest full stage-4 mesh summed into qfull
int sum_full_parts(emu_context* ctx)
{
    if (!ctx->qfull_part) return EMU_OK;
    return emu_ctx::reduce_mesh_into(ctx, ctx->qfull_part, ctx->qfull, ctx->stream);
}

long long* q_current(emu_context* ctx)
{
    return (ctx->cur_mesh == 0 || ctx->P.m4_reduced) ? ctx->qfull : ctx->qmesh[1];
}

// deposit of the current state into mesh slot 0 and a clean slot 1: the
// state the fused step loop expects at a step boundary (mixed path: the full
// deposit in qfull, converted into the combined layout of slot 0)
int deposit_current(emu_context* ctx)
{
    const DevState& S = ctx->S[ctx->cur];
    int r;
    if ((r = zero_mesh(ctx, 0))) return r;
    if ((r = zero_mesh(ctx, 1))) return r;
    if (ctx->mixed) {
        if ((r = deposit_full_q(ctx))) return r;
        emu::launch_full_to_comb(ctx->nf, ctx->P, ctx->qfull, ctx->qmesh[0], ctx->stream);
        if ((r = check_launch(ctx, "combined mesh"))) return r;
    } else {
        emu::launch_deposit(ctx->nf, ctx->P, S, S.f0, ctx->mesh[0], ctx->stream);
        if ((r = check_launch(ctx, "deposit"))) return r;
        if ((r = emu_ctx::reduce_mesh(ctx, ctx->mesh[0], false, ctx->stream))) return r;
    }
    ctx->cur_mesh = 0;
    ctx->fused_ready = true;
    return EMU_OK;
}

// ---- step bodies -----------------------------------------------------------
// fused FP64 RK4: stage s reads mesh[s-1], deposits mesh[s%4], zeros mesh[(s+1)%4]
// dep4 = false: stage 4 makes no deposit (a re-sort with deposit follows)
int enqueue_rk4_fp64(emu_context* ctx, cudaStream_t st, bool with_dt, bool dep4 = true)
{
    const DevState& S = ctx->S[ctx->cur];
    int r;
    for (int s = 1; s <= 4; s++) {
        const bool dep = s < 4 || dep4;
        emu::launch_rk4_stage(ctx->nf, ctx->P, S, s, ctx->mesh[s - 1], dep ? ctx->mesh[s % 4] : nullptr,
                              ctx->mesh[(s + 1) % 4], mesh_elems(ctx), ctx->ctl,
                              (s == 4 && with_dt) ? emu::DT_ADVANCE : -1, st);
        if (dep && (r = emu_ctx::reduce_mesh(ctx, ctx->mesh[s % 4], false, st))) return r;
    }
    return check_launch(ctx, "rk4 stage");
}

// mixed RK4: finalize(q[a] -> g, zero q[b]); stage deposits into q[b]; swap
int enqueue_rk4_mixed(emu_context* ctx, cudaStream_t st, bool with_dt, bool dep4 = true)
{
    const DevState& S = ctx->S[ctx->cur];
    int a = 0;
    for (int s = 1; s <= 4; s++) {
        const int b = 1 - a;
        // M_1..M_3 in the combined layout; M_4 in q[1] (read by stage 4's
        // compute_dt until the next step's first finalize zeroes it): full,
        // or with DevParams::m4_reduced combined with the diagonal slots and
        // the full layout in qfull on the steps after which it can be read
        const bool comb = s != 4 || ctx->P.m4_reduced;
        emu::launch_finalize_mixed(ctx->nf, ctx->P, ctx->qmesh[a], ctx->qmesh[b], ctx->gmesh, ctx->ctl, comb,
                                   (s == 3 && ctx->P.m4_reduced) ? m4_target(ctx) : nullptr, st);
        int r;
        if (s == 4 && !dep4) {
            // the re-sort that follows, made by stage 4's stores (see
            // enqueue_sc_before), then the deposit of the re-sorted state
            DevState& D = ctx->S[1 - ctx->cur];
            D.n = S.n;
            if ((r = enqueue_sc_before(ctx, st))) return r;
            emu::launch_rk4_stage_mixed(ctx->nf, ctx->P, S, 4, ctx->gmesh, nullptr, ctx->qmesh[1], m4_target(ctx),
                                        ctx->ctl, with_dt ? emu::DT_ADVANCE : -1, st, &D, ctx->idx);
            emu::launch_deposit_comb(ctx->nf, ctx->P, D, ctx->qmesh[0], st);
            if ((r = emu_ctx::reduce_mesh(ctx, ctx->qmesh[0], true, st))) return r;
            continue;
        }
        const bool dep = s < 4 || dep4;
        // (stage 3 before a re-sort made by stage 4: the re-sort keys)
        const bool keys = s == 3 && !dep4 && emu::sc_keys_in_stage3(ctx->P);
        emu::launch_rk4_stage_mixed(ctx->nf, ctx->P, S, s, ctx->gmesh, dep ? ctx->qmesh[b] : nullptr, ctx->qmesh[1],
                                    m4_target(ctx), ctx->ctl, (s == 4 && with_dt) ? emu::DT_ADVANCE : -1, st, nullptr,
                                    nullptr, keys ? ctx->keys : nullptr, keys ? ctx->idx : nullptr);
        if (dep && (r = emu_ctx::reduce_mesh(ctx, ctx->qmesh[b], true, st))) return r;
        a = b;
    }
    return check_launch(ctx, "rk4 mixed stage");
}

// Butcher tableau of the integrator (TimeIntegrator: FE, trapezoid, SSPRK3, RK4)
int tableau(const emu_params& p, int& ns, double A[4][4], double b[4])
{
    std::memset(A, 0, sizeof(double) * 16);
    std::memset(b, 0, sizeof(double) * 4);
    if (p.integration_type == 0) {
        ns = 1; b[0] = 1.0;
    } else if (p.rk_type == 2) {
        ns = 2; A[1][0] = 1.0; b[0] = 0.5; b[1] = 0.5;
    } else if (p.rk_type == 3) {
        ns = 3; A[1][0] = 1.0; A[2][0] = 0.25; A[2][1] = 0.25;
        b[0] = 1. / 6.; b[1] = 1. / 6.; b[2] = 2. / 3.;
    } else if (p.rk_type == 4) {
        ns = 4; A[1][0] = 0.5; A[2][1] = 0.5; A[3][2] = 1.0;
        b[0] = 1. / 6.; b[1] = 1. / 3.; b[2] = 1. / 3.; b[3] = 1. / 6.;
    } else {
        return EMU_ERR_ARG;
    }
    return EMU_OK;
}

// unfused explicit RK step with host dt (FP64 only)
int step_generic(emu_context* ctx, double dt)
{
    int ns;
    double A[4][4], b[4];
    if (tableau(ctx->prm, ns, A, b)) return fail(ctx, EMU_ERR_ARG, "unsupported integrator");
    DevState& S = ctx->S[ctx->cur];
    const long long kstride = (long long)ctx->NS * ctx->cap;
    if (!S.kgen) {
        CU(emu_ctx::dev_malloc(&ctx->S[0].kgen, sizeof(double) * 4 * kstride));
        ctx->S[1].kgen = ctx->S[0].kgen;
    }
    int r;
    for (int i = 0; i < ns; i++) {
        const double* Y = S.f0;
        if (i > 0) {
            double coef[3];
            for (int j = 0; j < i; j++) coef[j] = dt * A[i][j];
            emu::launch_stage_state(ctx->nf, S, S.kgen, i, coef, S.fs, ctx->stream);
            Y = S.fs;
        }
        if ((r = zero_mesh(ctx, 0))) return r;
        emu::launch_deposit(ctx->nf, ctx->P, S, Y, ctx->mesh[0], ctx->stream);
        if ((r = emu_ctx::reduce_mesh(ctx, ctx->mesh[0], false, ctx->stream))) return r;
        emu::launch_rhs(ctx->nf, ctx->P, S, Y, ctx->mesh[0], S.kgen + i * kstride, ctx->stream);
    }
    double w[4];
    for (int i = 0; i < ns; i++) w[i] = dt * b[i];
    emu::launch_combine(ctx->nf, ctx->P, S, S.kgen, ns, w, ctx->ctl, ctx->stream);
    if ((r = check_launch(ctx, "generic step"))) return r;
    ctx->cur_mesh = 0;
    ctx->fused_ready = false;
    return EMU_OK;
}

// deposit: the last stage of the step just taken made no deposit; the
// gather deposits the new state (cell-sorted) into the next step's first
// mesh instead (mesh[0] / qmesh[0], zeroed here first)
int resort(emu_context* ctx, bool deposit = false)
{
    if (deposit && ctx->mixed) {
        // (the step's stage 4 has made it, into the other buffer)
        ctx->cur = 1 - ctx->cur;
        ctx->steps_since_sort = 0;
        ctx->adj_valid = false;
        return EMU_OK;
    }
    DevState& src = ctx->S[ctx->cur];
    DevState& dst = ctx->S[1 - ctx->cur];
    dst.n = src.n;
    emu::launch_state_keys(ctx->P, src, ctx->keys, ctx->idx, ctx->stream);
    int r;
    if ((r = sort_perm(ctx, src.n))) return r;
    if (deposit) {
        // The target is zeroed here, not only by the step before: when the
        // run has already ended (the step was a no-op), the gather deposits
        // the unchanged state again, and it must replace the mesh, not add
        // to it.
        if (ctx->mixed) CU(cudaMemsetAsync(ctx->qmesh[0], 0, sizeof(long long) * mesh_elems(ctx), ctx->stream));
        else CU(cudaMemsetAsync(ctx->mesh[0], 0, sizeof(double) * mesh_elems(ctx), ctx->stream));
        emu::launch_gather_deposit(ctx->nf, ctx->mixed, ctx->P, src, dst, ctx->idx2, ctx->mesh[0], ctx->qmesh[0],
                                   ctx->stream);
        if (ctx->mixed) r = emu_ctx::reduce_mesh(ctx, ctx->qmesh[0], true, ctx->stream);
        else r = emu_ctx::reduce_mesh(ctx, ctx->mesh[0], false, ctx->stream);
        if (r) return r;
    } else {
        emu::launch_gather_state(ctx->nf, ctx->mixed, ctx->P, src, dst, ctx->idx2, ctx->stream);
    }
    if ((r = check_launch(ctx, "resort"))) return r;
    ctx->cur = 1 - ctx->cur;
    ctx->steps_since_sort = 0;
    ctx->adj_valid = false;   // slot order changed
    // the deposited meshes are order independent; stage 1 of the next step
    // reads the same mesh as before the re-sort
    return EMU_OK;
}

int enqueue_step_body(emu_context* ctx, cudaStream_t st, bool dep4)
{
    return ctx->mixed ? enqueue_rk4_mixed(ctx, st, true, dep4) : enqueue_rk4_fp64(ctx, st, true, dep4);
}

int build_graph(emu_context* ctx, int variant)
{
    cudaGraph_t g = nullptr;
    int r;
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(emu_ctx::device_lock());
        CU(cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal));
        r = enqueue_step_body(ctx, ctx->cap_stream, variant == 0);
        e = cudaStreamEndCapture(ctx->cap_stream, &g);
    }
    if (r) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e != cudaSuccess) return fail(ctx, EMU_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(ctx, EMU_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    ctx->graph[ctx->cur][variant] = ex;
    ctx->graph_P[ctx->cur][variant] = ctx->P;
    ctx->graph_S[ctx->cur][variant] = ctx->S[ctx->cur];
    ctx->graph_D[ctx->cur][variant] = ctx->S[1 - ctx->cur];
    return EMU_OK;
}

bool rk4_fused(const emu_context* ctx)
{
    return ctx->prm.integration_type == 1 && ctx->prm.rk_type == 4 && (ctx->mixed || ctx->prm.fused);
}

}  // namespace

// ===========================================================================
int emu_ctx::step_device(emu_context* ctx, bool last_stage_deposit)
{
    int r;
    if (ctx->coop) {
        double* const m[4] = {ctx->mesh[0], ctx->mesh[1], ctx->mesh[2], ctx->mesh[3]};
        cudaError_t e = emu::launch_rk4_step_coop(ctx->nf, ctx->P, ctx->S[ctx->cur], m, mesh_elems(ctx), ctx->ctl,
                                                  emu::DT_ADVANCE, ctx->stream);
        if (e != cudaSuccess) return fail(ctx, EMU_ERR_CUDA, std::string("cooperative step: ") + cudaGetErrorString(e));
    } else if (ctx->local) {
        // ranks of a local group rendezvous on the host at every deposit:
        // the stages are launched one by one
        if ((r = enqueue_step_body(ctx, ctx->stream, last_stage_deposit))) return r;
    } else {
        const int c = ctx->cur, v = last_stage_deposit ? 0 : 1;
        // the graph holds its kernels' arguments by value: re-capture when
        // the parameters or the particle arrays changed since (a reload of
        // a different set); a reload of an equal set reuses it
        if (ctx->graph[c][v] && (std::memcmp(&ctx->graph_P[c][v], &ctx->P, sizeof(DevParams)) != 0 ||
                                 std::memcmp(&ctx->graph_S[c][v], &ctx->S[c], sizeof(DevState)) != 0 ||
                                 std::memcmp(&ctx->graph_D[c][v], &ctx->S[1 - c], sizeof(DevState)) != 0)) {
            cudaGraphExecDestroy(ctx->graph[c][v]);
            ctx->graph[c][v] = nullptr;
        }
        if (!ctx->graph[c][v] && (r = build_graph(ctx, v))) return r;
        CU(cudaGraphLaunch(ctx->graph[c][v], ctx->stream));
    }
    ctx->cur_mesh = ctx->mixed ? 1 : 3;
    return EMU_OK;
}

int emu_ctx::sort_state_perm(emu_context* ctx, const DevState& S)
{
    emu::launch_state_keys(ctx->P, S, ctx->keys, ctx->idx, ctx->stream);
    return sort_perm(ctx, S.n);
}

int emu_ctx::resort_now(emu_context* ctx, unsigned* perm)
{
    int r;
    if ((r = resort(ctx))) return r;
    if (perm)
        CU(cudaMemcpyAsync(perm, ctx->idx2, sizeof(unsigned) * ctx->S[ctx->cur].n, cudaMemcpyDeviceToDevice,
                           ctx->stream));
    return EMU_OK;
}

int emu_ctx::reserve(emu_context* ctx, int64_t n)
{
    if (n > (int64_t)INT_MAX) return fail(ctx, EMU_ERR_LIMIT, "load: more than 2^31-1 particles");
    if (n <= 0) return fail(ctx, EMU_ERR_ARG, "load: no particles");
    int r;
    if ((r = ensure_capacity(ctx, n))) return r;
    return ensure_aos(ctx, n);
}

// the particles are in ctx->aos (records, load order); pupt_min and the
// weight sums/maxima are this rank's
int emu_ctx::load_from_aos(emu_context* ctx, int64_t n, double pupt_min, const double tot_in[2],
                           const double mx_in[2])
{
    int r;
    // (over all ranks of a sharded run)
    double vmin_neg = -pupt_min;
    if ((r = emu_ctx_reduce_scalars(ctx, &vmin_neg, 1, 1))) return r;
    ctx->P.vvac_max = emu_host::vvac_from_pupt_min(ctx->prm, -vmin_neg);
    if (ctx->mixed) {
        std::string why;
        double tot[2] = {tot_in[0], tot_in[1]}, mx[2] = {mx_in[0], mx_in[1]};
        if ((r = emu_ctx_reduce_scalars(ctx, tot, 2, 0))) return r;
        if ((r = emu_ctx_reduce_scalars(ctx, mx, 2, 1))) return r;
        if (!emu_host::fixed_point_scales_from(tot, mx, ctx->P.q_scale, ctx->P.q_unscale, why))
            return fail(ctx, EMU_ERR_LIMIT, "load: " + why);
        // the combined self-interaction mesh sums both species
        double tg[2] = {tot[0] + tot[1], tot[0] + tot[1]}, mg[2], gs[2], gu[2];
        mg[0] = mg[1] = std::max(mx[0], mx[1]);
        if (!emu_host::fixed_point_scales_from(tg, mg, gs, gu, why)) return fail(ctx, EMU_ERR_LIMIT, "load: " + why);
        ctx->P.g_scale = gs[0];
        ctx->P.g_unscale = gu[0];
    }
    emu::launch_cell_keys(ctx->P, ctx->aos, ctx->nreal, n, ctx->keys, ctx->idx, ctx->stream);
    if ((r = sort_perm(ctx, n))) return r;
    ctx->cur = 0;
    DevState& S = ctx->S[0];
    S.n = n;
    ctx->S[1].n = n;
    emu::launch_pack(ctx->nf, ctx->P, ctx->aos, ctx->idx2, n, S, ctx->stream);
    if (ctx->mixed) emu::launch_mixed_shadow(ctx->nf, S, ctx->stream);
    if ((r = check_launch(ctx, "pack"))) return r;
    // (step graphs re-capture themselves when P or S differ from their capture)
    // fused == 2: one cooperative launch per step when the grid fits
    // (a sharded run reduces every deposit between stages: per-stage kernels)
    ctx->coop = !ctx->mixed && !ctx->comm && !ctx->local && ctx->prm.fused == 2 && rk4_fused(ctx) &&
                emu::coop_step_fits(ctx->nf, ctx->P, n);
    ctx->loaded = true;
    ctx->adj_valid = false;
    ctx->steps_since_sort = 0;
    // (asynchronous from here: the callers wait for what they need)
    return deposit_current(ctx);
}

extern "C" {

int emu_abi_version(void) { return EMU_B200_ABI_VERSION; }
int emu_nattribs(int nf) { return 8 + 2 * (2 + nf * nf); }
int emu_nreal(int nf) { return 3 + emu_nattribs(nf); }
int emu_ncomp(int nf) { return 3 + 8 * nf * nf; }

int emu_last_error(const emu_context* ctx, char* buf, size_t len)
{
    const std::string& s = ctx ? ctx->err : g_host_err;
    if (buf && len) {
        std::strncpy(buf, s.c_str(), len - 1);
        buf[len - 1] = 0;
    }
    return (int)s.size();
}

int emu_create(const emu_params* p, emu_context** out)
{
    emu_context* ctx = nullptr;
    if (!p || !out) return fail(nullptr, EMU_ERR_ARG, "emu_create: null argument");
    *out = nullptr;
    std::string why;
    if (!emu_host::validate(*p, why)) return fail(nullptr, EMU_ERR_ARG, "emu_create: " + why);
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(nullptr, EMU_ERR_CUDA, std::string("emu_create: no CUDA device: ") + cudaGetErrorString(e));
    ctx = new emu_context();
    ctx->prm = *p;
    ctx->nf = p->nflavors;
    ctx->NH = ctx->nf * ctx->nf;
    ctx->NS = 2 * ctx->NH;
    ctx->ND = 8 * ctx->NH;
    ctx->nreal = emu_nreal(ctx->nf);
    ctx->mixed = p->precision == EMU_PREC_MIXED;
    emu::make_devparams(*p, ctx->P);
    if (ctx->prm.resort_interval < 0) {
        // automatic: a 27-cell stencil loses its per-CTA cell runs within a
        // step or two once particles leave their cells, a 1D stencil within
        // several
        const int cells = ctx->P.w[0] * ctx->P.w[1] * ctx->P.w[2];
        ctx->prm.resort_interval = cells > 9 ? 1 : 16;
    }
    // with a re-sort after every step, the deposits of stages 1-3 see
    // cell-sorted particles; otherwise every deposit ranks its keys
    ctx->P.rank_stages = ctx->prm.resort_interval != 1;
    int r = EMU_OK;
    auto bail = [&](int code) {
        g_host_err = ctx->err;
        emu_destroy(ctx);
        return code;
    };
    e = cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking);
    if (e != cudaSuccess) { ctx->err = cudaGetErrorString(e); return bail(EMU_ERR_CUDA); }
    e = cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { ctx->err = cudaGetErrorString(e); return bail(EMU_ERR_CUDA); }
    e = cudaEventCreateWithFlags(&ctx->upload_done, cudaEventDisableTiming);
    if (e != cudaSuccess) { ctx->err = cudaGetErrorString(e); return bail(EMU_ERR_CUDA); }
    ctx->stream = ctx->own;
    const size_t me = (size_t)mesh_elems(ctx), mq = (size_t)qmesh_elems(ctx);
    if (ctx->mixed) {
        for (int i = 0; i < 2 && !r; i++)
            if (emu_ctx::dev_malloc(&ctx->qmesh[i], sizeof(long long) * mq) != cudaSuccess) r = EMU_ERR_NOMEM;
        if (!r && emu_ctx::dev_malloc(&ctx->qfull, sizeof(long long) * mq) != cudaSuccess) r = EMU_ERR_NOMEM;
        if (!r && emu_ctx::dev_malloc(&ctx->gmesh, sizeof(float) * ctx->P.ncells * (ctx->nf == 3 ? emu::Comb<3>::NG : emu::Comb<2>::NG)) != cudaSuccess)
            r = EMU_ERR_NOMEM;
    } else {
        for (int i = 0; i < 4 && !r; i++)
            if (emu_ctx::dev_malloc(&ctx->mesh[i], sizeof(double) * me) != cudaSuccess) r = EMU_ERR_NOMEM;
    }
    if (!r && emu_ctx::dev_malloc(&ctx->planes, sizeof(double) * ctx->P.ncells * emu_ncomp(ctx->nf)) != cudaSuccess)
        r = EMU_ERR_NOMEM;
    if (!r && emu_ctx::dev_malloc(&ctx->ctl, sizeof(StepCtl)) != cudaSuccess) r = EMU_ERR_NOMEM;
    if (!r && emu_ctx::host_malloc(&ctx->ctl_host, sizeof(StepCtl)) != cudaSuccess) r = EMU_ERR_NOMEM;
    if (r) {
        ctx->err = "emu_create: device allocation failed";
        return bail(r);
    }
    // on the context's own stream: a device-wide synchronisation would
    // break another thread's graph capture
    std::memset(ctx->ctl_host, 0, sizeof(StepCtl));
    e = cudaMemsetAsync(ctx->ctl, 0, sizeof(StepCtl), ctx->own);
    for (int i = 0; i < 4; i++)
        if (ctx->mesh[i] && e == cudaSuccess) e = cudaMemsetAsync(ctx->mesh[i], 0, sizeof(double) * me, ctx->own);
    for (int i = 0; i < 2; i++)
        if (ctx->qmesh[i] && e == cudaSuccess) e = cudaMemsetAsync(ctx->qmesh[i], 0, sizeof(long long) * mq, ctx->own);
    if (ctx->qfull && e == cudaSuccess) e = cudaMemsetAsync(ctx->qfull, 0, sizeof(long long) * mq, ctx->own);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->own);
    if (e != cudaSuccess) {
        ctx->err = "emu_create: device initialisation failed";
        return bail(EMU_ERR_CUDA);
    }
    *out = ctx;
    return EMU_OK;
}

void emu_destroy(emu_context* ctx)
{
    if (!ctx) return;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    free_graphs(ctx);
    for (int i = 0; i < 2; i++) if (ctx->pblock[i]) emu_ctx::dev_free(ctx->pblock[i]);
    if (ctx->tblock) emu_ctx::dev_free(ctx->tblock);
    if (ctx->S[0].kgen) emu_ctx::dev_free(ctx->S[0].kgen);
    for (int i = 0; i < 4; i++) if (ctx->mesh[i]) emu_ctx::dev_free(ctx->mesh[i]);
    for (int i = 0; i < 2; i++) if (ctx->qmesh[i]) emu_ctx::dev_free(ctx->qmesh[i]);
    if (ctx->qfull) emu_ctx::dev_free(ctx->qfull);
    if (ctx->qfull_part) emu_ctx::dev_free(ctx->qfull_part);
    if (ctx->gmesh) emu_ctx::dev_free(ctx->gmesh);
    if (ctx->fmesh_tmp) emu_ctx::dev_free(ctx->fmesh_tmp);
    if (ctx->planes) emu_ctx::dev_free(ctx->planes);
    if (ctx->ctl) emu_ctx::dev_free(ctx->ctl);
    if (ctx->ctl_host) emu_ctx::host_free(ctx->ctl_host);
    if (ctx->aos) emu_ctx::dev_free(ctx->aos);
    for (void* a : {(void*)ctx->keys, (void*)ctx->keys2, (void*)ctx->idx, (void*)ctx->idx2})
        if (a) emu_ctx::dev_free(a);
    if (ctx->sort_tmp) emu_ctx::dev_free(ctx->sort_tmp);
    if (ctx->stats) emu_ctx::dev_free(ctx->stats);
    if (ctx->stats_host) emu_ctx::host_free(ctx->stats_host);
    emu_ctx::adjoint_free(ctx);
    emu_ctx_comm_free(ctx);
    if (ctx->own) cudaStreamDestroy(ctx->own);
    if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
    if (ctx->upload_done) cudaEventDestroy(ctx->upload_done);
    delete ctx;
}

int emu_set_stream(emu_context* ctx, void* s)
{
    if (!ctx) return EMU_ERR_ARG;
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->stream = s ? static_cast<cudaStream_t>(s) : ctx->own;
    return EMU_OK;
}

int emu_synchronize(emu_context* ctx)
{
    if (!ctx) return EMU_ERR_ARG;
    CU(cudaStreamSynchronize(ctx->stream));
    return EMU_OK;
}

// loads of at most this many records compute their statistics on the host
constexpr int64_t kHostStatsMax = 65536;

int emu_load_particles(emu_context* ctx, const double* records, int64_t n)
{
    if (!ctx || (n > 0 && !records) || n < 0) return fail(ctx, EMU_ERR_ARG, "emu_load_particles: bad arguments");
    int r;
    if ((r = emu_ctx::reserve(ctx, n))) return r;
    CU(cudaMemcpyAsync(ctx->aos, records, sizeof(double) * (size_t)n * ctx->nreal, cudaMemcpyHostToDevice,
                       ctx->stream));
    CU(cudaEventRecord(ctx->upload_done, ctx->stream));
    // scalars derived from the particles: Vvac_max (Init.cpp:657-660) and,
    // for the mixed path, the weight sums behind the fixed-point scales.  A
    // small set is scanned on the host while its copy is in flight; a large
    // one is reduced on the device (one round trip instead of host passes
    // over the records).
    double pupt_min = INFINITY, tot[2] = {0, 0}, mx[2] = {0, 0};
    if (n > kHostStatsMax) {
        if ((r = emu_ctx::record_stats(ctx, n, pupt_min, tot, mx))) {
            cudaEventSynchronize(ctx->upload_done);   // (the records stay in use until copied)
            return r;
        }
    } else {
        for (int64_t q = 0; q < n; q++) pupt_min = std::min(pupt_min, records[q * ctx->nreal + 3 + 7]);
        if (ctx->mixed) emu_host::weight_totals(ctx->prm, records, n, tot, mx);
    }
    r = emu_ctx::load_from_aos(ctx, n, pupt_min, tot, mx);
    // the caller may reuse the records (pinned memory is copied
    // asynchronously): wait for the copy, not for the sort and deposit, and
    // on the error paths too
    const cudaError_t e = cudaEventSynchronize(ctx->upload_done);
    if (r) return r;
    if (e != cudaSuccess) return fail(ctx, EMU_ERR_CUDA, std::string("emu_load_particles: ") + cudaGetErrorString(e));
    return EMU_OK;
}

int emu_get_particles(emu_context* ctx, double* records, int64_t n)
{
    if (!ctx || !records) return fail(ctx, EMU_ERR_ARG, "emu_get_particles: bad arguments");
    if (!ctx->loaded) return fail(ctx, EMU_ERR_STATE, "emu_get_particles: no particles loaded");
    const DevState& S = ctx->S[ctx->cur];
    if (n < S.n) return fail(ctx, EMU_ERR_ARG, "emu_get_particles: output too small");
    int r;
    if ((r = ensure_aos(ctx, S.n))) return r;
    emu::launch_unpack(ctx->nf, S, ctx->aos, ctx->stream);
    if ((r = check_launch(ctx, "unpack"))) return r;
    CU(cudaMemcpyAsync(records, ctx->aos, sizeof(double) * (size_t)S.n * ctx->nreal, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return EMU_OK;
}

int emu_num_particles(const emu_context* ctx, int64_t* n)
{
    if (!ctx || !n) return EMU_ERR_ARG;
    *n = ctx->loaded ? ctx->S[ctx->cur].n : 0;
    return EMU_OK;
}

int emu_deposit(emu_context* ctx)
{
    if (!ctx) return EMU_ERR_ARG;
    if (!ctx->loaded) return fail(ctx, EMU_ERR_STATE, "emu_deposit: no particles loaded");
    int r = deposit_current(ctx);
    if (r) return r;
    CU(cudaStreamSynchronize(ctx->stream));
    return EMU_OK;
}

int emu_get_mesh(emu_context* ctx, double* out)
{
    if (!ctx || !out) return fail(ctx, EMU_ERR_ARG, "emu_get_mesh: bad arguments");
    const long long nc = ctx->P.ncells;
    if (int r0 = require_full_m4(ctx, "emu_get_mesh")) return r0;
    if (ctx->mixed) emu::launch_mesh_out_q(ctx->nf, ctx->P, q_current(ctx), ctx->planes, ctx->stream);
    else emu::launch_mesh_out(ctx->nf, ctx->P, ctx->mesh[ctx->cur_mesh], ctx->planes, ctx->stream);
    int r;
    if ((r = check_launch(ctx, "mesh out"))) return r;
    CU(cudaMemcpyAsync(out + 3 * nc, ctx->planes + 3 * nc, sizeof(double) * nc * ctx->ND, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    for (long long c = 0; c < nc; c++) {
        out[c] = ctx->prm.rho_in;
        out[nc + c] = ctx->prm.T_in;
        out[2 * nc + c] = ctx->prm.Ye_in;
    }
    return EMU_OK;
}

int emu_interpolate_rhs(emu_context* ctx, double* rhs_records)
{
    if (!ctx || !rhs_records) return fail(ctx, EMU_ERR_ARG, "emu_interpolate_rhs: bad arguments");
    if (!ctx->loaded) return fail(ctx, EMU_ERR_STATE, "emu_interpolate_rhs: no particles loaded");
    DevState& S = ctx->S[ctx->cur];
    const long long kstride = (long long)ctx->NS * ctx->cap;
    if (!S.kgen) {
        CU(emu_ctx::dev_malloc(&ctx->S[0].kgen, sizeof(double) * 4 * kstride));
        ctx->S[1].kgen = ctx->S[0].kgen;
    }
    const double* mesh = nullptr;
    if (int r0 = require_full_m4(ctx, "emu_interpolate_rhs")) return r0;
    if (ctx->mixed) {
        // the FP64 interpolation of the fixed-point mesh
        if (!ctx->fmesh_tmp) CU(emu_ctx::dev_malloc(&ctx->fmesh_tmp, sizeof(double) * mesh_elems(ctx)));
        emu::launch_q_to_f64(ctx->nf, ctx->P, q_current(ctx), ctx->fmesh_tmp, ctx->stream);
        mesh = ctx->fmesh_tmp;
    } else {
        mesh = ctx->mesh[ctx->cur_mesh];
    }
    emu::launch_rhs(ctx->nf, ctx->P, S, S.f0, mesh, S.kgen, ctx->stream);
    int r;
    if ((r = ensure_aos(ctx, S.n))) return r;
    emu::launch_unpack_rhs(ctx->nf, S, S.kgen, ctx->aos, ctx->stream);
    if ((r = check_launch(ctx, "rhs"))) return r;
    CU(cudaMemcpyAsync(rhs_records, ctx->aos, sizeof(double) * (size_t)S.n * ctx->nreal, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return EMU_OK;
}

int emu_renormalize(emu_context* ctx, int64_t* bad)
{
    if (!ctx) return EMU_ERR_ARG;
    if (!ctx->loaded) return fail(ctx, EMU_ERR_STATE, "emu_renormalize: no particles loaded");
    emu::launch_ctl_set(ctx->ctl, 0.0, 0.0, 0.0, 1, 1, ctx->stream);
    emu::launch_renorm(ctx->nf, ctx->P, ctx->S[ctx->cur], ctx->ctl, ctx->stream);
    int r;
    if ((r = check_launch(ctx, "renormalize"))) return r;
    ctx->fused_ready = false;
    if ((r = sync_ctl(ctx))) return r;
    return status_of(ctx, bad);
}

int emu_compute_dt(emu_context* ctx, double* dt)
{
    if (!ctx || !dt) return EMU_ERR_ARG;
    emu::launch_ctl_set(ctx->ctl, 0.0, 0.0, 0.0, 1, 1, ctx->stream);
    // (after steps: the diagonal slots the steps' compute_dt read)
    if (ctx->mixed)
        emu::launch_dt_q(ctx->nf, ctx->P, q_current(ctx),
                         ctx->P.m4_reduced && ctx->cur_mesh == 1 ? ctx->qmesh[1] + mesh_elems(ctx) : nullptr, ctx->ctl,
                         emu::DT_QUERY, ctx->stream);
    else emu::launch_dt(ctx->nf, ctx->P, ctx->mesh[ctx->cur_mesh], ctx->ctl, emu::DT_QUERY, ctx->stream);
    int r;
    if ((r = check_launch(ctx, "compute_dt"))) return r;
    if ((r = sync_ctl(ctx))) return r;
    *dt = ctx->ctl_host->dt;
    return status_of(ctx, nullptr);
}

int emu_step(emu_context* ctx, double dt, int64_t* bad)
{
    if (!ctx) return EMU_ERR_ARG;
    if (!ctx->loaded) return fail(ctx, EMU_ERR_STATE, "emu_step: no particles loaded");
    if (!(dt >= 0.0) || !std::isfinite(dt)) return fail(ctx, EMU_ERR_ARG, "emu_step: dt must be finite and >= 0");
    int r;
    emu::launch_ctl_set(ctx->ctl, dt, 0.0, INFINITY, 1, 1, ctx->stream);
    if (rk4_fused(ctx)) {
        if (!ctx->fused_ready && (r = deposit_current(ctx))) return r;
        if (ctx->coop) {
            double* const m[4] = {ctx->mesh[0], ctx->mesh[1], ctx->mesh[2], ctx->mesh[3]};
            cudaError_t e = emu::launch_rk4_step_coop(ctx->nf, ctx->P, ctx->S[ctx->cur], m, mesh_elems(ctx), ctx->ctl,
                                                      -1, ctx->stream);
            r = e == cudaSuccess ? EMU_OK : fail(ctx, EMU_ERR_CUDA, std::string("cooperative step: ") +
                                                                      cudaGetErrorString(e));
        } else {
            r = ctx->mixed ? enqueue_rk4_mixed(ctx, ctx->stream, false) : enqueue_rk4_fp64(ctx, ctx->stream, false);
        }
        if (r) return r;
        if (ctx->mixed && (r = sum_full_parts(ctx))) return r;
        ctx->cur_mesh = ctx->mixed ? 1 : 3;
        ctx->fused_ready = true;
    } else {
        if (ctx->mixed) return fail(ctx, EMU_ERR_ARG, "emu_step: the mixed path integrates with RK4 only");
        if ((r = step_generic(ctx, dt))) return r;
    }
    if (++ctx->steps_since_sort >= ctx->prm.resort_interval && ctx->prm.resort_interval > 0)
        if ((r = resort(ctx))) return r;
    if ((r = sync_ctl(ctx))) return r;
    return status_of(ctx, bad);
}

int emu_evolve_begin(emu_context* ctx, double start_time, double end_time, int max_steps)
{
    if (!ctx) return EMU_ERR_ARG;
    if (!ctx->loaded) return fail(ctx, EMU_ERR_STATE, "emu_evolve: no particles loaded");
    if (!rk4_fused(ctx)) return fail(ctx, EMU_ERR_ARG, "emu_evolve: device-resident loop requires fused RK4");
    int r;
    if (!ctx->fused_ready && (r = deposit_current(ctx))) return r;
    emu::launch_ctl_set(ctx->ctl, 0.0, start_time, end_time, max_steps, 1, ctx->stream);
    if (ctx->mixed) {
        // the full mesh of the current state (after steps the step's first
        // mesh holds only the combined layout)
        if (ctx->cur_mesh != 0) {
            if ((r = deposit_full_q(ctx))) return r;
            ctx->cur_mesh = 0;   // qfull: the deposit of the current state
        }
        emu::launch_dt_q(ctx->nf, ctx->P, ctx->qfull, nullptr, ctx->ctl, emu::DT_INIT, ctx->stream);
    }
    else emu::launch_dt(ctx->nf, ctx->P, ctx->mesh[0], ctx->ctl, emu::DT_INIT, ctx->stream);
    return check_launch(ctx, "initial compute_dt");
}

int emu_evolve_steps(emu_context* ctx, int nsteps)
{
    if (!ctx) return EMU_ERR_ARG;
    int r;
    // the last of these steps deposits the full stage-4 mesh (the one a
    // caller can read after the call)
    if (ctx->mixed && ctx->P.m4_reduced && nsteps > 0) emu::launch_ctl_m4(ctx->ctl, nsteps, ctx->stream);
    for (int i = 0; i < nsteps; i++) {
        // when a re-sort follows this step, its gather makes the deposit of
        // the new state (in cell order) instead of the last stage
        const bool resort_next =
            ctx->prm.resort_interval > 0 && ctx->steps_since_sort + 1 >= ctx->prm.resort_interval;
        const bool fuse = resort_next && !ctx->coop;
        if ((r = emu_ctx::step_device(ctx, !fuse))) return r;
        if (resort_next) {
            ctx->steps_since_sort++;
            if ((r = resort(ctx, fuse))) return r;
        } else if (ctx->prm.resort_interval > 0) {
            ctx->steps_since_sort++;
        }
    }
    return nsteps > 0 ? sum_full_parts(ctx) : EMU_OK;
}

int emu_evolve_end(emu_context* ctx, emu_run_info* info)
{
    if (!ctx) return EMU_ERR_ARG;
    int r;
    if ((r = sync_ctl(ctx))) return r;
    const StepCtl& h = *ctx->ctl_host;
    if (info) {
        info->steps_done = h.step;
        info->status = h.status;
        info->bad_particle = h.bad == LLONG_MAX ? -1 : h.bad;
        info->time = h.t;
        info->dt_next = h.dt;
    }
    return status_of(ctx, nullptr);
}

int emu_evolve(emu_context* ctx, int nsteps, double start_time, double end_time, emu_run_info* info)
{
    int r;
    if ((r = emu_evolve_begin(ctx, start_time, end_time, nsteps))) return r;
    if ((r = emu_evolve_steps(ctx, nsteps))) return r;
    return emu_evolve_end(ctx, info);
}

int emu_set_wait_limit(emu_context* ctx, int64_t polls)
{
    if (!ctx) return EMU_ERR_ARG;
    ctx->P.wait_polls = polls < 0 ? emu::kBarrierSpins : (long long)polls;
    return EMU_OK;
}

int emu_flush_l2(emu_context* ctx, void* buf, int64_t bytes)
{
    if (!ctx || !buf) return EMU_ERR_ARG;
    emu::launch_flush(static_cast<double*>(buf), bytes / 8, ctx->stream);
    return check_launch(ctx, "flush");
}

int emu_profile_step(emu_context* ctx, float* kernel_ms, int max_kernels, int* nkernels)
{
    if (!ctx || !kernel_ms || !nkernels) return EMU_ERR_ARG;
    if (!rk4_fused(ctx)) return fail(ctx, EMU_ERR_ARG, "emu_profile_step: requires fused RK4");
    if (ctx->coop) {
        // one cooperative kernel per step
        if (max_kernels < 1) return fail(ctx, EMU_ERR_ARG, "emu_profile_step: kernel_ms too small");
        cudaEvent_t a, b;
        CU(cudaEventCreate(&a));
        CU(cudaEventCreate(&b));
        double* const m[4] = {ctx->mesh[0], ctx->mesh[1], ctx->mesh[2], ctx->mesh[3]};
        CU(cudaEventRecord(a, ctx->stream));
        cudaError_t e = emu::launch_rk4_step_coop(ctx->nf, ctx->P, ctx->S[ctx->cur], m, mesh_elems(ctx), ctx->ctl,
                                                  emu::DT_ADVANCE, ctx->stream);
        CU(cudaEventRecord(b, ctx->stream));
        if (e != cudaSuccess) return fail(ctx, EMU_ERR_CUDA, std::string("cooperative step: ") + cudaGetErrorString(e));
        CU(cudaEventSynchronize(b));
        CU(cudaEventElapsedTime(&kernel_ms[0], a, b));
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        *nkernels = 1;
        ctx->cur_mesh = 3;
        int r;
        if (ctx->prm.resort_interval > 0 && ++ctx->steps_since_sort >= ctx->prm.resort_interval)
            if ((r = resort(ctx))) return r;
        return EMU_OK;
    }
    const int nk = ctx->mixed ? 8 : 4;
    // timed as a step inside a longer run: the stage-4 mesh stays in the
    // combined layout (DevParams::m4_reduced) unless the run ends here
    if (ctx->mixed && ctx->P.m4_reduced) emu::launch_ctl_m4(ctx->ctl, 2, ctx->stream);
    const bool resort_due = ctx->prm.resort_interval > 0 && ctx->steps_since_sort + 1 >= ctx->prm.resort_interval;
    if (max_kernels < nk + (resort_due ? 1 : 0))
        return fail(ctx, EMU_ERR_ARG, "emu_profile_step: kernel_ms too small");
    std::vector<cudaEvent_t> ev(2 * nk + 4);
    for (auto& e : ev) CU(cudaEventCreate(&e));
    const DevState& S = ctx->S[ctx->cur];
    cudaStream_t st = ctx->stream;
    int k = 0;
    auto rec = [&](int i) { return cudaEventRecord(ev[i], st); };
    // (mixed: the re-sort made around stage 4, timed as one entry after the
    // stages: its keys (unless stage 3 stores them) and sort before stage 4
    // plus its deposit after it)
    const bool sc = ctx->mixed && resort_due;
    if (ctx->mixed) {
        int a = 0;
        for (int s = 1; s <= 4; s++) {
            const int b = 1 - a;
            rec(2 * k);
            emu::launch_finalize_mixed(ctx->nf, ctx->P, ctx->qmesh[a], ctx->qmesh[b], ctx->gmesh, ctx->ctl,
                                       s != 4 || ctx->P.m4_reduced,
                                       (s == 3 && ctx->P.m4_reduced) ? m4_target(ctx) : nullptr, st);
            rec(2 * k + 1);
            k++;
            int rr;
            if (s == 4 && sc) {
                DevState& D = ctx->S[1 - ctx->cur];
                D.n = S.n;
                rec(2 * nk);
                if ((rr = enqueue_sc_before(ctx, st))) return rr;
                rec(2 * nk + 1);
                rec(2 * k);
                emu::launch_rk4_stage_mixed(ctx->nf, ctx->P, S, 4, ctx->gmesh, nullptr, ctx->qmesh[1],
                                            m4_target(ctx), ctx->ctl, emu::DT_ADVANCE, st, &D, ctx->idx);
                rec(2 * k + 1);
                k++;
                rec(2 * nk + 2);
                emu::launch_deposit_comb(ctx->nf, ctx->P, D, ctx->qmesh[0], st);
                if ((rr = emu_ctx::reduce_mesh(ctx, ctx->qmesh[0], true, st))) return rr;
                rec(2 * nk + 3);
                continue;
            }
            const bool dep = s < 4 || !resort_due;
            rec(2 * k);
            const bool keys = s == 3 && sc && emu::sc_keys_in_stage3(ctx->P);
            emu::launch_rk4_stage_mixed(ctx->nf, ctx->P, S, s, ctx->gmesh, dep ? ctx->qmesh[b] : nullptr,
                                        ctx->qmesh[1], m4_target(ctx), ctx->ctl, s == 4 ? emu::DT_ADVANCE : -1, st,
                                        nullptr, nullptr, keys ? ctx->keys : nullptr, keys ? ctx->idx : nullptr);
            rec(2 * k + 1);
            k++;
            if (dep && (rr = emu_ctx::reduce_mesh(ctx, ctx->qmesh[b], true, st))) return rr;
            a = b;
        }
    } else {
        for (int s = 1; s <= 4; s++) {
            const bool dep = s < 4 || !resort_due;
            rec(2 * k);
            emu::launch_rk4_stage(ctx->nf, ctx->P, S, s, ctx->mesh[s - 1], dep ? ctx->mesh[s % 4] : nullptr,
                                  ctx->mesh[(s + 1) % 4], mesh_elems(ctx), ctx->ctl,
                                  s == 4 ? emu::DT_ADVANCE : -1, st);
            rec(2 * k + 1);
            k++;
            int rr;
            if (dep && (rr = emu_ctx::reduce_mesh(ctx, ctx->mesh[s % 4], false, st))) return rr;
        }
    }
    int r = check_launch(ctx, "profile step");
    if (r) return r;
    if (ctx->mixed && (r = sum_full_parts(ctx))) return r;
    ctx->cur_mesh = ctx->mixed ? 1 : 3;
    if (ctx->prm.resort_interval > 0) ctx->steps_since_sort++;
    if (sc) {
        if ((r = resort(ctx, true))) return r;   // (the buffers change places)
    } else if (resort_due) {
        // the re-sort that follows the step (keys, radix sort, gather and
        // the deposit of the new state) as one more entry
        rec(2 * k);
        if ((r = resort(ctx, true))) return r;
        rec(2 * k + 1);
        k++;
    }
    CU(cudaStreamSynchronize(st));
    for (int i = 0; i < k; i++) CU(cudaEventElapsedTime(&kernel_ms[i], ev[2 * i], ev[2 * i + 1]));
    if (sc) {
        float a = 0.f, b = 0.f;
        CU(cudaEventElapsedTime(&a, ev[2 * nk], ev[2 * nk + 1]));
        CU(cudaEventElapsedTime(&b, ev[2 * nk + 2], ev[2 * nk + 3]));
        kernel_ms[k++] = a + b;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    *nkernels = k;
    return EMU_OK;
}

int emu_write_plotfile(emu_context* ctx, const char* dir, double time, int step, int write_particles)
{
    if (!ctx || !dir) return fail(ctx, EMU_ERR_ARG, "emu_write_plotfile: bad arguments");
    const long long nc = ctx->P.ncells;
    std::vector<double> mesh((size_t)nc * emu_ncomp(ctx->nf));
    int r;
    if ((r = emu_get_mesh(ctx, mesh.data()))) return r;
    std::vector<double> parts;
    int64_t n = 0;
    if (write_particles) {
        emu_num_particles(ctx, &n);
        parts.resize((size_t)n * ctx->nreal);
        if ((r = emu_get_particles(ctx, parts.data(), n))) return r;
    }
    std::string why;
    if (!emu_host::write_plotfile(ctx->prm, dir, time, step, mesh.data(), write_particles ? parts.data() : nullptr,
                                  n, why))
        return fail(ctx, EMU_ERR_IO, "emu_write_plotfile: " + why);
    return EMU_OK;
}

}  // extern "C"
