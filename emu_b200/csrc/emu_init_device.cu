// emu_init_device.cu -- InitParticles on the device
// (FlavoredNeutrinoContainer::InitParticles,
// Source/FlavoredNeutrinoContainerInit.cpp:136-661): one thread per particle
// evaluates the same record function as the host generator
// (emu_init_record.h) straight into the context's record staging, then the
// regular load path sorts, packs and deposits.  This file is compiled without
// FMA contraction, so records agree bit for bit with emu_init_particles
// except where the record calls sin (simulation type 3) or exp (type 5).
// The load statistics (smallest pupt, weight sums and maxima) of any record
// set, the device init's and emu_load_particles', are reduced here too.
#include "emu_context.cuh"
#include "emu_init_record.h"

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

using emu_ctx::check_launch;
using emu_ctx::fail;

namespace {

constexpr int kStatBlock = 256;

// records of global particle indices rank, rank + nranks, ...
__global__ void k_init_records(emu_init::InitSpec s, const double* __restrict__ dirs, long long n, int rank,
                               int nranks, double* __restrict__ aos, int* bad)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long pidx = (long long)rank + i * nranks;
    if (!emu_init::init_record(s, dirs, pidx, aos + i * s.nr)) atomicOr(bad, 1);
}

// per-block (min pupt, sum |N|, sum |Nbar|, max |N|, max |Nbar|) over the
// records; the host reduces the blocks in order (deterministic)
__global__ void __launch_bounds__(kStatBlock) k_record_stats(const double* __restrict__ aos, long long n, int nr,
                                                             int nh, double* __restrict__ partial)
{
    __shared__ double sh[5][kStatBlock];
    double v[5] = {INFINITY, 0.0, 0.0, 0.0, 0.0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double* r = aos + i * nr;
        const double a = fabs(r[3 + 8]), b = fabs(r[3 + 10 + nh]);
        v[0] = fmin(v[0], r[3 + 7]);
        v[1] += a;
        v[2] += b;
        v[3] = fmax(v[3], a);
        v[4] = fmax(v[4], b);
    }
    for (int q = 0; q < 5; q++) sh[q][threadIdx.x] = v[q];
    __syncthreads();
    for (int w = kStatBlock / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            sh[0][threadIdx.x] = fmin(sh[0][threadIdx.x], sh[0][threadIdx.x + w]);
            sh[1][threadIdx.x] += sh[1][threadIdx.x + w];
            sh[2][threadIdx.x] += sh[2][threadIdx.x + w];
            sh[3][threadIdx.x] = fmax(sh[3][threadIdx.x], sh[3][threadIdx.x + w]);
            sh[4][threadIdx.x] = fmax(sh[4][threadIdx.x], sh[4][threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x < 5) partial[blockIdx.x * 5 + threadIdx.x] = sh[threadIdx.x][0];
}

}  // namespace

constexpr int kStatBlocks = 1184;

int emu_ctx::record_stats(emu_context* ctx, int64_t n, double& pupt_min, double tot[2], double mx[2])
{
    if (!ctx->stats) {
        CU(emu_ctx::dev_malloc(&ctx->stats, sizeof(double) * 5 * kStatBlocks));
        CU(emu_ctx::host_malloc(&ctx->stats_host, sizeof(double) * 5 * kStatBlocks));
    }
    const int nblk = (int)std::max<long long>(1, std::min<long long>((n + kStatBlock - 1) / kStatBlock, kStatBlocks));
    k_record_stats<<<nblk, kStatBlock, 0, ctx->stream>>>(ctx->aos, n, ctx->nreal, ctx->NH, ctx->stats);
    int r;
    if ((r = check_launch(ctx, "record statistics"))) return r;
    CU(cudaMemcpyAsync(ctx->stats_host, ctx->stats, sizeof(double) * 5 * nblk, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    const double* hp = ctx->stats_host;
    pupt_min = INFINITY;
    tot[0] = tot[1] = mx[0] = mx[1] = 0.0;
    for (int b = 0; b < nblk; b++) {
        pupt_min = std::min(pupt_min, hp[5 * b]);
        tot[0] += hp[5 * b + 1];
        tot[1] += hp[5 * b + 2];
        mx[0] = std::max(mx[0], hp[5 * b + 3]);
        mx[1] = std::max(mx[1], hp[5 * b + 4]);
    }
    return EMU_OK;
}

extern "C" int emu_init_particles_device(emu_context* ctx)
{
    if (!ctx) return EMU_ERR_ARG;
    emu_init::InitSpec s;
    std::vector<double> dirs;
    long long total = 0;
    std::string why;
    if (!emu_host::make_init_spec(ctx->prm, s, dirs, total, why))
        return fail(ctx, EMU_ERR_ARG, "emu_init_particles_device: " + why);
    const long long n = total > ctx->rank ? (total - ctx->rank + ctx->nranks - 1) / ctx->nranks : 0;
    int r;
    if ((r = emu_ctx::reserve(ctx, n))) return r;
    double* ddirs = nullptr;
    int* bad = nullptr;
    auto release = [&]() {
        if (ddirs) emu_ctx::dev_free(ddirs);
        if (bad) emu_ctx::dev_free(bad);
    };
    if (emu_ctx::dev_malloc(&ddirs, sizeof(double) * dirs.size()) != cudaSuccess || emu_ctx::dev_malloc(&bad, sizeof(int)) != cudaSuccess) {
        release();
        return fail(ctx, EMU_ERR_NOMEM, "emu_init_particles_device: scratch allocation failed");
    }
    int hbad = 0;
    cudaError_t e = cudaMemcpyAsync(ddirs, dirs.data(), sizeof(double) * dirs.size(), cudaMemcpyHostToDevice,
                                    ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int), ctx->stream);
    if (e == cudaSuccess) {
        k_init_records<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(s, ddirs, n, ctx->rank, ctx->nranks,
                                                                               ctx->aos, bad);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    release();
    if (e != cudaSuccess)
        return fail(ctx, EMU_ERR_CUDA, std::string("emu_init_particles_device: ") + cudaGetErrorString(e));
    if (hbad) return fail(ctx, EMU_ERR_ARG, "emu_init_particles_device: unknown simulation_type");
    double pupt_min, tot[2], mx[2];
    if ((r = emu_ctx::record_stats(ctx, n, pupt_min, tot, mx))) return r;
    return emu_ctx::load_from_aos(ctx, n, pupt_min, tot, mx);
}
