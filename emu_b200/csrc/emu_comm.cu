// emu_comm.cu -- particle sharding over GPUs: each rank holds a disjoint
// subset of the particles and a full (replicated) mesh; every deposit is
// summed over the ranks with one all-reduce before a stage reads it.  The
// int64 fixed-point mesh of the mixed path sums exactly, so its results do
// not depend on the rank count; the FP64 mesh sums in NCCL's order.
//
// The reference distributes boxes of cells over MPI ranks (AMReX
// DistributionMapping) and exchanges ghost cells and particles instead
// (main.cpp:85,137,166).  NCCL is loaded at run time (dlopen) when a
// communicator is attached, so the library itself does not depend on it.
#include "emu_context.cuh"

#include <nccl.h>

#include <dlfcn.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

using emu_ctx::check_launch;
using emu_ctx::fail;

namespace {

struct NcclApi {
    bool ok = false;
    std::string why;
    ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
    ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                              cudaStream_t) = nullptr;
    ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
    const char* (*GetErrorString)(ncclResult_t) = nullptr;
};

const NcclApi& nccl()
{
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        // EMU_NCCL_LIBRARY names the NCCL to use; otherwise an already loaded
        // NCCL (e.g. the one PyTorch brought) is reused by its soname
        const char* path = getenv("EMU_NCCL_LIBRARY");
        void* h = (path && *path) ? dlopen(path, RTLD_NOW | RTLD_GLOBAL) : nullptr;
        if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
        if (!h) {
            api.why = std::string("cannot load libnccl.so.2: ") + dlerror();
            return;
        }
        api.GetUniqueId = reinterpret_cast<decltype(api.GetUniqueId)>(dlsym(h, "ncclGetUniqueId"));
        api.CommInitRank = reinterpret_cast<decltype(api.CommInitRank)>(dlsym(h, "ncclCommInitRank"));
        api.AllReduce = reinterpret_cast<decltype(api.AllReduce)>(dlsym(h, "ncclAllReduce"));
        api.CommDestroy = reinterpret_cast<decltype(api.CommDestroy)>(dlsym(h, "ncclCommDestroy"));
        api.GetErrorString = reinterpret_cast<decltype(api.GetErrorString)>(dlsym(h, "ncclGetErrorString"));
        api.ok = api.GetUniqueId && api.CommInitRank && api.AllReduce && api.CommDestroy && api.GetErrorString;
        if (!api.ok) api.why = "libnccl.so.2 lacks a required symbol";
    });
    return api;
}

int nccl_fail(emu_context* ctx, ncclResult_t r, const char* what)
{
    return fail(ctx, EMU_ERR_CUDA, std::string(what) + ": " + nccl().GetErrorString(r));
}

}  // namespace

// ---------------------------------------------------------------------------
// Ranks that are contexts of one process (emu_local_group_*): the same
// sharded schedule with the exchange done by the library itself, so that it
// runs with several ranks on one GPU (NCCL takes one GPU per rank).  Each
// rank's host thread drives its context on its own stream; a reduction is a
// host rendezvous of the ranks plus stream-ordered work: every rank copies
// its contribution into its send buffer and records an event, and after the
// rendezvous every rank's stream waits for all those events and sums the
// send buffers in rank order (integer sums exact, FP64 sums in a fixed
// order), so no kernel waits on another.  A second rendezvous keeps a send
// buffer from being refilled before every rank has issued its reads.  Step
// graphs are not used by such ranks (a rendezvous is host work).
namespace {

struct LocalGroup {
    int nranks = 0;
    std::mutex mu;
    std::condition_variable cv;
    long long gen = 0;
    int arrived = 0;
    std::vector<void*> send;            // per rank: mesh-sized device buffer
    std::vector<cudaEvent_t> ready, done;
    size_t bytes = 0;
    double scal[64][8];
    bool broken = false;
};

constexpr int kLocalMaxRanks = 64;
constexpr std::chrono::seconds kRendezvousLimit(120);

// all ranks arrive (false: a rank did not come within the limit, or an
// earlier rendezvous failed)
bool rendezvous(LocalGroup& g)
{
    std::unique_lock<std::mutex> lk(g.mu);
    if (g.broken) return false;
    const long long my = g.gen;
    if (++g.arrived == g.nranks) {
        g.arrived = 0;
        g.gen++;
        g.cv.notify_all();
        return true;
    }
    if (!g.cv.wait_for(lk, kRendezvousLimit, [&] { return g.gen != my || g.broken; }) || g.broken) {
        g.broken = true;
        g.cv.notify_all();
        return false;
    }
    return true;
}

struct RankPtrs {
    const void* p[kLocalMaxRanks];
};

template <class T>
__global__ void k_sum_ranks(T* __restrict__ out, RankPtrs in, int nranks, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        T s = static_cast<const T*>(in.p[0])[i];
        for (int r = 1; r < nranks; r++) s += static_cast<const T*>(in.p[r])[i];
        out[i] = s;
    }
}

int local_reduce_mesh(emu_context* ctx, const void* src, void* mesh, bool int64, size_t count, cudaStream_t st)
{
    LocalGroup& g = *static_cast<LocalGroup*>(ctx->local);
    const int r = ctx->rank;
    if (count * 8 > g.bytes) return fail(ctx, EMU_ERR_STATE, "local group: mesh larger than the send buffers");
    for (int k = 0; k < g.nranks; k++) CU(cudaStreamWaitEvent(st, g.done[k], 0));
    CU(cudaMemcpyAsync(g.send[r], src, count * 8, cudaMemcpyDeviceToDevice, st));
    CU(cudaEventRecord(g.ready[r], st));
    if (!rendezvous(g)) return fail(ctx, EMU_ERR_STATE, "local group: a rank did not reach the mesh reduction");
    RankPtrs ptrs{};
    for (int k = 0; k < g.nranks; k++) {
        CU(cudaStreamWaitEvent(st, g.ready[k], 0));
        ptrs.p[k] = g.send[k];
    }
    const unsigned grid = (unsigned)std::min<long long>(((long long)count + 255) / 256, 148 * 8);
    if (int64) k_sum_ranks<long long><<<grid, 256, 0, st>>>(static_cast<long long*>(mesh), ptrs, g.nranks, count);
    else k_sum_ranks<double><<<grid, 256, 0, st>>>(static_cast<double*>(mesh), ptrs, g.nranks, count);
    CU(cudaGetLastError());
    CU(cudaEventRecord(g.done[r], st));
    if (!rendezvous(g)) return fail(ctx, EMU_ERR_STATE, "local group: a rank did not finish the mesh reduction");
    return EMU_OK;
}

int local_reduce_scalars(emu_context* ctx, double* v, int n, int op)
{
    LocalGroup& g = *static_cast<LocalGroup*>(ctx->local);
    {
        std::lock_guard<std::mutex> lk(g.mu);
        for (int i = 0; i < n; i++) g.scal[ctx->rank][i] = v[i];
    }
    if (!rendezvous(g)) return fail(ctx, EMU_ERR_STATE, "local group: a rank did not reach a scalar reduction");
    {
        std::lock_guard<std::mutex> lk(g.mu);
        for (int i = 0; i < n; i++) {
            double a = g.scal[0][i];
            for (int k = 1; k < g.nranks; k++) a = op ? std::max(a, g.scal[k][i]) : a + g.scal[k][i];
            v[i] = a;
        }
    }
    if (!rendezvous(g)) return fail(ctx, EMU_ERR_STATE, "local group: a rank did not finish a scalar reduction");
    return EMU_OK;
}

}  // namespace

int emu_ctx::reduce_mesh(emu_context* ctx, void* mesh, bool int64, cudaStream_t st)
{
    // (the mixed path's int64 meshes with their diagonal slots)
    const size_t count = (size_t)ctx->P.ncells * (ctx->ND + (int64 ? emu::kDiagSlots : 0));
    if (ctx->local) return local_reduce_mesh(ctx, mesh, mesh, int64, count, st);
    if (!ctx->comm) return EMU_OK;
    ncclResult_t r = nccl().AllReduce(mesh, mesh, count, int64 ? ncclInt64 : ncclFloat64, ncclSum,
                                      static_cast<ncclComm_t>(ctx->comm), st);
    return r == ncclSuccess ? EMU_OK : nccl_fail(ctx, r, "mesh all-reduce");
}

// a sharded mixed context's part of the full stage-4 mesh
static int alloc_full_part(emu_context* ctx)
{
    if (!ctx->mixed || !ctx->P.m4_reduced || ctx->qfull_part) return EMU_OK;
    const size_t bytes = sizeof(long long) * (size_t)ctx->P.ncells * ctx->ND;
    if (emu_ctx::dev_malloc(&ctx->qfull_part, bytes) != cudaSuccess)
        return fail(ctx, EMU_ERR_NOMEM, "attach: full mesh part");
    CU(cudaMemsetAsync(ctx->qfull_part, 0, bytes, ctx->stream));
    return EMU_OK;
}

int emu_ctx::reduce_mesh_into(emu_context* ctx, const long long* src, long long* dst, cudaStream_t st)
{
    const size_t count = (size_t)ctx->P.ncells * ctx->ND;
    if (ctx->local) return local_reduce_mesh(ctx, src, dst, true, count, st);
    if (!ctx->comm) return EMU_OK;
    ncclResult_t r = nccl().AllReduce(src, dst, count, ncclInt64, ncclSum, static_cast<ncclComm_t>(ctx->comm), st);
    return r == ncclSuccess ? EMU_OK : nccl_fail(ctx, r, "full mesh all-reduce");
}

// sum (op 0) or max (op 1) of host scalars over the ranks; synchronous
int emu_ctx_reduce_scalars(emu_context* ctx, double* v, int n, int op)
{
    if (ctx->local) return n > 8 ? fail(ctx, EMU_ERR_ARG, "reduce_scalars: too many values")
                                 : local_reduce_scalars(ctx, v, n, op);
    if (!ctx->comm) return EMU_OK;
    if (n > 8) return fail(ctx, EMU_ERR_ARG, "reduce_scalars: too many values");
    CU(cudaMemcpyAsync(ctx->red_scratch, v, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    ncclResult_t r = nccl().AllReduce(ctx->red_scratch, ctx->red_scratch, n, ncclFloat64, op ? ncclMax : ncclSum,
                                      static_cast<ncclComm_t>(ctx->comm), ctx->stream);
    if (r != ncclSuccess) return nccl_fail(ctx, r, "scalar all-reduce");
    CU(cudaMemcpyAsync(v, ctx->red_scratch, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return EMU_OK;
}

void emu_ctx_comm_free(emu_context* ctx)
{
    ctx->local = nullptr;   // (the group owns its buffers)
    if (ctx->comm) nccl().CommDestroy(static_cast<ncclComm_t>(ctx->comm));
    ctx->comm = nullptr;
    if (ctx->red_scratch) emu_ctx::dev_free(ctx->red_scratch);
    ctx->red_scratch = nullptr;
}

extern "C" {

int emu_comm_id(char* id)
{
    if (!id) return EMU_ERR_ARG;
    const NcclApi& a = nccl();
    if (!a.ok) return fail(nullptr, EMU_ERR_CUDA, "emu_comm_id: " + a.why);
    ncclUniqueId u;
    ncclResult_t r = a.GetUniqueId(&u);
    if (r != ncclSuccess) return fail(nullptr, EMU_ERR_CUDA, std::string("emu_comm_id: ") + a.GetErrorString(r));
    static_assert(sizeof(u.internal) == EMU_COMM_ID_BYTES, "NCCL unique id size");
    std::memcpy(id, u.internal, sizeof(u.internal));
    return EMU_OK;
}

int emu_attach_comm(emu_context* ctx, const char* id, int rank, int nranks)
{
    if (!ctx || !id || nranks < 1 || rank < 0 || rank >= nranks)
        return fail(ctx, EMU_ERR_ARG, "emu_attach_comm: bad arguments");
    if (ctx->comm) return fail(ctx, EMU_ERR_STATE, "emu_attach_comm: a communicator is already attached");
    if (ctx->loaded) return fail(ctx, EMU_ERR_STATE, "emu_attach_comm: attach before loading particles");
    const NcclApi& a = nccl();
    if (!a.ok) return fail(ctx, EMU_ERR_CUDA, "emu_attach_comm: " + a.why);
    ncclUniqueId u;
    std::memcpy(u.internal, id, sizeof(u.internal));
    ncclComm_t c = nullptr;
    ncclResult_t r = a.CommInitRank(&c, nranks, u, rank);
    if (r != ncclSuccess) return nccl_fail(ctx, r, "emu_attach_comm");
    ctx->comm = c;
    ctx->rank = rank;
    ctx->nranks = nranks;
    if (int e = alloc_full_part(ctx)) return e;
    CU(emu_ctx::dev_malloc(&ctx->red_scratch, 8 * sizeof(double)));
    return EMU_OK;
}

int emu_local_group_create(int nranks, void** group)
{
    if (!group || nranks < 1 || nranks > kLocalMaxRanks)
        return fail(nullptr, EMU_ERR_ARG, "emu_local_group_create: bad arguments");
    auto* g = new LocalGroup();
    g->nranks = nranks;
    g->send.assign(nranks, nullptr);
    g->ready.assign(nranks, nullptr);
    g->done.assign(nranks, nullptr);
    for (int k = 0; k < nranks; k++) {
        if (cudaEventCreateWithFlags(&g->ready[k], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&g->done[k], cudaEventDisableTiming) != cudaSuccess) {
            emu_local_group_destroy(g);
            return fail(nullptr, EMU_ERR_CUDA, "emu_local_group_create: event creation failed");
        }
    }
    *group = g;
    return EMU_OK;
}

void emu_local_group_destroy(void* group)
{
    auto* g = static_cast<LocalGroup*>(group);
    if (!g) return;
    cudaDeviceSynchronize();
    for (int k = 0; k < g->nranks; k++) {
        if (g->send[k]) emu_ctx::dev_free(g->send[k]);
        if (g->ready[k]) cudaEventDestroy(g->ready[k]);
        if (g->done[k]) cudaEventDestroy(g->done[k]);
    }
    delete g;
}

int emu_attach_local(emu_context* ctx, void* group, int rank)
{
    auto* g = static_cast<LocalGroup*>(group);
    if (!ctx || !g || rank < 0 || rank >= g->nranks) return fail(ctx, EMU_ERR_ARG, "emu_attach_local: bad arguments");
    if (ctx->comm || ctx->local) return fail(ctx, EMU_ERR_STATE, "emu_attach_local: a communicator is already attached");
    if (ctx->loaded) return fail(ctx, EMU_ERR_STATE, "emu_attach_local: attach before loading particles");
    const size_t bytes = (size_t)ctx->P.ncells * (ctx->ND + emu::kDiagSlots) * 8;
    {
        std::lock_guard<std::mutex> lk(g->mu);
        if (g->send[rank]) return fail(ctx, EMU_ERR_STATE, "emu_attach_local: rank already attached");
        if (g->bytes && g->bytes != bytes) return fail(ctx, EMU_ERR_ARG, "emu_attach_local: mesh size differs");
        g->bytes = bytes;
        void* b = nullptr;
        if (emu_ctx::dev_malloc(&b, bytes) != cudaSuccess) return fail(ctx, EMU_ERR_NOMEM, "emu_attach_local");
        g->send[rank] = b;
    }
    ctx->local = g;
    ctx->rank = rank;
    ctx->nranks = g->nranks;
    if (int e = alloc_full_part(ctx)) return e;
    return EMU_OK;
}

}  // extern "C"
