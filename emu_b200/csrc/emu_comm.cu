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

#include <cstring>
#include <mutex>
#include <string>

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
        // an already loaded NCCL (e.g. the one PyTorch brought) is reused
        void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
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

int emu_ctx::reduce_mesh(emu_context* ctx, void* mesh, bool int64, cudaStream_t st)
{
    if (!ctx->comm) return EMU_OK;
    const size_t count = (size_t)ctx->P.ncells * ctx->ND;
    ncclResult_t r = nccl().AllReduce(mesh, mesh, count, int64 ? ncclInt64 : ncclFloat64, ncclSum,
                                      static_cast<ncclComm_t>(ctx->comm), st);
    return r == ncclSuccess ? EMU_OK : nccl_fail(ctx, r, "mesh all-reduce");
}

// sum (op 0) or max (op 1) of host scalars over the ranks; synchronous
int emu_ctx_reduce_scalars(emu_context* ctx, double* v, int n, int op)
{
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
    CU(emu_ctx::dev_malloc(&ctx->red_scratch, 8 * sizeof(double)));
    return EMU_OK;
}

}  // extern "C"
