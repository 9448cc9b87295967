// emu_context.cuh -- the device context behind the C ABI handle, shared by
// the translation units that implement the C ABI (emu_capi.cu: particles,
// steps, output; emu_adjoint.cu: the discrete adjoint).
#pragma once
#include "emu_b200.h"
#include "emu_host.h"
#include "emu_kernels.cuh"

#include <mutex>
#include <string>

using emu::DevParams;
using emu::DevState;
using emu::StepCtl;

struct emu_adjoint;   // adjoint checkpoints and work arrays (emu_adjoint.cu)

struct emu_context {
    emu_params prm;
    DevParams P;
    int nf = 2, NH = 4, NS = 8, ND = 32, nreal = 23;
    bool mixed = false;
    cudaStream_t stream = nullptr;      // where work is launched
    cudaStream_t own = nullptr;         // the context's own stream
    cudaStream_t cap_stream = nullptr;  // private stream used for graph capture
    cudaEvent_t upload_done = nullptr;  // emu_load_particles: the records' copy has completed
    DevState S[2];                      // persistent particle arrays, double-buffered for re-sorts
    int cur = 0;                        // which of S[] is current
    void* pblock[2] = {nullptr, nullptr};
    void* tblock = nullptr;             // transient per-step arrays
    long long cap = 0;
    double* mesh[4] = {nullptr, nullptr, nullptr, nullptr};
    long long* qmesh[2] = {nullptr, nullptr};
    // mixed path: the full 8 NF^2 mesh of the state at the last deposit
    // (the step meshes M_1..M_3 hold only the combined self-interaction
    // layout; M_4 and this one are full, for compute_dt and the outputs)
    long long* qfull = nullptr;
    // sharded mixed path with DevParams::m4_reduced: this rank's part of the
    // full stage-4 mesh, summed into qfull after each emu_evolve_steps (the
    // device decides which steps deposit it; the sum of the latest parts is
    // the same however often it is taken)
    long long* qfull_part = nullptr;
    float* gmesh = nullptr;
    double* fmesh_tmp = nullptr;        // FP64 cell-major copy (mixed API calls)
    double* planes = nullptr;           // ncomp x ncells output staging
    StepCtl* ctl = nullptr;
    StepCtl* ctl_host = nullptr;        // pinned
    double* aos = nullptr;              // AoS staging (n x nreal)
    long long aos_cap = 0;
    unsigned *keys = nullptr, *keys2 = nullptr, *idx = nullptr, *idx2 = nullptr;
    void* sort_tmp = nullptr;
    size_t sort_tmp_bytes = 0;
    int cur_mesh = 0;
    bool fused_ready = false;
    bool loaded = false;
    // step graphs per particle buffer and variant (0: the last stage deposits
    // the new state; 1: it does not, the re-sort gather that follows does)
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    DevParams graph_P[2][2];            // kernel arguments each graph was captured with
    DevState graph_S[2][2];
    DevState graph_D[2][2];             // and the other buffer (the mixed stage 4 re-sorts into it)
    int steps_since_sort = 0;
    bool coop = false;                  // whole-step cooperative kernel (small FP64 problems)
    emu_adjoint* adj = nullptr;         // allocated by the first adjoint call
    // particle sharding over ranks (emu_attach_comm): every deposit is summed
    // over the ranks before a stage reads it
    void* comm = nullptr;               // ncclComm_t
    void* local = nullptr;              // or a LocalGroup: ranks that are contexts of one process
    int rank = 0, nranks = 1;
    double* red_scratch = nullptr;      // device scalars for load-time reductions
    double* stats = nullptr;            // per-block record statistics of a load (device)
    double* stats_host = nullptr;       // and their pinned host copy
    bool adj_valid = false;             // a recorded run matches the slot order
    std::string err;
};

namespace emu_ctx {

// Device-wide CUDA calls (allocation and release of device and pinned
// memory) fail while another thread's stream is being captured into a graph,
// and invalidate that capture. Contexts may be driven from several host
// threads at once, so these calls and the graph captures hold one
// process-wide (recursive) lock.
std::recursive_mutex& device_lock();
template <class T>
cudaError_t dev_malloc(T** p, size_t bytes)
{
    std::lock_guard<std::recursive_mutex> g(device_lock());
    return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}
template <class T>
cudaError_t host_malloc(T** p, size_t bytes)
{
    std::lock_guard<std::recursive_mutex> g(device_lock());
    return cudaMallocHost(reinterpret_cast<void**>(p), bytes);
}
inline cudaError_t dev_free(void* p)
{
    std::lock_guard<std::recursive_mutex> g(device_lock());
    return cudaFree(p);
}
inline cudaError_t host_free(void* p)
{
    std::lock_guard<std::recursive_mutex> g(device_lock());
    return cudaFreeHost(p);
}

// record msg on the context (or the thread's host error when c is null)
int fail(emu_context* c, int code, const std::string& msg);
// EMU_ERR_CUDA with what + the pending launch error, if any
int check_launch(emu_context* ctx, const char* what);
// one device-resident step of the fused RK4 loop (cooperative kernel or
// graph), without the periodic re-sort; dt comes from the device control.
// last_stage_deposit = false leaves the deposit of the new state to a
// re-sort with deposit that the caller makes next.
int step_device(emu_context* ctx, bool last_stage_deposit = true);
// sum a deposited mesh (FP64, or int64 for the mixed path) over the ranks of
// the attached communicator, enqueued on st; no-op without one
int reduce_mesh(emu_context* ctx, void* mesh, bool int64, cudaStream_t st);
// sum the ranks' full int64 meshes src into dst (ncells * 8 NF^2 values)
int reduce_mesh_into(emu_context* ctx, const long long* src, long long* dst, cudaStream_t st);
}  // namespace emu_ctx
// sum (op 0) or max (op 1) of n <= 8 host scalars over the ranks (synchronous)
int emu_ctx_reduce_scalars(emu_context* ctx, double* v, int n, int op);
// destroys the attached communicator (emu_destroy, after the graphs)
void emu_ctx_comm_free(emu_context* ctx);
namespace emu_ctx {
// device capacity for n particles (particle arrays and the record staging)
int reserve(emu_context* ctx, int64_t n);
// finish a load whose n records are in ctx->aos: global scalars (Vvac_max
// from this rank's smallest pupt, mixed fixed-point scales from its weight
// sums and maxima), cell sort, pack, initial deposit
int load_from_aos(emu_context* ctx, int64_t n, double pupt_min, const double tot[2], const double mx[2]);
// statistics of the n records in ctx->aos, reduced on the device per block
// and over the blocks in order on the host (synchronous): smallest pupt,
// sums and maxima of |N| and |Nbar|
int record_stats(emu_context* ctx, int64_t n, double& pupt_min, double tot[2], double mx[2]);
// re-sort the particles by cell now; when perm is not null it receives the
// gather permutation (new slot i holds old slot perm[i])
int resort_now(emu_context* ctx, unsigned* perm);
// the cell-sort gather permutation of the particles of S (positions, count
// and capacity of S; the context's sort buffers): ctx->idx2, new slot i
// holds slot idx2[i]
int sort_state_perm(emu_context* ctx, const DevState& S);
// frees the adjoint arrays (emu_destroy)
void adjoint_free(emu_context* ctx);

}  // namespace emu_ctx

#define CU(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return emu_ctx::fail(ctx, EMU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
