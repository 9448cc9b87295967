// emu_noalloc.cu -- deposit_to_mesh for callers that must not allocate
// device memory.
//
// Some host programs cannot let a library call cudaMalloc when they need a
// deposit.  A simulation code that hands all device memory to its own pool
// allocator at start-up has nothing left for a library to allocate from,
// and an allocation behind its back would fail or fragment the pool.  A
// time-critical step loop cannot afford cudaMalloc/cudaFree either:
// cudaFree synchronises the whole device and stalls every other stream.
// emu_deposit_noalloc serves them: the caller passes device pointers to the
// particle records and to the output mesh, and the only scratch the deposit
// needs (the cell-major FP64 accumulation mesh) is a fixed-size array in
// this file, compiled into the library.  Every GPU that loads the library
// holds that array until the process exits.
#include <cuda.h>

#include <mutex>
#include <string>

#include "emu_b200.h"
#include "emu_host.h"
#include "emu_kernels_impl.cuh"

namespace emu {

namespace {

// maximum accumulation size: ncells * 8 * nflavors^2 doubles (4 MiB)
constexpr long long kNoAllocScratchDoubles = 1ll << 19;
__device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// The array's device address, looked up once per device context.  A device
// reset (or a context the caller created) loads the module anew, so the
// address is keyed by the unique id of the context that was current at the
// lookup, and looked up again when another context is current.
constexpr int kMaxDevices = 64;
struct ScratchAddr {
    unsigned long long ctx_id = 0;
    double* ptr = nullptr;
};
std::mutex g_setup_mu;
ScratchAddr g_scratch_addr[kMaxDevices];

// driver entry points (through the runtime, no link against libcuda)
using CtxGetCurrent = CUresult(CUDAAPI*)(CUcontext*);
using CtxGetId = CUresult(CUDAAPI*)(CUcontext, unsigned long long*);
CtxGetCurrent g_ctx_current = nullptr;
CtxGetId g_ctx_id = nullptr;
std::once_flag g_entry_once;

// id of the calling thread's current context; 0 when there is none or the
// driver cannot say
unsigned long long current_context_id()
{
    std::call_once(g_entry_once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_current = reinterpret_cast<CtxGetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_id = reinterpret_cast<CtxGetId>(f);
    });
    if (!g_ctx_current || !g_ctx_id) return 0;
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (g_ctx_current(&c) != CUDA_SUCCESS || !c) return 0;
    if (g_ctx_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// failures are reported through emu_last_error(NULL, ...)
struct HostError {
    HostError& operator=(const std::string& m)
    {
        emu_host::set_error(m);
        return *this;
    }
};
HostError g_noalloc_err;

__global__ void k_na_zero(double* s, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) s[i] = 0.0;
}

// deposit straight from device particle records (rows of 3 + nattribs), in
// any order: every CTA ranks its keys first, so that each stencil is one run
template <int NF, int WX, int WY, int WZ>
__global__ void __launch_bounds__(kBlock) k_na_deposit(DevParams P, const double* __restrict__ recs, long long n,
                                                       double* __restrict__ acc)
{
    using SWt = SW<WX, WY, WZ>;
    constexpr int NH = NF * NF, NS = 2 * NH, NR = 3 + 8 + 2 * (2 + NH);
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < n;
    Stencil<double> st{};
    double fN[NS] = {};
    double vx = 0, vy = 0, vz = 0;
    if (active) {
        const double* r = recs + p * NR;
        make_stencil<double>(P, r[0], r[1], r[2], st);
        const double pupt = r[3 + 7];
        vx = r[3 + 4] / pupt;
        vy = r[3 + 5] / pupt;
        vz = r[3 + 6] / pupt;
#pragma unroll
        for (int sp = 0; sp < 2; sp++) {
            const int base = 3 + 8 + sp * (2 + NH);
#pragma unroll
            for (int e = 0; e < NH; e++) fN[sp * NH + e] = r[base + 2 + e] * r[base];
        }
    }
    tile_deposit_block<NF, SWt, double>(P, acc, active, st, fN, vx, vy, vz,
                                        [](double a, int) -> double { return a; }, true);
}

template <int NF>
__global__ void k_na_planes(DevParams P, const double* __restrict__ acc, double* __restrict__ out, double rho,
                            double T, double Ye)
{
    constexpr int ND = 8 * NF * NF;
    const long long nc = P.ncells;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nc * ND) {
        const long long c = i / ND;
        const int q = (int)(i % ND);
        out[(3 + q) * nc + c] = acc[i];
    }
    if (i < nc) {
        out[i] = rho;
        out[nc + i] = T;
        out[2 * nc + i] = Ye;
    }
}

// plain launch whose error is returned (not left in the thread's last-error
// slot, where a caller's earlier failure may sit)
template <class... KArgs, class... Args>
cudaError_t na_launch_one(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t st,
                          Args&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

template <int NF>
cudaError_t na_launch(const DevParams& P, const double* recs, long long n, double* acc, double* out,
                      const emu_params& p, cudaStream_t st)
{
    const long long ne = P.ncells * 8 * NF * NF;
    cudaError_t e = na_launch_one(k_na_zero, 148 * 4, 256, 0, st, acc, ne);
    if (e != cudaSuccess) return e;
    EMU_W_DISPATCH(P, {
        constexpr int bytes = tile_smem_bytes<NF, SW<WXv, WYv, WZv>, double>();
        if (bytes > 48 * 1024)
            e = cudaFuncSetAttribute(k_na_deposit<NF, WXv, WYv, WZv>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     bytes);
        if (e == cudaSuccess)
            e = na_launch_one(k_na_deposit<NF, WXv, WYv, WZv>, grid_for(n), kBlock, bytes, st, P, recs, n, acc);
    });
    if (e != cudaSuccess) return e;
    return na_launch_one(k_na_planes<NF>, grid_for(ne), kBlock, 0, st, P, (const double*)acc, out, p.rho_in,
                         p.T_in, p.Ye_in);
}

// The device address of the scratch array in the calling thread's current
// context, with that device current: looked up (cudaGetSymbolAddress) at
// the first call in a context.  Host code must not use the array's name as
// a pointer: on the host it names a stand-in, not device memory.
int scratch_address(double** out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        g_noalloc_err = std::string("emu_deposit_noalloc: no current device: ") + cudaGetErrorString(e);
        return EMU_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        g_noalloc_err = "emu_deposit_noalloc: device index out of range";
        return EMU_ERR_LIMIT;
    }
    std::lock_guard<std::mutex> lock(g_setup_mu);
    ScratchAddr& a = g_scratch_addr[dev];
    const unsigned long long id = current_context_id();
    if (!a.ptr || id == 0 || id != a.ctx_id) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) {
            a = ScratchAddr{};
            g_noalloc_err = std::string("emu_deposit_noalloc: cudaGetSymbolAddress failed: ") +
                            cudaGetErrorString(e);
            return EMU_ERR_CUDA;
        }
        // (the lookup makes the device's primary context current when no
        // context was)
        a.ptr = static_cast<double*>(ptr);
        a.ctx_id = current_context_id();
    }
    *out = a.ptr;
    return EMU_OK;
}

}  // namespace

}  // namespace emu

extern "C" int emu_deposit_noalloc(const emu_params* p, const double* d_records, int64_t n, double* d_mesh_out,
                                   void* stream)
{
    using namespace emu;
    if (!p || !d_mesh_out || n < 0 || (n > 0 && !d_records)) {
        g_noalloc_err = "emu_deposit_noalloc: bad arguments";
        return EMU_ERR_ARG;
    }
    std::string why;
    if (!emu_host::validate(*p, why)) {
        g_noalloc_err = "emu_deposit_noalloc: " + why;
        return EMU_ERR_ARG;
    }
    const int nf = p->nflavors;
    const long long ncells = (long long)p->ncell[0] * p->ncell[1] * p->ncell[2];
    const long long need = ncells * 8 * nf * nf;
    if (need > kNoAllocScratchDoubles) {
        g_noalloc_err = "emu_deposit_noalloc: mesh of " + std::to_string(ncells) + " cells x " +
                        std::to_string(8 * nf * nf) + " components exceeds the fixed scratch of " +
                        std::to_string(kNoAllocScratchDoubles) + " doubles; use emu_deposit";
        return EMU_ERR_LIMIT;
    }
    if (n > (int64_t)INT_MAX) {
        g_noalloc_err = "emu_deposit_noalloc: more than 2^31-1 particles";
        return EMU_ERR_LIMIT;
    }
    double* acc = nullptr;
    int r = scratch_address(&acc);
    if (r) return r;
    DevParams P;
    make_devparams(*p, P);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const cudaError_t e = nf == 2 ? na_launch<2>(P, d_records, n, acc, d_mesh_out, *p, st)
                                  : na_launch<3>(P, d_records, n, acc, d_mesh_out, *p, st);
    if (e != cudaSuccess) {
        // this call's own failure: clear it from the thread's last-error
        // slot, where the runtime also recorded it
        cudaGetLastError();
        g_noalloc_err = std::string("emu_deposit_noalloc: launch failed: ") + cudaGetErrorString(e);
        return EMU_ERR_CUDA;
    }
    return EMU_OK;
}
