// emu_noalloc.cu -- deposit_to_mesh for callers that must not allocate
// device memory.
//
// Some callers cannot call cudaMalloc at the point where they need a
// deposit: code running while a CUDA stream is being captured into a graph
// (allocation calls are not capturable), drivers that hand the GPU a fixed
// memory pool up front and forbid further allocation, or real-time loops
// that must not hit the allocator.  emu_deposit_noalloc serves them: the
// caller passes device pointers to the particle records and to the output
// mesh, and the only scratch the deposit needs (the cell-major FP64
// accumulation mesh) is a fixed-size array in this file, compiled into the
// library.  Every GPU that loads the library holds that array until the
// process exits.
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

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
double* g_scratch_addr[kMaxDevices] = {};   // device address of the array, per device

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

// deposit straight from device particle records (rows of 3 + nattribs)
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
                                        [](double a, int) -> double { return a; });
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

template <int NF>
void na_launch(const DevParams& P, const double* recs, long long n, double* acc, double* out, const emu_params& p,
               cudaStream_t st)
{
    const long long ne = P.ncells * 8 * NF * NF;
    k_na_zero<<<148 * 4, 256, 0, st>>>(acc, ne);
    EMU_W_DISPATCH(P, {
        constexpr int bytes = tile_smem_bytes<NF, SW<WXv, WYv, WZv>, double>();
        smem_optin(k_na_deposit<NF, WXv, WYv, WZv>, bytes);
        k_na_deposit<NF, WXv, WYv, WZv><<<grid_for(n), kBlock, bytes, st>>>(P, recs, n, acc);
    });
    k_na_planes<NF><<<grid_for(ne), kBlock, 0, st>>>(P, acc, out, p.rho_in, p.T_in, p.Ye_in);
}

// Once per device, with that device current: the device address of the
// scratch array.  Host code must not use the array's name as a pointer.
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
    if (!g_scratch_addr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) {
            g_noalloc_err = std::string("emu_deposit_noalloc: cudaGetSymbolAddress failed: ") +
                            cudaGetErrorString(e);
            return EMU_ERR_CUDA;
        }
        g_scratch_addr[dev] = static_cast<double*>(ptr);
    }
    *out = g_scratch_addr[dev];
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
    if (nf == 2) na_launch<2>(P, d_records, n, acc, d_mesh_out, *p, st);
    else na_launch<3>(P, d_records, n, acc, d_mesh_out, *p, st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_noalloc_err = std::string("emu_deposit_noalloc: launch failed: ") + cudaGetErrorString(e);
        return EMU_ERR_CUDA;
    }
    return EMU_OK;
}
