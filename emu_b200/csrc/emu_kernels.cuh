// emu_kernels.cuh -- device data layout and the host-side launchers of the
// evolution kernels (implemented in emu_kernels_impl.cuh, instantiated in
// emu_k_fp64_<nf>.cu, emu_k_mixed_<nf>.cu and emu_k_misc.cu).
//
// HBM layout (structure of arrays, particles cell-sorted, stride = cap):
//   pos[3], time, pup[4], Nn[2] (N, Nbar), Ll[2] (L, Lbar)        FP64
//   vhat[3] = pup/pupt, vscale = c^4/(2 pupt)                       FP64
//   f0[2*NF*NF]  state at the start of the step (nu then nubar)    FP64
//   fs, acc      fused RK4: stage state and running RK sum         FP64
//   kgen         unfused integrators: one RHS per stage            FP64
//   k32, ksum32  mixed RK4: previous stage RHS and weighted sum    FP32
//   f032         mixed, 1D TSC: f0 rounded to FP32 (all stages 1-3 read)  FP32
//   vhat32[3], N32[2]  mixed copies of the static fields           FP32
//   id           load index of each particle                       int64
// Meshes are cell-major: mesh[cell*ND + q] with q in GIdx order minus 3
// (ND = 8*NF*NF), FP64 (plain) or int64 fixed point (mixed).  The mixed
// path's int64 meshes are followed by kDiagSlots per cell (the diagonal
// N_ii, Nbar_ii that compute_dt reads, at mesh + ncells*ND).
#pragma once

#include "emu_device.cuh"

struct emu_params;

namespace emu {

// kernel parameters from the run parameters (emu_capi.cu)
void make_devparams(const emu_params& p, DevParams& P);

// Mixed stages 1-3 read the step-start state only rounded to FP32.  With 1D
// TSC stencils (the 1,1,3 stencil widths) they read an FP32 copy of it, kept
// by stage 4: half the bytes.  In 3D, where stage 4 stores a re-sorted state
// every step, the copy's scattered stores cost more than the reads save
// (C5: 26.30 -> 27.19 ms per step; C3: 0.275 -> 0.266 ms).
template <int WX, int WY, int WZ>
__host__ __device__ constexpr bool mixed_f0_copy_w()
{
    return WX == 1 && WY == 1 && WZ == 3;
}
inline bool mixed_f0_copy(const DevParams& P)
{
    return P.w[0] == 1 && P.w[1] == 1 && P.w[2] == 3;
}

// The keys of the re-sort made by stage 4 (the stencil keys after the step)
// are stored by stage 3 of that step, except with 1D TSC stencils (a
// re-sort every 16 steps), where a kernel of their own computes them before
// the sort and stage 3 keeps no code for them (C5: 26.30 -> 25.89 ms per
// step with the fused diagonal slots; C3 0.2655 -> 0.2692 ms when its stage
// 3 held the key path too).
template <int WX, int WY, int WZ>
__host__ __device__ constexpr bool sc_keys_in_stage3_w()
{
    return !(WX == 1 && WY == 1 && WZ == 3);
}
inline bool sc_keys_in_stage3(const DevParams& P)
{
    return !(P.w[0] == 1 && P.w[1] == 1 && P.w[2] == 3);
}

struct DevState {
    long long n = 0, cap = 0;
    double* pos[3] = {};
    double* time = nullptr;
    double* pup[4] = {};
    double* Nn[2] = {};
    double* Ll[2] = {};
    double* vhat[3] = {};
    double* vscale = nullptr;
    double* f0 = nullptr;
    double* fs = nullptr;
    double* acc = nullptr;
    double* kgen = nullptr;        // [ns][2NH][cap]
    float* k32 = nullptr;
    float* ksum32 = nullptr;
    float* vhat32[3] = {};
    float* N32[2] = {};
    // mixed path with 1D TSC stencils (mixed_f0_copy): f0 rounded to FP32,
    // kept with f0 by every kernel that writes f0 (stages 1-3 form their FP32
    // stage state from it); null otherwise
    float* f032 = nullptr;
    long long* id = nullptr;
    // slot of each particle in its CTA's key-ranked deposit order (a
    // permutation of each 128-particle tile's active slots): the rank the
    // last stage 4 computed for the new positions, which stages 1-3 of the
    // next step deposit at; identity after a load or a re-sort
    int* rslot = nullptr;
};

// Device-side step control: the timestep, time and error state live on the
// device so that whole runs proceed without host round trips.
struct StepCtl {
    double dt;           // timestep of the step in progress
    double t;            // integrator time at the start of the step in progress
    double end_time;
    long long bad;       // smallest load index that failed Renormalize (LLONG_MAX: none)
    int status;          // OR of status bits
    int done;            // 1: no more steps; stage kernels return immediately
    int step;            // steps completed
    int max_step;        // stop once this many steps are completed
    int last;            // the step in progress is the final one (clipped to end_time)
    unsigned int blocks_done;
    unsigned long long vmax_bits[2];   // max V_adaptive, V_stupid (non-negative doubles as bits)
    unsigned int bar_count, bar_gen;   // grid barrier of the cooperative step kernel
    double* dt_hist;     // when set: dt of step k is written to dt_hist[k] (recorded runs)
    // mixed path with DevParams::m4_reduced: stage 3 deposits the stage-4
    // mesh in full (the layout get_mesh and plotfiles read) from step
    // m4_full_from on and on the final step of a run, and otherwise only the
    // combined layout stage 4 interpolates; the diagonal N_ii compute_dt
    // reads are deposited apart in both cases.  m4_full: whether the latest
    // stage-3 deposit was the full one.
    int m4_full_from;
    int m4_full;
};

enum DtMode : int { DT_QUERY = 0, DT_INIT = 1, DT_ADVANCE = 2 };

constexpr int kBlock = 128;
// default limit of a grid-barrier wait (polls of 64 ns sleeps, ~0.3 s or more)
constexpr long long kBarrierSpins = 1ll << 22;

// launchers (all asynchronous on the given stream)
void launch_pack(int nf, const DevParams& P, const double* aos, const unsigned* perm, long long n, DevState S,
                 cudaStream_t st);
void launch_unpack(int nf, const DevState& S, double* aos, cudaStream_t st);
void launch_unpack_rhs(int nf, const DevState& S, const double* K, double* aos, cudaStream_t st);
void launch_cell_keys(const DevParams& P, const double* aos, int nreal, long long n, unsigned* keys,
                      unsigned* idx, cudaStream_t st);
void launch_deposit(int nf, const DevParams& P, const DevState& S, const double* f, double* mesh, cudaStream_t st);
void launch_deposit_q(int nf, const DevParams& P, const DevState& S, const double* f, long long* mesh,
                      cudaStream_t st);
void launch_rhs(int nf, const DevParams& P, const DevState& S, const double* f, const double* mesh, double* K,
                cudaStream_t st);
void launch_stage_state(int nf, const DevState& S, const double* K, int nterms, const double* coef, double* out,
                        cudaStream_t st);
void launch_combine(int nf, const DevParams& P, const DevState& S, const double* K, int ns, const double* b,
                    StepCtl* ctl, cudaStream_t st);
// dt_mode: DT_ADVANCE on stage 4 of the device-resident loop (compute_dt of
// the stage-4 mesh fused in), -1 otherwise
void launch_rk4_stage(int nf, const DevParams& P, const DevState& S, int s, const double* mesh_in,
                      double* mesh_out, double* mesh_zero, long long nzero, StepCtl* ctl, int dt_mode,
                      cudaStream_t st);
// whole FP64 RK4 step in one cooperative launch; returns false (nothing
// launched) when the grid cannot be co-resident
bool coop_step_fits(int nf, const DevParams& P, long long n);
cudaError_t launch_rk4_step_coop(int nf, const DevParams& P, const DevState& S, double* const mesh[4], long long nmesh,
                                 StepCtl* ctl, int dt_mode, cudaStream_t st);
// qmesh_m4: stage 3's target for the full stage-4 mesh (DevParams::m4_reduced)
// D, inv (stage 4 only): the stage that makes the cell re-sort following the
// step: particle p's new state and unchanged fields go to slot inv[p] of D
// (the radix sort of the keys and launch_sc_invert before it; the combined
// deposit of D, launch_deposit_comb, after it).  kout, iout (stage 3 of a
// step followed by such a re-sort): each particle's stencil key after the
// step and the identity index, which that sort orders.
void launch_rk4_stage_mixed(int nf, const DevParams& P, const DevState& S, int s, const float* gmesh,
                            long long* qmesh_out, const long long* qmesh_dt, long long* qmesh_m4, StepCtl* ctl,
                            int dt_mode, cudaStream_t st, const DevState* D = nullptr,
                            const unsigned* inv = nullptr, unsigned* kout = nullptr, unsigned* iout = nullptr);
// the combined deposit of a cell-sorted mixed state into qmesh (zeroed)
void launch_deposit_comb(int nf, const DevParams& P, const DevState& S, long long* qmesh, cudaStream_t st);
// the same keys in a kernel of their own (when !sc_keys_in_stage3)
void launch_sc_keys(const DevParams& P, const DevState& S, const StepCtl* ctl, unsigned* keys, unsigned* idx,
                    cudaStream_t st);
// inv[perm[i]] = i
void launch_sc_invert(const unsigned* perm, unsigned* inv, long long n, cudaStream_t st);
// comb: qread holds the combined layout (else the full mesh).  qzero is
// zeroed with its diagonal slots (ncells * (8 NF^2 + kDiagSlots)); qzero_m4
// (before stage 3, or nullptr) on the steps that deposit the full stage-4
// mesh there (StepCtl::m4_full_from).
void launch_finalize_mixed(int nf, const DevParams& P, const long long* qread, long long* qzero, float* gmesh,
                           StepCtl* ctl, bool comb, long long* qzero_m4, cudaStream_t st);
void launch_dt(int nf, const DevParams& P, const double* mesh, StepCtl* ctl, int mode, cudaStream_t st);
// a full int64 mesh in the combined layout (mixed path)
void launch_full_to_comb(int nf, const DevParams& P, const long long* qfull, long long* qcomb, cudaStream_t st);
// diag: the mesh's diagonal slots (DevParams::m4_reduced), or nullptr to
// read the full mesh
void launch_dt_q(int nf, const DevParams& P, const long long* mesh, const long long* diag, StepCtl* ctl, int mode,
                 cudaStream_t st);
void launch_renorm(int nf, const DevParams& P, const DevState& S, StepCtl* ctl, cudaStream_t st);
void launch_mesh_out(int nf, const DevParams& P, const double* mesh, double* out, cudaStream_t st);
void launch_mesh_out_q(int nf, const DevParams& P, const long long* mesh, double* out, cudaStream_t st);
void launch_q_to_f64(int nf, const DevParams& P, const long long* mesh, double* out, cudaStream_t st);
void launch_ctl_hist(StepCtl* ctl, double* hist, cudaStream_t st);
void launch_ctl_set(StepCtl* ctl, double dt, double t, double end_time, int max_step, int reset_status,
                    cudaStream_t st);
// the next nsteps steps: the last of them deposits the full stage-4 mesh
void launch_ctl_m4(StepCtl* ctl, int nsteps, cudaStream_t st);
void launch_mixed_shadow(int nf, const DevState& S, cudaStream_t st);
void launch_flush(double* buf, long long n, cudaStream_t st);
// cell re-sort: keys of the current positions, then gather every array
void launch_state_keys(const DevParams& P, const DevState& S, unsigned* keys, unsigned* idx, cudaStream_t st);
// re-sort gather that also deposits the gathered state into mesh (FP64) or
// qmesh (mixed int64); the target must be zeroed
void launch_gather_deposit(int nf, bool mixed, const DevParams& P, const DevState& src, const DevState& dst,
                           const unsigned* perm, double* mesh, long long* qmesh, cudaStream_t st);
void launch_gather_state(int nf, bool mixed, const DevParams& P, const DevState& src, const DevState& dst,
                         const unsigned* perm, cudaStream_t st);

}  // namespace emu
