// emu_k_misc.cu -- launchers of the small kernels and the flavor-count
// dispatch of the large ones (whose instantiations live in
// emu_k_fp64_<nf>.cu and emu_k_mixed_<nf>.cu so that they compile in
// parallel).
#include "emu_kernels_impl.cuh"

namespace emu {

#define EMU_EXTERN(NF)                                                                                          \
    extern template void launch_rk4_stage_t<NF>(const DevParams&, const DevState&, int, const double*, double*,  \
                                                double*, long long, StepCtl*, int, cudaStream_t);                \
    extern template void launch_deposit_t<NF>(const DevParams&, const DevState&, const double*, double*,         \
                                              cudaStream_t);                                                     \
    extern template void launch_rhs_t<NF>(const DevParams&, const DevState&, const double*, const double*,       \
                                          double*, cudaStream_t);                                                \
    extern template void launch_rk4_stage_mixed_t<NF>(const DevParams&, const DevState&, int, const float*,      \
                                                      long long*, const long long*, long long*, StepCtl*, int,   \
                                                      cudaStream_t, const DevState*, const unsigned*, unsigned*, \
                                                      unsigned*);                                                \
    extern template void launch_deposit_comb_t<NF>(const DevParams&, const DevState&, long long*, cudaStream_t);  \
    extern template void launch_deposit_q_t<NF>(const DevParams&, const DevState&, const double*, long long*,    \
                                                cudaStream_t);                                                   \
    extern template bool coop_step_fits_t<NF>(const DevParams&, long long);                                      \
    extern template void launch_gather_deposit_t<NF>(bool, const DevParams&, const DevState&, const DevState&,    \
                                                     const unsigned*, double*, long long*, cudaStream_t);        \
    extern template cudaError_t launch_rk4_step_coop_t<NF>(const DevParams&, const DevState&, double* const*,    \
                                                           long long, StepCtl*, int, cudaStream_t);
EMU_EXTERN(2)
EMU_EXTERN(3)

#define EMU_NF_DISPATCH(nf, KERNEL_CALL) \
    do {                                 \
        if ((nf) == 2) {                 \
            constexpr int NFv = 2;       \
            KERNEL_CALL;                 \
        } else {                         \
            constexpr int NFv = 3;       \
            KERNEL_CALL;                 \
        }                                \
    } while (0)


void launch_pack(int nf, const DevParams& P, const double* aos, const unsigned* perm, long long n, DevState S,
                 cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_pack<NFv><<<grid_for(n), kBlock, 0, st>>>(P, aos, perm, n, S)));
}

void launch_unpack(int nf, const DevState& S, double* aos, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_unpack<NFv><<<grid_for(S.n), kBlock, 0, st>>>(S, aos)));
}

void launch_unpack_rhs(int nf, const DevState& S, const double* K, double* aos, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_unpack_rhs<NFv><<<grid_for(S.n), kBlock, 0, st>>>(S, K, aos)));
}

void launch_cell_keys(const DevParams& P, const double* aos, int nreal, long long n, unsigned* keys, unsigned* idx,
                      cudaStream_t st)
{
    k_cell_keys_aos<<<grid_for(n), kBlock, 0, st>>>(P, aos, nreal, n, keys, idx);
}

void launch_state_keys(const DevParams& P, const DevState& S, unsigned* keys, unsigned* idx, cudaStream_t st)
{
    k_cell_keys_soa<<<grid_for(S.n), kBlock, 0, st>>>(P, S, keys, idx);
}

void launch_gather_state(int nf, bool mixed, const DevParams& P, const DevState& src, const DevState& dst,
                         const unsigned* perm, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_gather_state<NFv><<<grid_for(src.n), kBlock, 0, st>>>(src, dst, perm, mixed ? 1 : 0)));
}

void launch_gather_deposit(int nf, bool mixed, const DevParams& P, const DevState& src, const DevState& dst,
                           const unsigned* perm, double* mesh, long long* qmesh, cudaStream_t st)
{
    if (nf == 2) launch_gather_deposit_t<2>(mixed, P, src, dst, perm, mesh, qmesh, st);
    else launch_gather_deposit_t<3>(mixed, P, src, dst, perm, mesh, qmesh, st);
}

void launch_deposit(int nf, const DevParams& P, const DevState& S, const double* f, double* mesh, cudaStream_t st)
{
    if (nf == 2) launch_deposit_t<2>(P, S, f, mesh, st); else launch_deposit_t<3>(P, S, f, mesh, st);
}

void launch_deposit_q(int nf, const DevParams& P, const DevState& S, const double* f, long long* mesh,
                      cudaStream_t st)
{
    if (nf == 2) launch_deposit_q_t<2>(P, S, f, mesh, st); else launch_deposit_q_t<3>(P, S, f, mesh, st);
}

void launch_rhs(int nf, const DevParams& P, const DevState& S, const double* f, const double* mesh, double* K,
                cudaStream_t st)
{
    if (nf == 2) launch_rhs_t<2>(P, S, f, mesh, K, st); else launch_rhs_t<3>(P, S, f, mesh, K, st);
}

void launch_stage_state(int nf, const DevState& S, const double* K, int nterms, const double* coef, double* out,
                        cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_stage_state<NFv><<<grid_for(S.n), kBlock, 0, st>>>(
                            S, K, nterms, coef[0], nterms > 1 ? coef[1] : 0.0, nterms > 2 ? coef[2] : 0.0, out)));
}

void launch_combine(int nf, const DevParams& P, const DevState& S, const double* K, int ns, const double* b,
                    StepCtl* ctl, cudaStream_t st)
{
    double w[4] = {0, 0, 0, 0};
    for (int i = 0; i < ns && i < 4; i++) w[i] = b[i];
    EMU_NF_DISPATCH(nf, (k_combine<NFv><<<grid_for(S.n), kBlock, 0, st>>>(P, S, K, ns, w[0], w[1], w[2], w[3], ctl)));
}

void launch_rk4_stage(int nf, const DevParams& P, const DevState& S, int s, const double* mesh_in, double* mesh_out,
                      double* mesh_zero, long long nzero, StepCtl* ctl, int dt_mode, cudaStream_t st)
{
    if (nf == 2) launch_rk4_stage_t<2>(P, S, s, mesh_in, mesh_out, mesh_zero, nzero, ctl, dt_mode, st);
    else launch_rk4_stage_t<3>(P, S, s, mesh_in, mesh_out, mesh_zero, nzero, ctl, dt_mode, st);
}

bool coop_step_fits(int nf, const DevParams& P, long long n)
{
    return nf == 2 ? coop_step_fits_t<2>(P, n) : coop_step_fits_t<3>(P, n);
}

cudaError_t launch_rk4_step_coop(int nf, const DevParams& P, const DevState& S, double* const mesh[4], long long nmesh,
                                 StepCtl* ctl, int dt_mode, cudaStream_t st)
{
    return nf == 2 ? launch_rk4_step_coop_t<2>(P, S, mesh, nmesh, ctl, dt_mode, st)
                   : launch_rk4_step_coop_t<3>(P, S, mesh, nmesh, ctl, dt_mode, st);
}

void launch_rk4_stage_mixed(int nf, const DevParams& P, const DevState& S, int s, const float* gmesh,
                            long long* qmesh_out, const long long* qmesh_dt, long long* qmesh_m4, StepCtl* ctl,
                            int dt_mode, cudaStream_t st, const DevState* D, const unsigned* inv, unsigned* kout,
                            unsigned* iout)
{
    if (nf == 2)
        launch_rk4_stage_mixed_t<2>(P, S, s, gmesh, qmesh_out, qmesh_dt, qmesh_m4, ctl, dt_mode, st, D, inv, kout, iout);
    else
        launch_rk4_stage_mixed_t<3>(P, S, s, gmesh, qmesh_out, qmesh_dt, qmesh_m4, ctl, dt_mode, st, D, inv, kout, iout);
}

void launch_sc_keys(const DevParams& P, const DevState& S, const StepCtl* ctl, unsigned* keys, unsigned* idx,
                    cudaStream_t st)
{
    k_sc_keys<<<grid_for(S.n), kBlock, 0, st>>>(P, S, ctl, keys, idx);
}

void launch_deposit_comb(int nf, const DevParams& P, const DevState& S, long long* qmesh, cudaStream_t st)
{
    if (nf == 2) launch_deposit_comb_t<2>(P, S, qmesh, st);
    else launch_deposit_comb_t<3>(P, S, qmesh, st);
}


void launch_sc_invert(const unsigned* perm, unsigned* inv, long long n, cudaStream_t st)
{
    k_sc_invert<<<grid_for(n), kBlock, 0, st>>>(perm, inv, n);
}

static unsigned reduce_grid(long long ncells)
{
    long long g = (ncells + kBlock - 1) / kBlock;
    if (g > 1184) g = 1184;
    if (g < 1) g = 1;
    return (unsigned)g;
}

void launch_finalize_mixed(int nf, const DevParams& P, const long long* qread, long long* qzero, float* gmesh,
                           StepCtl* ctl, bool comb, long long* qzero_m4, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (launch_pdl(k_finalize_mixed<NFv>, reduce_grid(P.ncells * Comb<NFv>::NG), kBlock, 0, st, P,
                                    qread, qzero, gmesh, ctl, comb ? 1 : 0, qzero_m4)));
}

void launch_dt(int nf, const DevParams& P, const double* mesh, StepCtl* ctl, int mode, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_dt<NFv, double><<<reduce_grid(P.ncells), kBlock, 0, st>>>(P, mesh, ctl, mode, nullptr)));
}

void launch_full_to_comb(int nf, const DevParams& P, const long long* qfull, long long* qcomb, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_full_to_comb<NFv><<<reduce_grid(P.ncells * 4), kBlock, 0, st>>>(P, qfull,
                                                                                                        qcomb)));
}

void launch_dt_q(int nf, const DevParams& P, const long long* mesh, const long long* diag, StepCtl* ctl, int mode,
                 cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_dt<NFv, long long><<<reduce_grid(P.ncells), kBlock, 0, st>>>(P, mesh, ctl, mode, diag)));
}

void launch_renorm(int nf, const DevParams& P, const DevState& S, StepCtl* ctl, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_renorm<NFv><<<grid_for(S.n), kBlock, 0, st>>>(P, S, ctl)));
}

void launch_mesh_out(int nf, const DevParams& P, const double* mesh, double* out, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_mesh_out<NFv><<<grid_for(P.ncells * 8 * NFv * NFv), kBlock, 0, st>>>(P, mesh, out)));
}

void launch_mesh_out_q(int nf, const DevParams& P, const long long* mesh, double* out, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_mesh_out_q<NFv><<<grid_for(P.ncells * 8 * NFv * NFv), kBlock, 0, st>>>(P, mesh, out)));
}

void launch_q_to_f64(int nf, const DevParams& P, const long long* mesh, double* out, cudaStream_t st)
{
    EMU_NF_DISPATCH(nf, (k_q_to_f64<NFv><<<grid_for(P.ncells * 8 * NFv * NFv), kBlock, 0, st>>>(P, mesh, out)));
}

void launch_ctl_hist(StepCtl* ctl, double* hist, cudaStream_t st) { k_ctl_hist<<<1, 1, 0, st>>>(ctl, hist); }

void launch_ctl_set(StepCtl* ctl, double dt, double t, double end_time, int max_step, int reset_status,
                    cudaStream_t st)
{
    k_ctl_set<<<1, 1, 0, st>>>(ctl, dt, t, end_time, max_step, reset_status);
}

void launch_ctl_m4(StepCtl* ctl, int nsteps, cudaStream_t st)
{
    k_ctl_m4<<<1, 1, 0, st>>>(ctl, nsteps);
}

void launch_mixed_shadow(int nf, const DevState& S, cudaStream_t st)
{
    k_mixed_shadow<<<grid_for(S.n), kBlock, 0, st>>>(S, 2 * nf * nf);
}

void launch_flush(double* buf, long long n, cudaStream_t st)
{
    k_flush<<<148 * 8, 256, 0, st>>>(buf, n);
}

}  // namespace emu
