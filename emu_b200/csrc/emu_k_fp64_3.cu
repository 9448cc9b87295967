// emu_k_fp64_3.cu -- FP64 stage / deposit / RHS kernels for 3 flavors.
#include "emu_kernels_impl.cuh"

namespace emu {
template void launch_rk4_stage_t<3>(const DevParams&, const DevState&, int, const double*, double*, double*,
                                    long long, StepCtl*, int, cudaStream_t);
template void launch_deposit_t<3>(const DevParams&, const DevState&, const double*, double*, cudaStream_t);
template void launch_gather_deposit_t<3>(bool, const DevParams&, const DevState&, const DevState&, const unsigned*,
                                         double*, long long*, cudaStream_t);
template void launch_rhs_t<3>(const DevParams&, const DevState&, const double*, const double*, double*,
                              cudaStream_t);
template bool coop_step_fits_t<3>(const DevParams&, long long);
template cudaError_t launch_rk4_step_coop_t<3>(const DevParams&, const DevState&, double* const*, long long,
                                               StepCtl*, int, cudaStream_t);
}  // namespace emu
