// emu_k_mixed_2.cu -- mixed-precision stage / deposit kernels for 2 flavors.
#include "emu_kernels_impl.cuh"

namespace emu {
template void launch_rk4_stage_mixed_t<2>(const DevParams&, const DevState&, int, const float*, long long*,
                                          const long long*, long long*, StepCtl*, int, cudaStream_t,
                                          const DevState*, const unsigned*, unsigned*, unsigned*);
template void launch_deposit_comb_t<2>(const DevParams&, const DevState&, long long*, cudaStream_t);
template void launch_deposit_q_t<2>(const DevParams&, const DevState&, const double*, long long*, cudaStream_t);
}  // namespace emu
