/*
 * Minimal stand-in for the AMReX header that the reference's
 * Source/ParticleInterpolator.H and Source/Constants.H include, so those two
 * files compile unmodified, where they lie, inside the oracle harness
 * (oracle/ref_harness.cpp).  TEST INFRASTRUCTURE ONLY.
 */
#ifndef EMU_ORACLE_SHIM_AMREX_REAL_H_
#define EMU_ORACLE_SHIM_AMREX_REAL_H_
#include <cassert>
namespace amrex {
using Real = double;
using ParticleReal = double;
inline namespace literals {
constexpr Real operator""_rt(long double x) { return Real(x); }
}
}  // namespace amrex
#define AMREX_GPU_DEVICE
#define AMREX_GPU_HOST_DEVICE
#define AMREX_FORCE_INLINE inline
#define AMREX_ASSERT(x) assert(x)
#endif
