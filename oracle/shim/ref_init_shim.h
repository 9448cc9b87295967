/*
 * Stand-ins for the AMReX names that the helper functions at the top of the
 * reference's Source/FlavoredNeutrinoContainerInit.cpp use (uniform_sphere_xyz,
 * minerbo_Z, minerbo_closure and their neighbours), so that those lines
 * compile unmodified inside oracle/_ref/ref_init_tu.cpp, which
 * oracle/build_oracle.py assembles from the reference file where it lies.
 * TEST INFRASTRUCTURE ONLY.
 */
#ifndef EMU_ORACLE_SHIM_REF_INIT_H_
#define EMU_ORACLE_SHIM_REF_INIT_H_
#include <array>
#include <cassert>
#include <cmath>
#include <cstdio>
#include <ostream>
#include <stdexcept>
#include <streambuf>
#include <vector>

#define AMREX_GPU_HOST_DEVICE
#define AMREX_ASSERT(x) assert(x)

namespace amrex {
using Real = double;
template <class T, int N>
using GpuArray = std::array<T, N>;
namespace Gpu {
template <class T>
using ManagedVector = std::vector<T>;
}
using IntVect = std::array<int, 3>;
namespace MathConst {
constexpr Real pi = 3.14159265358979323846;
}
// the helpers' random draws are not called by the oracle's wrappers
inline Real Random() { return 0.5; }
struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};
inline std::ostream& Print()
{
    static NullBuf b;
    static std::ostream s(&b);
    return s;
}
[[noreturn]] inline void Error(const char* m) { throw std::runtime_error(m); }
}  // namespace amrex
#endif
