// host_shim.h -- compile the device solver headers (yspec_b200/csrc/*.cuh)
// as plain host C++ for the CPU checks of tests/test_adjoint_host.py:
// device qualifiers become nothing, the explicitly rounded device
// intrinsics become the plain operations, read-only loads plain loads.
#pragma once
#include <algorithm>
#include <cmath>
#include <cuda_runtime.h>
#undef __device__
#undef __forceinline__
#undef __global__
#undef __noinline__
#define __device__
#define __forceinline__ inline
#define __noinline__
inline double __dmul_rn(double a, double b) { return a * b; }
inline double __dadd_rn(double a, double b) { return a + b; }
inline double __dsub_rn(double a, double b) { return a - b; }
template <class T> inline T __ldg(const T* p) { return *p; }
inline void sincos(double x, double* s, double* c)
{
    *s = std::sin(x);
    *c = std::cos(x);
}
using std::max;
using std::min;
