// ysg_cplx.cuh -- FP64 complex arithmetic for the sm_100a kernels.
//
// Multiplication is the plain (ac-bd, ad+bc) form, the same one gfortran
// emits for complex(dp) without IEEE special-case handling.  Division uses
// Smith's algorithm (R. L. Smith, CACM 5(8), 1962), which is also what
// Fortran complex division rounds like.  sqrt uses the textbook stable form
// t = sqrt((|x|+|z|)/2); log uses log(hypot) + i atan2.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace ysg {

// 16-byte aligned so that a complex value moves with one 128-bit load or
// store (shared, global and local memory alike).
struct __align__(16) cd {
    double x, y;
};

__host__ __device__ __forceinline__ cd mk(double re, double im = 0.0) { return cd{re, im}; }
__host__ __device__ __forceinline__ cd operator+(cd a, cd b) { return cd{a.x + b.x, a.y + b.y}; }
__host__ __device__ __forceinline__ cd operator-(cd a, cd b) { return cd{a.x - b.x, a.y - b.y}; }
__host__ __device__ __forceinline__ cd operator-(cd a) { return cd{-a.x, -a.y}; }
__host__ __device__ __forceinline__ cd operator*(cd a, cd b)
{
    return cd{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
__host__ __device__ __forceinline__ cd operator*(double s, cd a) { return cd{s * a.x, s * a.y}; }
__host__ __device__ __forceinline__ cd operator*(cd a, double s) { return cd{a.x * s, a.y * s}; }
__host__ __device__ __forceinline__ cd operator/(cd a, double s) { return cd{a.x / s, a.y / s}; }
__host__ __device__ __forceinline__ cd operator+(cd a, double s) { return cd{a.x + s, a.y}; }
__host__ __device__ __forceinline__ cd operator+(double s, cd a) { return cd{s + a.x, a.y}; }
__host__ __device__ __forceinline__ cd operator-(cd a, double s) { return cd{a.x - s, a.y}; }
__host__ __device__ __forceinline__ cd operator-(double s, cd a) { return cd{s - a.x, -a.y}; }
__host__ __device__ __forceinline__ cd& operator+=(cd& a, cd b) { a.x += b.x; a.y += b.y; return a; }
__host__ __device__ __forceinline__ cd& operator-=(cd& a, cd b) { a.x -= b.x; a.y -= b.y; return a; }

// Smith's algorithm for a / b.
__host__ __device__ __forceinline__ cd operator/(cd a, cd b)
{
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x;
        double den = b.x + b.y * r;
        return cd{(a.x + a.y * r) / den, (a.y - a.x * r) / den};
    } else {
        double r = b.x / b.y;
        double den = b.x * r + b.y;
        return cd{(a.x * r + a.y) / den, (a.y * r - a.x) / den};
    }
}
__host__ __device__ __forceinline__ cd operator/(double s, cd b) { return cd{s, 0.0} / b; }

__host__ __device__ __forceinline__ cd conj(cd a) { return cd{a.x, -a.y}; }
__host__ __device__ __forceinline__ double cabs(cd a) { return hypot(a.x, a.y); }
__host__ __device__ __forceinline__ cd imul(cd a) { return cd{-a.y, a.x}; }   // i*a

__host__ __device__ __forceinline__ cd csqrt(cd z)
{
    if (z.x == 0.0 && z.y == 0.0) return cd{0.0, z.y};
    double t = sqrt((fabs(z.x) + hypot(z.x, z.y)) * 0.5);
    if (z.x >= 0.0) return cd{t, z.y / (2.0 * t)};
    return cd{fabs(z.y) / (2.0 * t), copysign(t, z.y)};
}

__host__ __device__ __forceinline__ cd clog(cd z) { return cd{log(hypot(z.x, z.y)), atan2(z.y, z.x)}; }

}  // namespace ysg
