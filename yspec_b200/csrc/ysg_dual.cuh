// ysg_dual.cuh -- first-order dual numbers for the tangent-linear solver.
//
// A dual value carries a value and its derivative along one direction of
// the earth model: (v, d) stands for v + d eps with eps^2 = 0.  Every
// operation returns the exact derivative of the operation the value part
// performs, so a solver compiled with these types yields the directional
// derivative of its own discrete output (step counts, start levels and
// rescaling decisions are taken from the value part and held fixed, as they
// are piecewise constant in the model).
//
//   dreal: real dual, value and derivative doubles
//   dcplx: complex dual, value and derivative complex (cd)
//
// The value parts are computed with the same cd / double operations as the
// primal solver, so they reproduce its results to rounding.
#pragma once
#include "ysg_cplx.cuh"

namespace ysg {

struct dreal {
    double v, d;
    __host__ __device__ __forceinline__ dreal() {}
    __host__ __device__ __forceinline__ dreal(double a) : v(a), d(0.0) {}
    __host__ __device__ __forceinline__ dreal(double a, double b) : v(a), d(b) {}
    // found only through argument-dependent lookup, so sqrt(double) keeps
    // resolving to the math library's function
    friend __host__ __device__ __forceinline__ dreal sqrt(dreal a)
    {
        const double s = ::sqrt(a.v);
        return dreal(s, s > 0.0 ? a.d / (2.0 * s) : 0.0);
    }
};

struct dcplx {
    cd v, d;
    __host__ __device__ __forceinline__ dcplx() {}
    __host__ __device__ __forceinline__ dcplx(cd a) : v(a), d{0.0, 0.0} {}
    __host__ __device__ __forceinline__ dcplx(double a) : v{a, 0.0}, d{0.0, 0.0} {}
    __host__ __device__ __forceinline__ dcplx(dreal a) : v{a.v, 0.0}, d{a.d, 0.0} {}
    __host__ __device__ __forceinline__ dcplx(cd a, cd b) : v(a), d(b) {}
};

#define YSG_D __host__ __device__ __forceinline__

// ---- real duals ----
YSG_D dreal operator-(dreal a) { return dreal(-a.v, -a.d); }
YSG_D dreal operator+(dreal a, dreal b) { return dreal(a.v + b.v, a.d + b.d); }
YSG_D dreal operator-(dreal a, dreal b) { return dreal(a.v - b.v, a.d - b.d); }
YSG_D dreal operator*(dreal a, dreal b) { return dreal(a.v * b.v, a.d * b.v + a.v * b.d); }
YSG_D dreal operator/(dreal a, dreal b)
{
    const double q = a.v / b.v;
    return dreal(q, (a.d - q * b.d) / b.v);
}
YSG_D dreal operator+(dreal a, double s) { return dreal(a.v + s, a.d); }
YSG_D dreal operator+(double s, dreal a) { return dreal(s + a.v, a.d); }
YSG_D dreal operator-(dreal a, double s) { return dreal(a.v - s, a.d); }
YSG_D dreal operator-(double s, dreal a) { return dreal(s - a.v, -a.d); }
YSG_D dreal operator*(dreal a, double s) { return dreal(a.v * s, a.d * s); }
YSG_D dreal operator*(double s, dreal a) { return dreal(s * a.v, s * a.d); }
YSG_D dreal operator/(dreal a, double s) { return dreal(a.v / s, a.d / s); }
YSG_D dreal operator/(double s, dreal b)
{
    const double q = s / b.v;
    return dreal(q, -q * b.d / b.v);
}

// ---- complex duals ----
YSG_D dcplx operator-(dcplx a) { return dcplx(-a.v, -a.d); }
YSG_D dcplx operator+(dcplx a, dcplx b) { return dcplx(a.v + b.v, a.d + b.d); }
YSG_D dcplx operator-(dcplx a, dcplx b) { return dcplx(a.v - b.v, a.d - b.d); }
YSG_D dcplx operator*(dcplx a, dcplx b) { return dcplx(a.v * b.v, a.d * b.v + a.v * b.d); }
YSG_D dcplx operator/(dcplx a, dcplx b)
{
    const cd q = a.v / b.v;
    return dcplx(q, (a.d - q * b.d) / b.v);
}
YSG_D dcplx& operator+=(dcplx& a, dcplx b) { a.v += b.v; a.d += b.d; return a; }
YSG_D dcplx& operator-=(dcplx& a, dcplx b) { a.v -= b.v; a.d -= b.d; return a; }

// with a constant complex (cd)
YSG_D dcplx operator+(dcplx a, cd b) { return dcplx(a.v + b, a.d); }
YSG_D dcplx operator+(cd b, dcplx a) { return dcplx(b + a.v, a.d); }
YSG_D dcplx operator-(dcplx a, cd b) { return dcplx(a.v - b, a.d); }
YSG_D dcplx operator-(cd b, dcplx a) { return dcplx(b - a.v, -a.d); }
YSG_D dcplx operator*(dcplx a, cd b) { return dcplx(a.v * b, a.d * b); }
YSG_D dcplx operator*(cd b, dcplx a) { return dcplx(b * a.v, b * a.d); }
YSG_D dcplx operator/(dcplx a, cd b) { return dcplx(a.v / b, a.d / b); }
YSG_D dcplx operator/(cd b, dcplx a)
{
    const cd q = b / a.v;
    return dcplx(q, -(q * a.d) / a.v);
}

// with a constant real
YSG_D dcplx operator+(dcplx a, double s) { return dcplx(a.v + s, a.d); }
YSG_D dcplx operator+(double s, dcplx a) { return dcplx(s + a.v, a.d); }
YSG_D dcplx operator-(dcplx a, double s) { return dcplx(a.v - s, a.d); }
YSG_D dcplx operator-(double s, dcplx a) { return dcplx(s - a.v, -a.d); }
YSG_D dcplx operator*(dcplx a, double s) { return dcplx(a.v * s, a.d * s); }
YSG_D dcplx operator*(double s, dcplx a) { return dcplx(s * a.v, s * a.d); }
YSG_D dcplx operator/(dcplx a, double s) { return dcplx(a.v / s, a.d / s); }
YSG_D dcplx operator/(double s, dcplx a) { return cd{s, 0.0} / a; }

// with a real dual
YSG_D dcplx operator+(dcplx a, dreal b) { return dcplx(a.v + b.v, a.d + b.d); }
YSG_D dcplx operator+(dreal b, dcplx a) { return dcplx(b.v + a.v, b.d + a.d); }
YSG_D dcplx operator-(dcplx a, dreal b) { return dcplx(a.v - b.v, a.d - b.d); }
YSG_D dcplx operator-(dreal b, dcplx a) { return dcplx(b.v - a.v, b.d - a.d); }
YSG_D dcplx operator*(dcplx a, dreal b) { return dcplx(a.v * b.v, a.d * b.v + a.v * b.d); }
YSG_D dcplx operator*(dreal b, dcplx a) { return dcplx(b.v * a.v, b.d * a.v + b.v * a.d); }
YSG_D dcplx operator/(dcplx a, dreal b)
{
    const cd q = a.v / b.v;
    return dcplx(q, (a.d - b.d * q) / b.v);
}
YSG_D dcplx operator/(dreal b, dcplx a) { return dcplx(b) / a; }

// a real dual with a constant complex
YSG_D dcplx operator+(dreal b, cd a) { return dcplx(b.v + a, cd{b.d, 0.0}); }
YSG_D dcplx operator+(cd a, dreal b) { return dcplx(a + b.v, cd{b.d, 0.0}); }
YSG_D dcplx operator-(dreal b, cd a) { return dcplx(b.v - a, cd{b.d, 0.0}); }
YSG_D dcplx operator-(cd a, dreal b) { return dcplx(a - b.v, cd{-b.d, 0.0}); }
YSG_D dcplx operator*(dreal b, cd a) { return dcplx(b.v * a, b.d * a); }
YSG_D dcplx operator*(cd a, dreal b) { return dcplx(a * b.v, a * b.d); }
YSG_D dcplx operator/(cd a, dreal b)
{
    const cd q = a / b.v;
    return dcplx(q, -(b.d * q) / b.v);
}
YSG_D dcplx operator/(dreal b, cd a) { return dcplx(b.v / a, b.d / a); }

YSG_D dcplx conj(dcplx a) { return dcplx(conj(a.v), conj(a.d)); }
YSG_D dcplx imul(dcplx a) { return dcplx(imul(a.v), imul(a.d)); }
YSG_D dcplx mk(dreal re) { return dcplx(re); }
// |a|^2 = a conj(a): derivative 2 Re(conj(a) da)
YSG_D dreal norm2(dcplx a)
{
    return dreal(a.v.x * a.v.x + a.v.y * a.v.y, 2.0 * (a.v.x * a.d.x + a.v.y * a.d.y));
}
YSG_D dreal cabs(dcplx a)
{
    const double m = cabs(a.v);
    return dreal(m, m > 0.0 ? (a.v.x * a.d.x + a.v.y * a.d.y) / m : 0.0);
}
// principal square root: d sqrt(z) = dz / (2 sqrt(z))
YSG_D dcplx csqrt(dcplx z)
{
    const cd s = csqrt(z.v);
    const bool zero = s.x == 0.0 && s.y == 0.0;
    return dcplx(s, zero ? cd{0.0, 0.0} : z.d / (2.0 * s));
}

#undef YSG_D

// value part, for decisions taken on the primal value
__host__ __device__ __forceinline__ double val(double a) { return a; }
__host__ __device__ __forceinline__ double val(dreal a) { return a.v; }
__host__ __device__ __forceinline__ cd val(cd a) { return a; }
__host__ __device__ __forceinline__ cd val(dcplx a) { return a.v; }

}  // namespace ysg
