// ysg_rhs_adjoint.cuh -- GENERATED by gen_rhs_adjoint.py from the right-hand
// sides of ysg_ode.cuh; do not edit.  For each system: tr() applies the
// transposed system matrix, cgrad() accumulates the gradient of k . A y
// with respect to each entry of the coefficient struct (complex, in the
// convention dL = Re(sum s_e da_e)).
#pragma once
#include "ysg_ode.cuh"

namespace ysg {
inline namespace YSG_VARIANT {

struct TorCoefBar {
    cd t, k, s;
    __device__ void zero() { t = mk(0.0); k = mk(0.0); s = mk(0.0); }
};

struct RadCoefBar {
    cd t, k, s;
    __device__ void zero() { t = mk(0.0); k = mk(0.0); s = mk(0.0); }
};

struct SolidCoefBar {
    cd t11, t12, k11, k22, s11, s12, s22, t21, t22, t31, t33, k33, s13, s23;
    __device__ void zero() { t11 = mk(0.0); t12 = mk(0.0); k11 = mk(0.0); k22 = mk(0.0); s11 = mk(0.0); s12 = mk(0.0); s22 = mk(0.0); t21 = mk(0.0); t22 = mk(0.0); t31 = mk(0.0); t33 = mk(0.0); k33 = mk(0.0); s13 = mk(0.0); s23 = mk(0.0); }
};

struct FluidCoefBar {
    cd t11, t12, k11, s11, s12, s22, t21, t22, k22;
    __device__ void zero() { t11 = mk(0.0); t12 = mk(0.0); k11 = mk(0.0); s11 = mk(0.0); s12 = mk(0.0); s22 = mk(0.0); t21 = mk(0.0); t22 = mk(0.0); k22 = mk(0.0); }
};

// TorSys: 2 components, coefficients TorCoef
struct TorSysAdj {
    static constexpr int N = 2;
    using Coef = TorCoef;
    using Bar = TorCoefBar;
    // g = A^T k
    __device__ static __forceinline__ void tr(const TorCoef& a, const cd* k, cd* g)
    {
        g[0] = a.t * k[0] + a.s * k[1];
        g[1] = a.k * k[0] + (-1.0 * a.t) * k[1];
    }
    // s.e += k . (dA/da_e) y
    __device__ static __forceinline__ void cgrad(const cd* k, const cd* y, TorCoefBar& s)
    {
        s.t += k[0] * y[0] + -1.0 * (k[1] * y[1]);
        s.k += k[0] * y[1];
        s.s += k[1] * y[0];
    }
};

// RadSys: 2 components, coefficients RadCoef
struct RadSysAdj {
    static constexpr int N = 2;
    using Coef = RadCoef;
    using Bar = RadCoefBar;
    // g = A^T k
    __device__ static __forceinline__ void tr(const RadCoef& a, const cd* k, cd* g)
    {
        g[0] = a.t * k[0] + a.s * k[1];
        g[1] = a.k * k[0] + (-1.0 * a.t) * k[1];
    }
    // s.e += k . (dA/da_e) y
    __device__ static __forceinline__ void cgrad(const cd* k, const cd* y, RadCoefBar& s)
    {
        s.t += k[0] * y[0] + -1.0 * (k[1] * y[1]);
        s.k += k[0] * y[1];
        s.s += k[1] * y[0];
    }
};

// MinorSolidG: 14 components, coefficients SolidCoef
struct MinorSolidGAdj {
    static constexpr int N = 14;
    using Coef = SolidCoef;
    using Bar = SolidCoefBar;
    // g = A^T k
    __device__ static __forceinline__ void tr(const SolidCoef& a, const cd* k, cd* g)
    {
        g[0] = a.t11 * k[0] + a.t22 * k[0] + a.t33 * k[0] + a.s13 * k[1] + a.s23 * k[2] + (-1.0 * a.s12) * k[4] + (-1.0 * a.s22) * k[5] + a.s11 * k[9];
        g[1] = a.t22 * k[1] + (-1.0 * a.t12) * k[2] + (-1.0 * a.s22) * k[6] + (-1.0 * a.s23) * k[7] + (-2.0 * a.t31) * k[9] + a.s12 * k[10] + (2.0 * a.s13) * k[11];
        g[2] = (-1.0 * a.t21) * k[1] + a.t11 * k[2] + a.t31 * k[4] + a.s12 * k[6] + (-1.0 * a.s13) * k[7] + (-2.0 * a.s23) * k[8] + (-1.0 * a.s11) * k[10];
        g[3] = a.k33 * k[0] + (-1.0 * a.t31) * k[1] + a.t11 * k[3] + a.t22 * k[3] + (-1.0 * a.t33) * k[3] + a.s12 * k[7] + a.s22 * k[8] + (-1.0 * a.s11) * k[11];
        g[4] = a.t33 * k[4] + (-2.0 * a.t12) * k[5] + (-1.0 * a.s23) * k[6] + (2.0 * a.t21) * k[9] + (-1.0 * a.s13) * k[10] + (2.0 * a.s12) * k[12];
        g[5] = (-1.0 * a.k22) * k[0] + (-1.0 * a.t21) * k[4] + a.t11 * k[5] + (-1.0 * a.t22) * k[5] + a.t33 * k[5] + a.s13 * k[6] + (-1.0 * a.s11) * k[12];
        g[6] = (-1.0 * a.k22) * k[1] + (-1.0 * a.t22) * k[6] + a.t21 * k[10] + (2.0 * a.t31) * k[12] + (2.0 * a.s13) * k[13];
        g[7] = (-1.0 * a.k33) * k[4] + (-1.0 * a.t33) * k[7] + (-2.0 * a.t12) * k[8] + (-1.0 * a.t31) * k[10] + (2.0 * a.t21) * k[11] + (-2.0 * a.s12) * k[13];
        g[8] = a.k22 * k[3] + (-1.0 * a.k33) * k[5] + a.t31 * k[6] + (-1.0 * a.t21) * k[7] + (-1.0 * a.t22) * k[8] + (-1.0 * a.t33) * k[8] + a.t11 * k[8] + a.s11 * k[13];
        g[9] = a.k11 * k[0] + a.t12 * k[4] + a.t22 * k[9] + a.t33 * k[9] + (-1.0 * a.t11) * k[9] + (-1.0 * a.s23) * k[10] + a.s22 * k[12];
        g[10] = (-1.0 * a.k11) * k[2] + a.t12 * k[6] + (-1.0 * a.t11) * k[10] + (2.0 * a.s23) * k[13];
        g[11] = (-1.0 * a.k11) * k[3] + a.t12 * k[7] + (-1.0 * a.k33) * k[9] + (-1.0 * a.t11) * k[11] + a.t22 * k[11] + (-1.0 * a.t33) * k[11] + (-1.0 * a.s22) * k[13];
        g[12] = (-1.0 * a.k11) * k[5] + a.k22 * k[9] + (-1.0 * a.t11) * k[12] + (-1.0 * a.t22) * k[12] + a.t33 * k[12];
        g[13] = a.k11 * k[8] + (-1.0 * a.k22) * k[11] + a.k33 * k[12] + (-1.0 * a.t11) * k[13] + (-1.0 * a.t22) * k[13] + (-1.0 * a.t33) * k[13];
    }
    // s.e += k . (dA/da_e) y
    __device__ static __forceinline__ void cgrad(const cd* k, const cd* y, SolidCoefBar& s)
    {
        s.t11 += k[0] * y[0] + k[2] * y[2] + k[3] * y[3] + k[5] * y[5] + k[8] * y[8] + -1.0 * (k[9] * y[9]) + -1.0 * (k[10] * y[10]) + -1.0 * (k[11] * y[11]) + -1.0 * (k[12] * y[12]) + -1.0 * (k[13] * y[13]);
        s.t12 += -1.0 * (k[2] * y[1]) + k[4] * y[9] + -2.0 * (k[5] * y[4]) + k[6] * y[10] + k[7] * y[11] + -2.0 * (k[8] * y[7]);
        s.k11 += k[0] * y[9] + -1.0 * (k[2] * y[10]) + -1.0 * (k[3] * y[11]) + -1.0 * (k[5] * y[12]) + k[8] * y[13];
        s.k22 += -1.0 * (k[0] * y[5]) + -1.0 * (k[1] * y[6]) + k[3] * y[8] + k[9] * y[12] + -1.0 * (k[11] * y[13]);
        s.s11 += k[9] * y[0] + -1.0 * (k[10] * y[2]) + -1.0 * (k[11] * y[3]) + -1.0 * (k[12] * y[5]) + k[13] * y[8];
        s.s12 += -1.0 * (k[4] * y[0]) + k[6] * y[2] + k[7] * y[3] + k[10] * y[1] + 2.0 * (k[12] * y[4]) + -2.0 * (k[13] * y[7]);
        s.s22 += -1.0 * (k[5] * y[0]) + -1.0 * (k[6] * y[1]) + k[8] * y[3] + k[12] * y[9] + -1.0 * (k[13] * y[11]);
        s.t21 += -1.0 * (k[1] * y[2]) + -1.0 * (k[4] * y[5]) + -1.0 * (k[7] * y[8]) + 2.0 * (k[9] * y[4]) + k[10] * y[6] + 2.0 * (k[11] * y[7]);
        s.t22 += k[0] * y[0] + k[1] * y[1] + k[3] * y[3] + -1.0 * (k[5] * y[5]) + -1.0 * (k[6] * y[6]) + -1.0 * (k[8] * y[8]) + k[9] * y[9] + k[11] * y[11] + -1.0 * (k[12] * y[12]) + -1.0 * (k[13] * y[13]);
        s.t31 += -1.0 * (k[1] * y[3]) + k[4] * y[2] + k[6] * y[8] + -2.0 * (k[9] * y[1]) + -1.0 * (k[10] * y[7]) + 2.0 * (k[12] * y[6]);
        s.t33 += k[0] * y[0] + -1.0 * (k[3] * y[3]) + k[4] * y[4] + k[5] * y[5] + -1.0 * (k[7] * y[7]) + -1.0 * (k[8] * y[8]) + k[9] * y[9] + -1.0 * (k[11] * y[11]) + k[12] * y[12] + -1.0 * (k[13] * y[13]);
        s.k33 += k[0] * y[3] + -1.0 * (k[4] * y[7]) + -1.0 * (k[5] * y[8]) + -1.0 * (k[9] * y[11]) + k[12] * y[13];
        s.s13 += k[1] * y[0] + k[6] * y[5] + -1.0 * (k[7] * y[2]) + -1.0 * (k[10] * y[4]) + 2.0 * (k[11] * y[1]) + 2.0 * (k[13] * y[6]);
        s.s23 += k[2] * y[0] + -1.0 * (k[6] * y[4]) + -1.0 * (k[7] * y[1]) + -2.0 * (k[8] * y[2]) + -1.0 * (k[10] * y[9]) + 2.0 * (k[13] * y[10]);
    }
};

// MinorFluidG: 5 components, coefficients FluidCoef
struct MinorFluidGAdj {
    static constexpr int N = 5;
    using Coef = FluidCoef;
    using Bar = FluidCoefBar;
    // g = A^T k
    __device__ static __forceinline__ void tr(const FluidCoef& a, const cd* k, cd* g)
    {
        g[0] = a.t11 * k[0] + a.t22 * k[0] + a.s12 * k[1] + a.s22 * k[2] + (-1.0 * a.s11) * k[3];
        g[1] = (-2.0 * a.t12) * k[2] + (2.0 * a.t21) * k[3] + (-2.0 * a.s12) * k[4];
        g[2] = a.k22 * k[0] + (-1.0 * a.t21) * k[1] + a.t11 * k[2] + (-1.0 * a.t22) * k[2] + a.s11 * k[4];
        g[3] = (-1.0 * a.k11) * k[0] + a.t12 * k[1] + (-1.0 * a.t11) * k[3] + a.t22 * k[3] + (-1.0 * a.s22) * k[4];
        g[4] = a.k11 * k[2] + (-1.0 * a.k22) * k[3] + (-1.0 * a.t11) * k[4] + (-1.0 * a.t22) * k[4];
    }
    // s.e += k . (dA/da_e) y
    __device__ static __forceinline__ void cgrad(const cd* k, const cd* y, FluidCoefBar& s)
    {
        s.t11 += k[0] * y[0] + k[2] * y[2] + -1.0 * (k[3] * y[3]) + -1.0 * (k[4] * y[4]);
        s.t12 += k[1] * y[3] + -2.0 * (k[2] * y[1]);
        s.k11 += -1.0 * (k[0] * y[3]) + k[2] * y[4];
        s.s11 += -1.0 * (k[3] * y[0]) + k[4] * y[2];
        s.s12 += k[1] * y[0] + -2.0 * (k[4] * y[1]);
        s.s22 += k[2] * y[0] + -1.0 * (k[4] * y[3]);
        s.t21 += -1.0 * (k[1] * y[2]) + 2.0 * (k[3] * y[1]);
        s.t22 += k[0] * y[0] + -1.0 * (k[2] * y[2]) + k[3] * y[3] + -1.0 * (k[4] * y[4]);
        s.k22 += k[0] * y[2] + -1.0 * (k[3] * y[4]);
    }
};

// BvecSolidG: 14 components, coefficients SolidCoef
struct BvecSolidGAdj {
    static constexpr int N = 14;
    using Coef = SolidCoef;
    using Bar = SolidCoefBar;
    // g = A^T k
    __device__ static __forceinline__ void tr(const SolidCoef& a, const cd* k, cd* g)
    {
        g[0] = (-1.0 * a.t11) * k[0] + (-1.0 * a.t22) * k[0] + (-1.0 * a.k22) * k[3] + a.k11 * k[6];
        g[1] = (-1.0 * a.t11) * k[1] + (-1.0 * a.t33) * k[1] + (-1.0 * a.k33) * k[4] + (-1.0 * a.t12) * k[5] + a.k11 * k[9];
        g[2] = (-1.0 * a.s12) * k[0] + (-2.0 * a.s13) * k[1] + a.t21 * k[3] + (2.0 * a.t31) * k[4] + (-1.0 * a.s23) * k[5] + (-1.0 * a.t12) * k[6];
        g[3] = (-1.0 * a.s22) * k[0] + (-1.0 * a.s23) * k[1] + a.t12 * k[2] + a.t22 * k[3] + (-1.0 * a.t11) * k[3] + (-1.0 * a.t12) * k[7] + (-1.0 * a.k11) * k[11];
        g[4] = (-1.0 * a.s23) * k[0] + a.t33 * k[4] + (-1.0 * a.t11) * k[4] + (-1.0 * a.t12) * k[8] + (-1.0 * a.k11) * k[12];
        g[5] = a.t31 * k[0] + (-1.0 * a.t21) * k[1] + (-1.0 * a.t22) * k[5] + (-1.0 * a.t33) * k[5] + (-1.0 * a.k33) * k[8] + a.k22 * k[10];
        g[6] = a.s11 * k[0] + (-1.0 * a.t21) * k[2] + (-1.0 * a.s13) * k[5] + a.t11 * k[6] + (-1.0 * a.t22) * k[6] + a.t21 * k[7] + a.t31 * k[8] + a.k22 * k[11];
        g[7] = a.s12 * k[0] + (-1.0 * a.s13) * k[1] + (-1.0 * a.t21) * k[3] + a.t31 * k[4] + (-2.0 * a.s23) * k[5] + a.t12 * k[6];
        g[8] = a.s13 * k[0] + (-1.0 * a.t21) * k[4] + (-1.0 * a.t22) * k[8] + a.t33 * k[8] + (-1.0 * a.k22) * k[13];
        g[9] = a.s11 * k[1] + (-1.0 * a.t31) * k[2] + a.s12 * k[5] + a.t11 * k[9] + (-1.0 * a.t33) * k[9] + a.t21 * k[10] + a.k33 * k[12];
        g[10] = a.s12 * k[1] + (-1.0 * a.t31) * k[3] + a.s22 * k[5] + a.t12 * k[9] + a.t22 * k[10] + (-1.0 * a.t33) * k[10] + a.k33 * k[13];
        g[11] = a.s12 * k[2] + (-1.0 * a.s11) * k[3] + a.s22 * k[6] + (-1.0 * a.s12) * k[7] + a.s23 * k[9] + (-1.0 * a.s13) * k[10] + a.t11 * k[11] + a.t22 * k[11] + (-1.0 * a.t31) * k[13];
        g[12] = a.s13 * k[2] + (-1.0 * a.s11) * k[4] + a.s23 * k[6] + (-1.0 * a.s12) * k[8] + a.t11 * k[12] + a.t33 * k[12] + a.t21 * k[13];
        g[13] = a.s13 * k[3] + (-1.0 * a.s12) * k[4] + a.s23 * k[7] + (-1.0 * a.s22) * k[8] + a.t12 * k[12] + a.t22 * k[13] + a.t33 * k[13];
    }
    // s.e += k . (dA/da_e) y
    __device__ static __forceinline__ void cgrad(const cd* k, const cd* y, SolidCoefBar& s)
    {
        s.t11 += -1.0 * (k[0] * y[0]) + -1.0 * (k[1] * y[1]) + -1.0 * (k[3] * y[3]) + -1.0 * (k[4] * y[4]) + k[6] * y[6] + k[9] * y[9] + k[11] * y[11] + k[12] * y[12];
        s.t12 += k[2] * y[3] + -1.0 * (k[5] * y[1]) + -1.0 * (k[6] * y[2]) + k[6] * y[7] + -1.0 * (k[7] * y[3]) + -1.0 * (k[8] * y[4]) + k[9] * y[10] + k[12] * y[13];
        s.k11 += k[6] * y[0] + k[9] * y[1] + -1.0 * (k[11] * y[3]) + -1.0 * (k[12] * y[4]);
        s.k22 += -1.0 * (k[3] * y[0]) + k[10] * y[5] + k[11] * y[6] + -1.0 * (k[13] * y[8]);
        s.s11 += k[0] * y[6] + k[1] * y[9] + -1.0 * (k[3] * y[11]) + -1.0 * (k[4] * y[12]);
        s.s12 += k[0] * y[7] + -1.0 * (k[0] * y[2]) + k[1] * y[10] + k[2] * y[11] + -1.0 * (k[4] * y[13]) + k[5] * y[9] + -1.0 * (k[7] * y[11]) + -1.0 * (k[8] * y[12]);
        s.s22 += -1.0 * (k[0] * y[3]) + k[5] * y[10] + k[6] * y[11] + -1.0 * (k[8] * y[13]);
        s.t21 += -1.0 * (k[1] * y[5]) + -1.0 * (k[2] * y[6]) + k[3] * y[2] + -1.0 * (k[3] * y[7]) + -1.0 * (k[4] * y[8]) + k[7] * y[6] + k[10] * y[9] + k[13] * y[12];
        s.t22 += -1.0 * (k[0] * y[0]) + k[3] * y[3] + -1.0 * (k[5] * y[5]) + -1.0 * (k[6] * y[6]) + -1.0 * (k[8] * y[8]) + k[10] * y[10] + k[11] * y[11] + k[13] * y[13];
        s.t31 += k[0] * y[5] + -1.0 * (k[2] * y[9]) + -1.0 * (k[3] * y[10]) + 2.0 * (k[4] * y[2]) + k[4] * y[7] + k[8] * y[6] + -1.0 * (k[13] * y[11]);
        s.t33 += -1.0 * (k[1] * y[1]) + k[4] * y[4] + -1.0 * (k[5] * y[5]) + k[8] * y[8] + -1.0 * (k[9] * y[9]) + -1.0 * (k[10] * y[10]) + k[12] * y[12] + k[13] * y[13];
        s.k33 += -1.0 * (k[4] * y[1]) + -1.0 * (k[8] * y[5]) + k[12] * y[9] + k[13] * y[10];
        s.s13 += k[0] * y[8] + -2.0 * (k[1] * y[2]) + -1.0 * (k[1] * y[7]) + k[2] * y[12] + k[3] * y[13] + -1.0 * (k[5] * y[6]) + -1.0 * (k[10] * y[11]);
        s.s23 += -1.0 * (k[0] * y[4]) + -1.0 * (k[1] * y[3]) + -1.0 * (k[5] * y[2]) + -2.0 * (k[5] * y[7]) + k[6] * y[12] + k[7] * y[13] + k[9] * y[11];
    }
};

// MinorSolidNC: 5 components, coefficients SolidCoef
struct MinorSolidNCAdj {
    static constexpr int N = 5;
    using Coef = SolidCoef;
    using Bar = SolidCoefBar;
    // g = A^T k
    __device__ static __forceinline__ void tr(const SolidCoef& a, const cd* k, cd* g)
    {
        g[0] = a.t11 * k[0] + a.t22 * k[0] + a.s12 * k[1] + a.s22 * k[2] + (-1.0 * a.s11) * k[3];
        g[1] = (-2.0 * a.t12) * k[2] + (2.0 * a.t21) * k[3] + (-2.0 * a.s12) * k[4];
        g[2] = a.k22 * k[0] + (-1.0 * a.t21) * k[1] + a.t11 * k[2] + (-1.0 * a.t22) * k[2] + a.s11 * k[4];
        g[3] = (-1.0 * a.k11) * k[0] + a.t12 * k[1] + (-1.0 * a.t11) * k[3] + a.t22 * k[3] + (-1.0 * a.s22) * k[4];
        g[4] = a.k11 * k[2] + (-1.0 * a.k22) * k[3] + (-1.0 * a.t11) * k[4] + (-1.0 * a.t22) * k[4];
    }
    // s.e += k . (dA/da_e) y
    __device__ static __forceinline__ void cgrad(const cd* k, const cd* y, SolidCoefBar& s)
    {
        s.t11 += k[0] * y[0] + k[2] * y[2] + -1.0 * (k[3] * y[3]) + -1.0 * (k[4] * y[4]);
        s.t12 += k[1] * y[3] + -2.0 * (k[2] * y[1]);
        s.k11 += -1.0 * (k[0] * y[3]) + k[2] * y[4];
        s.k22 += k[0] * y[2] + -1.0 * (k[3] * y[4]);
        s.s11 += -1.0 * (k[3] * y[0]) + k[4] * y[2];
        s.s12 += k[1] * y[0] + -2.0 * (k[4] * y[1]);
        s.s22 += k[2] * y[0] + -1.0 * (k[4] * y[3]);
        s.t21 += -1.0 * (k[1] * y[2]) + 2.0 * (k[3] * y[1]);
        s.t22 += k[0] * y[0] + -1.0 * (k[2] * y[2]) + k[3] * y[3] + -1.0 * (k[4] * y[4]);
    }
};

// MinorFluidNC: 2 components, coefficients FluidCoef
struct MinorFluidNCAdj {
    static constexpr int N = 2;
    using Coef = FluidCoef;
    using Bar = FluidCoefBar;
    // g = A^T k
    __device__ static __forceinline__ void tr(const FluidCoef& a, const cd* k, cd* g)
    {
        g[0] = a.t11 * k[0] + a.s11 * k[1];
        g[1] = a.k11 * k[0] + (-1.0 * a.t11) * k[1];
    }
    // s.e += k . (dA/da_e) y
    __device__ static __forceinline__ void cgrad(const cd* k, const cd* y, FluidCoefBar& s)
    {
        s.t11 += k[0] * y[0] + -1.0 * (k[1] * y[1]);
        s.k11 += k[0] * y[1];
        s.s11 += k[1] * y[0];
    }
};

// BvecSolidNC: 4 components, coefficients SolidCoef
struct BvecSolidNCAdj {
    static constexpr int N = 4;
    using Coef = SolidCoef;
    using Bar = SolidCoefBar;
    // g = A^T k
    __device__ static __forceinline__ void tr(const SolidCoef& a, const cd* k, cd* g)
    {
        g[0] = (-1.0 * a.t11) * k[0] + (-1.0 * a.t12) * k[1] + (-1.0 * a.k11) * k[2];
        g[1] = (-1.0 * a.t21) * k[0] + (-1.0 * a.t22) * k[1] + (-1.0 * a.k22) * k[3];
        g[2] = (-1.0 * a.s11) * k[0] + (-1.0 * a.s12) * k[1] + a.t11 * k[2] + a.t21 * k[3];
        g[3] = (-1.0 * a.s12) * k[0] + (-1.0 * a.s22) * k[1] + a.t12 * k[2] + a.t22 * k[3];
    }
    // s.e += k . (dA/da_e) y
    __device__ static __forceinline__ void cgrad(const cd* k, const cd* y, SolidCoefBar& s)
    {
        s.t11 += -1.0 * (k[0] * y[0]) + k[2] * y[2];
        s.t12 += -1.0 * (k[1] * y[0]) + k[2] * y[3];
        s.k11 += -1.0 * (k[2] * y[0]);
        s.k22 += -1.0 * (k[3] * y[1]);
        s.s11 += -1.0 * (k[0] * y[2]);
        s.s12 += -1.0 * (k[0] * y[3]) + -1.0 * (k[1] * y[2]);
        s.s22 += -1.0 * (k[1] * y[3]);
        s.t21 += -1.0 * (k[0] * y[1]) + k[3] * y[2];
        s.t22 += -1.0 * (k[1] * y[1]) + k[3] * y[3];
    }
};

}  // namespace YSG_VARIANT
}  // namespace ysg
