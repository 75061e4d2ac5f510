// k_legendre.cu -- Legendre / geometry table of yspec.f90:155-170.
//
// Restates module_function.f90:6-132 (legendre).  The reference restarts the
// three-term P_l recursion from l = 2 for every l; the recursion values do
// not depend on where it stops, so one thread per receiver carries it
// forward once over l = 2..lmax and produces the identical sequence.  The
// FP32 roundings of the reference (sqrt(real(l*(l+1))), the single-precision
// products in f1/f2) are kept.  This file is compiled with -fmad=false so
// every product and sum rounds separately, as in the reference, making the
// table bit-identical to an unfused FP64 evaluation; cos and sin of the
// epicentral angle come from the host.
//
// Table layout: T[((l * nr) + k) * 8 + q], q = X_l0, X_l1, X_l2, dX_l0,
// dX_l1, dX_l2, X_l1/sin, X_l2/sin.
#include "ysg_kernels.h"

namespace ysg {

__global__ void k_legendre(int nr, int lmax, const double* __restrict__ delta,
                           const double* __restrict__ ctv, const double* __restrict__ stv,
                           double* __restrict__ T)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nr) return;
    const double FOURPI = 12.56637061;
    const double theta = delta[k], ct = ctv[k], st = stv[k];
    const bool tiny = fabs(theta) <= 1.0e-5;
    double p1 = 1.0, p2 = ct;        // P_{l-1}, P_l after the recursion up to l
    for (int l = 0; l <= lmax; l++) {
        double x[3] = {0.0, 0.0, 0.0}, xp[3] = {0.0, 0.0, 0.0}, xc[3] = {0.0, 0.0, 0.0};
        const double fct = sqrt((double)(float)(2 * l + 1) / FOURPI);
        const double sfl3 = (double)sqrtf((float)(l * (l + 1)));
        const double compar = (double)(float)(2 * l + 1) / FOURPI;
        const double small = 1.0e-16 * compar;
        if (l >= 2) {
            double x3 = ((double)(float)(2 * l - 1) * ct * p2 - (double)(float)(l - 1) * p1) /
                        (double)(float)l;
            p1 = p2;
            p2 = x3;
        }
        if (l <= 1 || tiny) {
            x[0] = fct;
            if (l > 0) {
                x[0] = ct * fct;
                x[1] = -st * fct / sfl3;
                xp[0] = -st * fct;
                xp[1] = -0.5 * ct * fct * sfl3;
                xc[1] = fabs(theta) < 1.0e-5 ? xp[1] : x[1] / st;
            }
        } else {
            const int lp1 = l + 1, mp1 = 3;
            double x1 = p1, x2 = p2, x3;
            const double cot = ct / st, cosec = 1.0 / st;
            x3 = x2 * fct;
            x2 = (double)(float)l * (x1 - ct * x2) * fct / st;
            x[0] = x3;
            x[1] = x2;
            double sum = x3 * x3;
            xp[0] = -x2;
            xp[1] = (double)(float)(l * (l + 1)) * x3 - cot * x2;
            x[1] = -x[1] / sfl3;
            xc[1] = x[1] * cosec;
            xp[1] = -xp[1] / sfl3;
            sum = sum + 2.0 * x[1] * x[1];
            if (!(sum - compar > small)) {
                x1 = x3;
                x2 = -x2 / (double)sqrtf((float)(l * (l + 1)));
                for (int i = 3; i <= mp1; i++) {
                    const int kk = i - 1;
                    const double f1 = (double)sqrtf((float)(l + i - 1) * (float)(l - i + 2));
                    const double f2 = (double)sqrtf((float)(l + i - 2) * (float)(l - i + 3));
                    const double xm = (double)kk;
                    x3 = -(2.0 * cot * (xm - 1.0) * x2 + f2 * x1) / f1;
                    sum = sum + 2.0 * x3 * x3;
                    if (sum - compar > small && i != lp1) break;
                    x[i - 1] = x3;
                    xc[i - 1] = x[i - 1] * cosec;
                    x1 = x2;
                    xp[i - 1] = -(f1 * x2 + xm * cot * x3);
                    x2 = x3;
                }
            }
        }
        double* o = T + ((size_t)l * nr + k) * 8;
        o[0] = x[0]; o[1] = x[1]; o[2] = x[2];
        o[3] = xp[0]; o[4] = xp[1]; o[5] = xp[2];
        o[6] = xc[1]; o[7] = xc[2];
    }
}

cudaError_t launch_legendre(int nr, int lmax, const double* delta, const double* ct,
                            const double* st, double* T, cudaStream_t s)
{
    if (nr <= 0) return cudaSuccess;
    const int bs = 64;
    k_legendre<<<(nr + bs - 1) / bs, bs, 0, s>>>(nr, lmax, delta, ct, st, T);
    return cudaGetLastError();
}

}  // namespace ysg
