// k_lsum.cu -- receiver l-sum of yspec.f90:291-293, :316-335, :396-419.
//
// For every frequency j and receiver k:
//   ur += sum_l sum_m uu_m X_l|m| s_m e^{i m phi_k}
//   ut += sum_l sum_m (vv_m dX_l|m| + i m ww_m X_l|m|) s_m e^{i m phi_k}
//   up += sum_l sum_m (i m vv_m X_l|m|/sin - ww_m dX_l|m|) s_m e^{i m phi_k}
// with s_m = (-1)^m for m < 0.  The phase factor does not depend on l, so
// each thread accumulates the five per-m sums over l and applies
// e^{i m phi_k} once at the end.  The block stages an l-chunk of the
// coefficient rows (32 frequencies) and of the Legendre table (8 receivers)
// in shared memory, so each coefficient load is reused by 8 receivers.
#include "ysg_kernels.h"

namespace ysg {

constexpr int LS_J = 32;    // frequencies per block
constexpr int LS_K = 8;     // receivers per block
constexpr int LS_L = 4;     // degrees per shared-memory chunk

__global__ void __launch_bounds__(LS_J* LS_K) k_lsum(int nw, int nr, int L, const cd* __restrict__ coef,
                                                    const double* __restrict__ T, int lmin,
                                                    const cd* __restrict__ E, cd* __restrict__ ur,
                                                    cd* __restrict__ ut, cd* __restrict__ up)
{
    __shared__ cd sc[LS_L][NCOEF][LS_J];
    __shared__ double sx[LS_L][LS_K][8];
    const int tj = threadIdx.x, tk = threadIdx.y;
    const int j = blockIdx.x * LS_J + tj;
    const int k = blockIdx.y * LS_K + tk;
    const int tid = tk * LS_J + tj;
    cd ar[5], at[5], ap[5];
    for (int m = 0; m < 5; m++) ar[m] = at[m] = ap[m] = mk(0.0);
    for (int l0 = 0; l0 < L; l0 += LS_L) {
        __syncthreads();
        for (int e = tid; e < LS_L * NCOEF * LS_J; e += LS_J * LS_K) {
            int jj = e % LS_J, q = (e / LS_J) % NCOEF, ll = e / (LS_J * NCOEF);
            int gj = blockIdx.x * LS_J + jj, gl = l0 + ll;
            sc[ll][q][jj] = (gj < nw && gl < L) ? coef[((size_t)gl * NCOEF + q) * nw + gj] : mk(0.0);
        }
        for (int e = tid; e < LS_L * LS_K * 8; e += LS_J * LS_K) {
            int q = e % 8, kk = (e / 8) % LS_K, ll = e / (8 * LS_K);
            int gk = blockIdx.y * LS_K + kk, gl = l0 + ll;
            sx[ll][kk][q] = (gk < nr && gl < L) ? T[((size_t)(gl + lmin) * nr + gk) * 8 + q] : 0.0;
        }
        __syncthreads();
        const int nl = min(LS_L, L - l0);
        for (int ll = 0; ll < nl; ll++) {
            const double* x = sx[ll][tk];
            // m = 0
            ar[2] += sc[ll][2][tj] * x[0];
            at[2] += sc[ll][7][tj] * x[3];
            // |m| = 1, 2 : X index a, sign s for negative m
#pragma unroll
            for (int a = 1; a <= 2; a++) {
                const double X = x[a], XP = x[3 + a], XC = x[5 + a];
                const double sgn = (a & 1) ? -1.0 : 1.0;
#pragma unroll
                for (int sm = -1; sm <= 1; sm += 2) {
                    const int m = sm * a;
                    const int slot = m + 2;
                    const double s = sm < 0 ? sgn : 1.0;
                    const cd uu = sc[ll][slot][tj], vv = sc[ll][5 + slot][tj];
                    const cd ww = sc[ll][10 + slot][tj];
                    ar[slot] += uu * (s * X);
                    // toroidal (zero coefficients for l <= 1): i m ww X, -ww dX
                    at[slot] += vv * (s * XP) + imul(ww) * ((double)m * s * X);
                    ap[slot] += imul(vv) * ((double)m * s * XC) - ww * (s * XP);
                }
            }
        }
    }
    if (j < nw && k < nr) {
        cd sr = ar[2], st = at[2], sp = ap[2];
        for (int slot = 0; slot < 5; slot++) {
            if (slot == 2) continue;
            cd e = E[(size_t)k * 5 + slot];
            sr += e * ar[slot];
            st += e * at[slot];
            sp += e * ap[slot];
        }
        size_t o = (size_t)k * nw + j;
        ur[o] = sr;
        ut[o] = st;
        up[o] = sp;
    }
}

cudaError_t launch_lsum(int nw, int nr, int lmin, int lmax, const cd* coef, const double* T,
                        const cd* E, cd* ur, cd* ut, cd* up, cudaStream_t s)
{
    if (nw <= 0 || nr <= 0) return cudaSuccess;
    dim3 block(LS_J, LS_K);
    dim3 grid((nw + LS_J - 1) / LS_J, (nr + LS_K - 1) / LS_K);
    k_lsum<<<grid, block, 0, s>>>(nw, nr, lmax - lmin + 1, coef, T, lmin, E, ur, ut, up);
    return cudaGetLastError();
}

}  // namespace ysg
