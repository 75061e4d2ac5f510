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

// ---------------------------------------------------------------------------
// The same sum on the FP64 tensor cores (mma.sync m8n8k4 .f64; tcgen05 has
// no FP64 kind).  Every term is a product of a coefficient row, complex and
// indexed (l, j), with a Legendre row, real and indexed (l, k), summed over
// l: a matrix product with l as the inner dimension.  A CTA covers 16
// frequencies x 32 receivers as eight 8x8 warp tiles; each warp keeps all
// 30 real accumulators of its tile (ar, at, ap for the five m, re and im)
// in registers.  The degrees are staged 8 at a time (two MMA steps) into
// shared memory with cp.async, double-buffered so the next stage loads
// while the tensor cores work on this one; elements beyond the band, the
// receivers or lmax are zero-filled by the copy itself.  Row strides are
// padded so that a warp's fragment loads are conflict-free.  Per MMA step
// each warp issues 44 MMAs: the signs s = (-1)^m for m < 0 and the factors
// +-m of the i m terms scale the Legendre fragments, never the
// accumulators, and the phase factors e^{i m phi_k} are applied once, in
// the epilogue.
//
// Every CTA reads its frequency tile's coefficient rows and its receiver
// tile's Legendre rows for all degrees, so which tiles are in flight
// together decides the DRAM traffic: neither array fits L2 at c5 sizes.
// The 1-D grid is rasterised in groups of F frequency tiles: consecutive
// CTAs take the F frequency tiles of one receiver tile, then those of the
// next, so the CTAs in flight share F tiles of coefficients and about
// (CTAs in flight / F) tiles of Legendre rows through L2.  The launcher
// picks F to minimise the modelled re-reads with that working set within
// half of L2.
// ---------------------------------------------------------------------------
constexpr int LM_J = 16;                  // frequencies per CTA
constexpr int LM_K = 32;                  // receivers per CTA
constexpr int LM_S = 8;                   // degrees per pipeline stage (two MMA steps of 4)
constexpr int LM_SA = NCOEF * LM_J + 2;   // degree-row stride of the coefficients, complex values
constexpr int LM_KX = 10;                 // receiver stride of the Legendre rows, doubles (8 used)
constexpr int LM_SB = LM_K * LM_KX + 8;   // degree-row stride of the Legendre rows, doubles
constexpr int LM_THREADS = 256;
constexpr size_t LM_STAGE_BYTES = (size_t)LM_S * LM_SA * 16 + (size_t)LM_S * LM_SB * 8;

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// 16-byte asynchronous copy global -> shared; src_bytes = 0 fills zeros
// (the source address is then not read).
__device__ __forceinline__ void cp16(void* dst, const void* src, int src_bytes)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes)
                 : "memory");
}

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Issue the copies of stage l0 .. l0+7 into one buffer.
__device__ __forceinline__ void lm_stage(unsigned char* buf, int l0, int j0, int k0, int nw, int nr,
                                         int L, int lmin, const cd* __restrict__ coef,
                                         const double* __restrict__ T)
{
    cd* cs = reinterpret_cast<cd*>(buf);
    double* bs = reinterpret_cast<double*>(buf + (size_t)LM_S * LM_SA * 16);
    for (int e = threadIdx.x; e < LM_S * NCOEF * LM_J; e += LM_THREADS) {
        const int j = e % LM_J, q = (e / LM_J) % NCOEF, ll = e / (LM_J * NCOEF);
        const int gj = j0 + j, gl = l0 + ll;
        const bool in = gj < nw && gl < L;
        const cd* src = in ? coef + ((size_t)gl * NCOEF + q) * nw + gj : coef;
        cp16(cs + ll * LM_SA + q * LM_J + j, src, in ? 16 : 0);
    }
    for (int e = threadIdx.x; e < LM_S * LM_K * 4; e += LM_THREADS) {
        const int c = e & 3, k = (e >> 2) % LM_K, ll = e / (4 * LM_K);
        const int gk = k0 + k, gl = l0 + ll;
        const bool in = gk < nr && gl < L;
        const double* src = in ? T + ((size_t)(gl + lmin) * nr + gk) * 8 + 2 * c : T;
        cp16(bs + ll * LM_SB + k * LM_KX + 2 * c, src, in ? 16 : 0);
    }
}

__global__ void __launch_bounds__(LM_THREADS, 1) k_lsum_mma(int nw, int nr, int L, int lmin, int group,
                                                           const cd* __restrict__ coef,
                                                           const double* __restrict__ T,
                                                           const cd* __restrict__ E,
                                                           cd* __restrict__ ur, cd* __restrict__ ut,
                                                           cd* __restrict__ up)
{
    extern __shared__ __align__(16) unsigned char lm_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // grouped rasterisation (above): group g holds frequency tiles
    // g F .. g F + Fg - 1 of every receiver tile, frequency tile fastest
    const int nft = (nw + LM_J - 1) / LM_J, nrt = (nr + LM_K - 1) / LM_K;
    const long long b = blockIdx.x;
    const int grp = (int)(b / ((long long)group * nrt));
    const int f0 = grp * group;
    const int fg = min(group, nft - f0);
    const int idx = (int)(b - (long long)grp * group * nrt);
    const int k0 = (idx / fg) * LM_K, j0 = (f0 + idx % fg) * LM_J;
    const int jsub = warp & 1, ksub = warp >> 1;
    const int fr = lane >> 2, fc = lane & 3;      // fragment row / column of this lane
    // acc[slot][0..5]: ar re, ar im, at re, at im, ap re, ap im
    double acc[5][6][2];
#pragma unroll
    for (int m = 0; m < 5; m++)
#pragma unroll
        for (int q = 0; q < 6; q++) acc[m][q][0] = acc[m][q][1] = 0.0;
    const int nst = (L + LM_S - 1) / LM_S;
    lm_stage(lm_smem, 0, j0, k0, nw, nr, L, lmin, coef, T);
    cp_commit();
    for (int st = 0; st < nst; st++) {
        unsigned char* buf = lm_smem + (size_t)(st & 1) * LM_STAGE_BYTES;
        if (st + 1 < nst) {
            lm_stage(lm_smem + (size_t)((st + 1) & 1) * LM_STAGE_BYTES, (st + 1) * LM_S, j0, k0, nw, nr,
                     L, lmin, coef, T);
            cp_commit();
            cp_wait<1>();
        } else {
            cp_wait<0>();
        }
        __syncthreads();
        const cd* cs = reinterpret_cast<const cd*>(buf);
        const double* bs = reinterpret_cast<const double*>(buf + (size_t)LM_S * LM_SA * 16);
#pragma unroll
        for (int kk = 0; kk < LM_S / 4; kk++) {
            const cd* ca = cs + (kk * 4 + fc) * LM_SA + jsub * 8 + fr;
            const double* cb = bs + (kk * 4 + fc) * LM_SB + (ksub * 8 + fr) * LM_KX;
            double b[8];
#pragma unroll
            for (int x = 0; x < 8; x++) b[x] = cb[x];
            // m = 0 (slot 2): ar += uu X0, at += vv dX0
            {
                const cd u = ca[2 * LM_J], v = ca[7 * LM_J];
                dmma(acc[2][0], u.x, b[0]);
                dmma(acc[2][1], u.y, b[0]);
                dmma(acc[2][2], v.x, b[3]);
                dmma(acc[2][3], v.y, b[3]);
            }
#pragma unroll
            for (int slot = 0; slot < 5; slot++) {
                if (slot == 2) continue;
                const int m = slot - 2, a = m < 0 ? -m : m;
                const double s = (m < 0 && (a & 1)) ? -1.0 : 1.0;
                const double sX = s * b[a], sXP = s * b[3 + a];
                const double msX = (double)m * sX, msXC = (double)m * s * b[5 + a];
                const cd u = ca[slot * LM_J], v = ca[(5 + slot) * LM_J], w = ca[(10 + slot) * LM_J];
                // ar += uu sX
                dmma(acc[slot][0], u.x, sX);
                dmma(acc[slot][1], u.y, sX);
                // at += vv sXP + i ww msX
                dmma(acc[slot][2], v.x, sXP);
                dmma(acc[slot][2], w.y, -msX);
                dmma(acc[slot][3], v.y, sXP);
                dmma(acc[slot][3], w.x, msX);
                // ap += i vv msXC - ww sXP
                dmma(acc[slot][4], v.y, -msXC);
                dmma(acc[slot][4], w.x, -sXP);
                dmma(acc[slot][5], v.x, msXC);
                dmma(acc[slot][5], w.y, -sXP);
            }
        }
        __syncthreads();              // this buffer is refilled two stages on
    }
    // epilogue: this lane holds (j, k) = (j0 + jsub 8 + fr, k0 + ksub 8 + 2 fc + c)
    const int j = j0 + jsub * 8 + fr;
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const int k = k0 + ksub * 8 + 2 * fc + c;
        if (j >= nw || k >= nr) continue;
        cd sr = mk(acc[2][0][c], acc[2][1][c]);
        cd st = mk(acc[2][2][c], acc[2][3][c]);
        cd sp = mk(acc[2][4][c], acc[2][5][c]);
#pragma unroll
        for (int slot = 0; slot < 5; slot++) {
            if (slot == 2) continue;
            const cd e = E[(size_t)k * 5 + slot];
            sr += e * mk(acc[slot][0][c], acc[slot][1][c]);
            st += e * mk(acc[slot][2][c], acc[slot][3][c]);
            sp += e * mk(acc[slot][4][c], acc[slot][5][c]);
        }
        const size_t o = (size_t)k * nw + j;
        ur[o] = sr;
        ut[o] = st;
        up[o] = sp;
    }
}

bool lsum_uses_mma(int nr) { return nr >= 8; }

// Group width F of the rasterisation: the modelled DRAM reads are the
// coefficients once per group of receiver tiles in flight together plus
// the Legendre rows once per group of frequency tiles; the working set (F
// coefficient tiles, inflight / F Legendre tiles) should stay within half
// of L2, else the smallest working set is taken.
int lsum_group_width(int nft, int nrt, int L, int inflight, double l2_bytes)
{
    const double coef_tile = (double)LM_J * NCOEF * L * 16.0, leg_tile = (double)LM_K * L * 64.0;
    const double coef_tot = nft * coef_tile, leg_tot = nrt * leg_tile;
    int best = 1;
    double best_reads = 0.0, best_ws = 0.0;
    bool best_fits = false;
    for (int F = 1; F <= nft; F++) {
        const int R = std::max(1, inflight / F);
        const double ws = F * coef_tile + std::min(R, nrt) * leg_tile;
        const double reads = coef_tot * (double)((nrt + R - 1) / R) + leg_tot * (double)((nft + F - 1) / F);
        const bool fits = ws <= 0.5 * l2_bytes;
        const bool better = F == 1 || (fits && (!best_fits || reads < best_reads)) ||
                            (!fits && !best_fits && ws < best_ws);
        if (better) {
            best = F;
            best_reads = reads;
            best_ws = ws;
            best_fits = fits;
        }
    }
    return best;
}

cudaError_t launch_lsum(int nw, int nr, int lmin, int lmax, const cd* coef, const double* T,
                        const cd* E, cd* ur, cd* ut, cd* up, cudaStream_t s)
{
    if (nw <= 0 || nr <= 0) return cudaSuccess;
    const int L = lmax - lmin + 1;
    if (lsum_uses_mma(nr)) {
        const long long nft = (nw + LM_J - 1) / LM_J, nrt = (nr + LM_K - 1) / LM_K;
        if (nft * nrt > 0x7fffffffLL) return cudaErrorInvalidValue;
        const size_t smem = 2 * LM_STAGE_BYTES;
        cudaError_t e = cudaFuncSetAttribute(k_lsum_mma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        int dev = 0, nsm = 0, l2 = 0, per = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_lsum_mma, LM_THREADS, smem)) != cudaSuccess)
            return e;
        const int group = lsum_group_width((int)nft, (int)nrt, L, nsm * std::max(per, 1), (double)l2);
        k_lsum_mma<<<(unsigned)(nft * nrt), LM_THREADS, smem, s>>>(nw, nr, L, lmin, group, coef, T, E, ur, ut, up);
        return cudaGetLastError();
    }
    dim3 block(LS_J, LS_K);
    dim3 grid((nw + LS_J - 1) / LS_J, (nr + LS_K - 1) / LS_K);
    k_lsum<<<grid, block, 0, s>>>(nw, nr, L, coef, T, lmin, E, ur, ut, up);
    return cudaGetLastError();
}

}  // namespace ysg
