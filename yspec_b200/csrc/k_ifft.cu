// k_ifft.cu -- time series of yspec.f90:432-486 (module_fourier.f90:55-145).
//
// Per receiver and component the reference builds a length-n row (zero
// outside bins i1..i2, cosine taper, Hermitian extension), runs the
// Numerical-Recipes radix-2 decimation-in-time FFT with isign = +1
// (fourrow_dp, module_fourier.f90:7-50), divides by dt*n, multiplies by
// e^{eps t}, dimensionalises and rotates to Z/N/E.  Its twiddles use the
// single-precision pi of nrtype.f90, so the transform is the same
// butterfly network with angles m*pi_f/mmax; reproducing that network
// (not a DFT with exact pi) is what keeps the traces within 1e-9.
//
// The network is split at stage p1 = ceil(log2(n)/2): after bit reversal
// the first p1 stages act inside contiguous blocks of b1 = 2^p1 elements
// (pass A), the remaining stages act on the b1 residue classes i mod b1
// (pass B), which are independent.  Pass A reads the spectra directly and
// builds the row on the fly; pass B applies the post-processing and writes
// the real traces.  Intermediate rows live in a scratch buffer.
#include "ysg_kernels.h"

namespace ysg {

constexpr int TILE_A = 512;

__device__ __forceinline__ unsigned bitrev(unsigned g, int p) { return __brev(g) >> (32 - p); }

// All extents below are powers of two: index arithmetic uses shifts and
// masks (log2 by count of trailing zeros), never integer division.
__device__ __forceinline__ int lg2(int v) { return __ffs(v) - 1; }

// Element i (0-based, natural order) of the filtered Hermitian row.
__device__ __forceinline__ cd row_value(unsigned i, const TraceDev& td, const cd* __restrict__ spec,
                                        const double* __restrict__ filt)
{
    const unsigned n = (unsigned)td.nt, n2 = n / 2;
    bool cj = false;
    if (i > n2) {
        i = n - i;
        cj = true;
    }
    const int I = (int)i + 1;                     // 1-based bin
    if (I < td.i1 || I > td.i2) return mk(0.0);
    cd v = spec[I - td.i1] * filt[i];
    return cj ? conj(v) : v;
}

__global__ void __launch_bounds__(TILE_A / 2) k_ifft_a(TraceDev td, const cd* __restrict__ ur,
                                                      const cd* __restrict__ ut,
                                                      const cd* __restrict__ up,
                                                      const double* __restrict__ filt,
                                                      const cd* __restrict__ tw, cd* __restrict__ scr)
{
    __shared__ cd d[TILE_A];
    const int n = td.nt, p = td.log2n, b1 = td.b1;
    const int tile = min(TILE_A, n);
    const int row = blockIdx.y;                   // 3 k + c
    const int k = row / 3, c = row - 3 * k;
    const cd* spec = (c == 0 ? ur : (c == 1 ? ut : up)) + (size_t)k * td.nw;
    const unsigned base = (unsigned)blockIdx.x * tile;
    for (int t = threadIdx.x; t < tile; t += blockDim.x)
        d[t] = row_value(bitrev(base + t, p), td, spec, filt);
    __syncthreads();
    const int half = tile / 2, hb = b1 / 2, n2 = n / 2;
    const int lhb = lg2(hb), ln2 = lg2(n2);
    for (int s = 0, mh = 1; mh < b1; s++, mh <<= 1) {
        for (int t = threadIdx.x; t < half; t += blockDim.x) {
            const int sb = t >> lhb, tt = t & (hb - 1);
            const int grp = tt >> s, pos = tt & (mh - 1);
            const int i = sb * b1 + grp * 2 * mh + pos, j = i + mh;
            const cd w = tw[(size_t)pos << (ln2 - s)];
            const cd tmp = w * d[j];
            const cd di = d[i];
            d[j] = di - tmp;
            d[i] = di + tmp;
        }
        __syncthreads();
    }
    cd* dst = scr + (size_t)row * n + base;
    for (int t = threadIdx.x; t < tile; t += blockDim.x) dst[t] = d[t];
}

__global__ void __launch_bounds__(256) k_ifft_b(TraceDev td, int G, const cd* __restrict__ tw,
                                               const double* __restrict__ expt,
                                               const cd* __restrict__ scr, double* __restrict__ out)
{
    extern __shared__ cd sb[];                    // [B2][G]
    const int n = td.nt, b1 = td.b1, B2 = n / b1, n2 = n / 2;
    const int row = blockIdx.y;
    const int k = row / 3, c = row - 3 * k;
    const int r0 = blockIdx.x * G;
    const cd* src = scr + (size_t)row * n;
    const int lG = lg2(G), lB2 = lg2(B2);
    for (int e = threadIdx.x; e < G * B2; e += blockDim.x) {
        const int g = e & (G - 1), u = e >> lG;
        sb[e] = src[(size_t)r0 + g + (size_t)b1 * u];
    }
    __syncthreads();
    const int nbf = G * B2 / 2;
    for (int mu = 1, lmu = 0; mu < B2; mu <<= 1, lmu++) {
        const int stride = 1 << (lB2 - lmu - 1);
        for (int t = threadIdx.x; t < nbf; t += blockDim.x) {
            const int g = t & (G - 1), tt = t >> lG;
            const int grp = tt >> lmu, posu = tt & (mu - 1);
            const int u = grp * 2 * mu + posu, v = u + mu;
            const int r = r0 + g;
            const cd w = tw[(size_t)(r + b1 * posu) * stride];
            const cd tmp = w * sb[v * G + g];
            const cd du = sb[u * G + g];
            sb[v * G + g] = du - tmp;
            sb[u * G + g] = du + tmp;
        }
        __syncthreads();
    }
    (void)n2;
    double* o = out + (size_t)td.nout * 4 * k;
    for (int e = threadIdx.x; e < G * B2; e += blockDim.x) {
        const int g = e & (G - 1), u = e >> lG;
        const int i = r0 + g + b1 * u;
        if (i >= td.nout) continue;
        // data/(dt*n), * e^{eps t}, * amplitude scale (yspec.f90:439-460)
        const double v = ((sb[e].x / td.scale) * expt[i]) * td.amp_norm;
        o[(size_t)(c + 1) * td.nout + i] = v;
        if (c == 0) o[i] = ((double)i * td.dt) * td.t_norm;
    }
}

// Rotation to north / east, yspec.f90:466-473.
__global__ void k_rotate(int nout, int nr, const double* __restrict__ cs, double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (i >= nout || k >= nr) return;
    double* o = out + (size_t)nout * 4 * k;
    const double ca = cs[2 * k], sa = cs[2 * k + 1];
    const double t1 = o[(size_t)2 * nout + i], t2 = o[(size_t)3 * nout + i];
    o[(size_t)2 * nout + i] = -(t1 * ca) + t2 * sa;
    o[(size_t)3 * nout + i] = t1 * sa + t2 * ca;
}

size_t ifft_scratch_bytes(int nt, int nr) { return (size_t)3 * nr * nt * sizeof(cd); }

cudaError_t launch_ifft(const TraceDev& td, const cd* ur, const cd* ut, const cd* up,
                        const double* filt, const cd* tw, const double* expt, const double* cs_azep,
                        cd* scratch, double* out, cudaStream_t s)
{
    if (td.nr <= 0) return cudaSuccess;
    const int n = td.nt;
    const int tile = n < TILE_A ? n : TILE_A;
    dim3 ga(n / tile, 3 * td.nr);
    k_ifft_a<<<ga, tile / 2, 0, s>>>(td, ur, ut, up, filt, tw, scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int B2 = n / td.b1;
    int G = 512 / B2;
    if (G < 1) G = 1;
    if (G > td.b1) G = td.b1;
    int threads = G * B2 / 2;
    if (threads > 256) threads = 256;
    if (threads < 32) threads = 32;
    dim3 gb(td.b1 / G, 3 * td.nr);
    k_ifft_b<<<gb, threads, (size_t)G * B2 * sizeof(cd), s>>>(td, G, tw, expt, scratch, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dim3 gr((td.nout + 255) / 256, td.nr);
    k_rotate<<<gr, 256, 0, s>>>(td.nout, td.nr, cs_azep, out);
    return cudaGetLastError();
}

}  // namespace ysg
