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
// the real traces.  Intermediate rows live in a scratch buffer.  Inside a
// pass each thread runs up to three stages at a time in registers (below).
#include "ysg_kernels.h"

namespace ysg {

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

// ---------------------------------------------------------------------------
// Register-blocked passes.  The butterfly network and
// its twiddle indices are unchanged (stage s pairs i and i + 2^s inside
// groups of 2^(s+1), twiddle tw[(i mod 2^s) << (log2(n/2) - s)]); only the
// work split changes.  Each thread holds 8 values and runs up to three
// consecutive stages on them in registers (a "round"); between rounds the
// values go through shared memory.  A round over stages s0 .. s0+m-1 acts on
// subsets {base + j + 2^s0 k : k < 2^m}, j < 2^s0, which those stages never
// mix with anything else.  Pass A covers stages 0 .. p1-1 inside blocks of
// b1 bit-reversed positions (tiles of 2048 positions per CTA), pass B the
// remaining stages on the residue classes r = i mod b1 (2048 / B2 classes
// per CTA, B2 = n / b1); pass B counts positions in units of b1 (u = i div
// b1), so a subset there is {r + b1 (base + j + 2^s0u k)}.
// ---------------------------------------------------------------------------
constexpr int FT = 2048;                 // values per CTA in either pass

// m stages (M = m) starting at stage s on this thread's values: subset q
// holds v[q 2^M + k], k < 2^M, at positions pos0[q] + dstep k (in units of
// i), so the lower value of a butterfly of stage s+st sits at
// pos0[q] + dstep (k mod 2^st) inside its group.
template <int M>
__device__ __forceinline__ void fft_round(cd (&v)[8], int s, const int (&pos0)[8 >> M], int dstep, int ln2,
                                          const cd* __restrict__ tw)
{
#pragma unroll
    for (int st = 0; st < M; st++) {
        const int sh = ln2 - (s + st);
#pragma unroll
        for (int q = 0; q < (8 >> M); q++)
#pragma unroll
            for (int k = 0; k < (1 << M); k++) {
                if (k & (1 << st)) continue;
                const int pos = pos0[q] + dstep * (k & ((1 << st) - 1));
                const cd w = tw[(size_t)pos << sh];
                cd& a = v[q * (1 << M) + k];
                cd& b = v[q * (1 << M) + k + (1 << st)];
                const cd tmp = w * b;
                b = a - tmp;
                a = a + tmp;
            }
    }
}

// One round of pass A on stages s0 .. s0+M-1: load (from the spectra for
// the first round, else from shared memory), butterflies, store (to the
// scratch row for the last round, else to shared memory).
template <int M>
__device__ __forceinline__ void round_a(cd (&v)[8], int s0, bool first, bool last, const TraceDev& td,
                                       unsigned base, int T, const cd* __restrict__ spec,
                                       const double* __restrict__ filt, const cd* __restrict__ tw,
                                       cd* buf, cd* __restrict__ dst)
{
    const int D = 1 << s0, ln2 = td.log2n - 1;
    int pos0[8 >> M];
#pragma unroll
    for (int q = 0; q < (8 >> M); q++) {
        const int sg = q * T + (int)threadIdx.x;          // subset index
        pos0[q] = ((sg >> s0) << (s0 + M)) + (sg & (D - 1));
    }
#pragma unroll
    for (int q = 0; q < (8 >> M); q++)
#pragma unroll
        for (int k = 0; k < (1 << M); k++) {
            const int pos = pos0[q] + D * k;
            v[q * (1 << M) + k] = first ? row_value(bitrev(base + pos, td.log2n), td, spec, filt) : buf[pos];
        }
    int tp[8 >> M];
#pragma unroll
    for (int q = 0; q < (8 >> M); q++) tp[q] = pos0[q] & (D - 1);   // position inside the group
    fft_round<M>(v, s0, tp, D, ln2, tw);
    if (!last && !first) __syncthreads();
#pragma unroll
    for (int q = 0; q < (8 >> M); q++)
#pragma unroll
        for (int k = 0; k < (1 << M); k++) {
            const int pos = pos0[q] + D * k;
            if (last) dst[pos] = v[q * (1 << M) + k];
            else buf[pos] = v[q * (1 << M) + k];
        }
    if (!last) __syncthreads();
}

__global__ void __launch_bounds__(FT / 8) k_ifft_a2(TraceDev td, const cd* __restrict__ ur,
                                                   const cd* __restrict__ ut, const cd* __restrict__ up,
                                                   const double* __restrict__ filt,
                                                   const cd* __restrict__ tw, cd* __restrict__ scr)
{
    __shared__ cd buf[FT];
    const int n = td.nt;
    const int tile = min(FT, n), T = tile / 8;
    const int p1 = lg2(td.b1);
    const int row = blockIdx.y;                   // 3 k + c
    const int k = row / 3, c = row - 3 * k;
    const cd* spec = (c == 0 ? ur : (c == 1 ? ut : up)) + (size_t)k * td.nw;
    const unsigned base = (unsigned)blockIdx.x * tile;
    cd* dst = scr + (size_t)row * n + base;
    cd v[8];
    for (int s0 = 0; s0 < p1; s0 += 3) {
        const int m = min(3, p1 - s0);
        const bool first = s0 == 0, last = s0 + m >= p1;
        if (m == 3) round_a<3>(v, s0, first, last, td, base, T, spec, filt, tw, buf, dst);
        else if (m == 2) round_a<2>(v, s0, first, last, td, base, T, spec, filt, tw, buf, dst);
        else round_a<1>(v, s0, first, last, td, base, T, spec, filt, tw, buf, dst);
    }
}

// One round of pass B on stages p1 + s0 .. p1 + s0 + M - 1 (s0 counted in
// units of b1).  Values of residue class r0 + g at u sit in buf[u G + g].
template <int M>
__device__ __forceinline__ void round_b(cd (&v)[8], int s0, bool first, bool last, const TraceDev& td,
                                        int G, int lG, int r0, int T, const cd* __restrict__ src,
                                        const cd* __restrict__ tw, const double* __restrict__ expt,
                                        cd* buf, double* __restrict__ o, int c)
{
    const int D = 1 << s0, ln2 = td.log2n - 1, b1 = td.b1;
    const int p1 = lg2(b1);
    int up0[8 >> M], gq[8 >> M];
#pragma unroll
    for (int q = 0; q < (8 >> M); q++) {
        const int sg = q * T + (int)threadIdx.x;
        gq[q] = sg & (G - 1);
        const int su = sg >> lG;                          // subset index in u
        up0[q] = ((su >> s0) << (s0 + M)) + (su & (D - 1));
    }
#pragma unroll
    for (int q = 0; q < (8 >> M); q++)
#pragma unroll
        for (int k = 0; k < (1 << M); k++) {
            const int u = up0[q] + D * k;
            v[q * (1 << M) + k] = first ? src[(size_t)(r0 + gq[q]) + (size_t)b1 * u] : buf[u * G + gq[q]];
        }
    int tp[8 >> M];
#pragma unroll
    for (int q = 0; q < (8 >> M); q++) tp[q] = r0 + gq[q] + b1 * (up0[q] & (D - 1));
    fft_round<M>(v, p1 + s0, tp, b1 * D, ln2, tw);
    if (!last && !first) __syncthreads();
#pragma unroll
    for (int q = 0; q < (8 >> M); q++)
#pragma unroll
        for (int k = 0; k < (1 << M); k++) {
            const int u = up0[q] + D * k;
            const cd x = v[q * (1 << M) + k];
            if (!last) {
                buf[u * G + gq[q]] = x;
                continue;
            }
            const int i = r0 + gq[q] + b1 * u;
            if (i >= td.nout) continue;
            // data/(dt*n), * e^{eps t}, * amplitude scale (yspec.f90:439-460)
            o[(size_t)(c + 1) * td.nout + i] = ((x.x / td.scale) * expt[i]) * td.amp_norm;
            if (c == 0) o[i] = ((double)i * td.dt) * td.t_norm;
        }
    if (!last) __syncthreads();
}

__global__ void __launch_bounds__(FT / 8) k_ifft_b2(TraceDev td, int G, const cd* __restrict__ tw,
                                                   const double* __restrict__ expt,
                                                   const cd* __restrict__ scr, double* __restrict__ out)
{
    __shared__ cd buf[FT];
    const int n = td.nt, b1 = td.b1, B2 = n / b1;
    const int pB = lg2(B2), lG = lg2(G), T = G * B2 / 8;
    const int row = blockIdx.y;
    const int k = row / 3, c = row - 3 * k;
    const int r0 = blockIdx.x * G;
    const cd* src = scr + (size_t)row * n;
    double* o = out + (size_t)td.nout * 4 * k;
    cd v[8];
    for (int s0 = 0; s0 < pB; s0 += 3) {
        const int m = min(3, pB - s0);
        const bool first = s0 == 0, last = s0 + m >= pB;
        if (m == 3) round_b<3>(v, s0, first, last, td, G, lG, r0, T, src, tw, expt, buf, o, c);
        else if (m == 2) round_b<2>(v, s0, first, last, td, G, lG, r0, T, src, tw, expt, buf, o, c);
        else round_b<1>(v, s0, first, last, td, G, lG, r0, T, src, tw, expt, buf, o, c);
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
    if (n < 8 || n > (1 << 20)) return cudaErrorInvalidValue;
    // one row per receiver and component in grid.y (at most 65535): receivers
    // go in chunks; each chunk's rows start at the top of the scratch buffer
    const int chunk = 65535 / 3;
    for (int k0 = 0; k0 < td.nr; k0 += chunk) {
        TraceDev sub = td;
        sub.nr = td.nr - k0 < chunk ? td.nr - k0 : chunk;
        const size_t so = (size_t)k0 * td.nw;
        const cd *sur = ur + so, *sut = ut + so, *sup = up + so;
        double* sout = out + (size_t)k0 * td.nout * 4;
        const int tile = n < FT ? n : FT;
        dim3 ga(n / tile, 3 * sub.nr);
        k_ifft_a2<<<ga, tile / 8, 0, s>>>(sub, sur, sut, sup, filt, tw, scratch);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        const int B2 = n / td.b1;
        int G = FT / B2;
        if (G > td.b1) G = td.b1;
        dim3 gb(td.b1 / G, 3 * sub.nr);
        k_ifft_b2<<<gb, G * B2 / 8, 0, s>>>(sub, G, tw, expt, scratch, sout);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        dim3 gr((td.nout + 255) / 256, sub.nr);
        k_rotate<<<gr, 256, 0, s>>>(td.nout, sub.nr, cs_azep + 2 * (size_t)k0, sout);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace ysg
