// k_ifft_noalloc.cu -- the time-series stage without any device allocation.
//
// Some callers cannot let the library allocate device memory: a host that
// reserves the whole GPU for its own pool at start-up, a host whose rules
// forbid hidden allocations, or code where a cudaMalloc would synchronise
// the device and stall its other streams.  ysg_traces_noalloc serves them:
// it runs the same filter + Hermitian extension + inverse FFT +
// post-processing as ysg_event_traces, but reads the spectra from and
// writes the traces to device buffers the caller owns, and keeps its
// intermediate rows in one fixed array compiled into the library.
//
// That array (g_trace_scratch, 2^20 complex values = 16 MiB) is held on
// every GPU that loads the library until the process exits.  Rows are
// processed in chunks of whole receivers that fit it; one transform row
// must fit three times, so nt <= 262144.  Every call shares the array and
// leaves the last call's rows in it: nothing in it needs to start at zero
// (each chunk is fully written before it is read), and two calls whose work
// overlaps on the GPU (different streams, or different host threads on the
// same device) race on it and must be serialised by the caller.
//
// The device address of the array is looked up with cudaGetSymbolAddress
// on the first call made on each device (with that device current) and
// cached by device ordinal; that first call should come before any stream
// capture.  The cache assumes the device's primary context, the one the
// runtime API uses, for the life of the process: after cudaDeviceReset, or
// from a separate driver-API context on the same device, the cached address
// is stale and this entry point must not be used.  The
// taper, FFT twiddles, e^{eps t} and the rotation angles are formed on the
// device, so apart from the launches nothing is allocated or copied.
#include <mutex>

#include <cuda_runtime.h>

#include "yspec_gpu.h"
#include "ysg_cplx.cuh"

// Records a CUDA failure for ysg_last_cuda_error() (capi.cu).
int ysg_cuda_fail_at(cudaError_t e, const char* file, int line);

namespace {

constexpr size_t kScratchComplex = (size_t)1 << 20;
constexpr int kMaxRowsY = 65535;        // grid.y limit: 3 rows per receiver

}  // namespace

static __device__ __align__(256) ysg::cd g_trace_scratch[kScratchComplex];

namespace {

using ysg::cd;
using ysg::mk;

constexpr int kTile = 512;
const double kPiD = (double)3.14159265358979323846f;   // nrtype.f90 pi_d (single-precision literal)

struct Noalloc {
    int nt, i1, i2, nw, nr, nout, log2n, b1;
    int k0;                       // first receiver of the chunk
    double df, dt, ep, scale, t_norm, amp_norm, w1, w2, w3, w4;
    bool filter;
};

__device__ __forceinline__ double taper(const Noalloc& a, int i)
{
    // module_fourier.f90:96-116, bin i (0-based) at frequency i*df
    if (!a.filter) return 1.0;
    const double w = (double)i * a.df;
    if (w < a.w1) return 0.0;
    if (w < a.w2) return 0.5 * (1.0 - cos(kPiD * (w - a.w1) / (a.w2 - a.w1)));
    if (w < a.w3) return 1.0;
    if (w < a.w4) return 0.5 * (1.0 - cos(kPiD * (a.w4 - w) / (a.w4 - a.w3)));
    return 0.0;
}

__device__ __forceinline__ cd twiddle(int pos, int mh)
{
    // exp(i pos pi_d / mh), the butterfly factor of fourrow_dp (isign = +1)
    double s, c;
    sincos((double)pos * (kPiD / (double)mh), &s, &c);
    return mk(c, s);
}

__device__ __forceinline__ cd row_value(unsigned i, const Noalloc& a, const cd* spec)
{
    const unsigned n = (unsigned)a.nt, n2 = n / 2;
    bool cj = false;
    if (i > n2) {
        i = n - i;
        cj = true;
    }
    const int I = (int)i + 1;
    if (I < a.i1 || I > a.i2) return mk(0.0);
    cd v = spec[I - a.i1] * taper(a, (int)i);
    return cj ? ysg::conj(v) : v;
}

__global__ void k_noalloc_a(Noalloc a, const cd* __restrict__ ur, const cd* __restrict__ ut,
                            const cd* __restrict__ up, cd* __restrict__ scr)
{
    __shared__ cd d[kTile];
    const int n = a.nt, p = a.log2n, b1 = a.b1;
    const int tile = min(kTile, n);
    const int row = blockIdx.y;                       // within the chunk: 3 k + c
    const int k = a.k0 + row / 3, c = row % 3;
    const cd* spec = (c == 0 ? ur : (c == 1 ? ut : up)) + (size_t)k * a.nw;
    const unsigned base = (unsigned)blockIdx.x * tile;
    for (int t = threadIdx.x; t < tile; t += blockDim.x)
        d[t] = row_value(__brev(base + t) >> (32 - p), a, spec);
    __syncthreads();
    const int half = tile / 2, hb = b1 / 2;
    for (int mh = 1; mh < b1; mh <<= 1) {
        for (int t = threadIdx.x; t < half; t += blockDim.x) {
            const int sb = t / hb, tt = t - sb * hb;
            const int grp = tt / mh, pos = tt - grp * mh;
            const int i = sb * b1 + grp * 2 * mh + pos, j = i + mh;
            const cd tmp = twiddle(pos, mh) * d[j];
            const cd di = d[i];
            d[j] = di - tmp;
            d[i] = di + tmp;
        }
        __syncthreads();
    }
    cd* dst = scr + (size_t)row * n + base;
    for (int t = threadIdx.x; t < tile; t += blockDim.x) dst[t] = d[t];
}

__global__ void k_noalloc_b(Noalloc a, int G, const cd* __restrict__ scr, double* __restrict__ out)
{
    extern __shared__ cd sb[];
    const int n = a.nt, b1 = a.b1, B2 = n / b1;
    const int row = blockIdx.y;
    const int k = a.k0 + row / 3, c = row % 3;
    const int r0 = blockIdx.x * G;
    const cd* src = scr + (size_t)row * n;
    for (int e = threadIdx.x; e < G * B2; e += blockDim.x)
        sb[e] = src[(size_t)r0 + e % G + (size_t)b1 * (e / G)];
    __syncthreads();
    for (int mu = 1; mu < B2; mu <<= 1) {
        for (int t = threadIdx.x; t < G * B2 / 2; t += blockDim.x) {
            const int g = t % G, tt = t / G;
            const int grp = tt / mu, posu = tt - grp * mu;
            const int u = grp * 2 * mu + posu, v = u + mu;
            const cd tmp = twiddle(r0 + g + b1 * posu, b1 * mu) * sb[v * G + g];
            const cd du = sb[u * G + g];
            sb[v * G + g] = du - tmp;
            sb[u * G + g] = du + tmp;
        }
        __syncthreads();
    }
    double* o = out + (size_t)a.nout * 4 * k;
    for (int e = threadIdx.x; e < G * B2; e += blockDim.x) {
        const int i = r0 + e % G + b1 * (e / G);
        if (i >= a.nout) continue;
        const double t = (double)i * a.dt;
        o[(size_t)(c + 1) * a.nout + i] = ((sb[e].x / a.scale) * exp(a.ep * t)) * a.amp_norm;
        if (c == 0) o[i] = t * a.t_norm;
    }
}

__global__ void k_noalloc_rotate(Noalloc a, int nrc, const double* __restrict__ azep,
                                 double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = a.k0 + blockIdx.y;
    if (i >= a.nout || blockIdx.y >= (unsigned)nrc) return;
    double* o = out + (size_t)a.nout * 4 * k;
    double sa, ca;
    sincos(azep[k], &sa, &ca);
    const double t1 = o[(size_t)2 * a.nout + i], t2 = o[(size_t)3 * a.nout + i];
    o[(size_t)2 * a.nout + i] = -(t1 * ca) + t2 * sa;
    o[(size_t)3 * a.nout + i] = t1 * sa + t2 * ca;
}

std::mutex g_mu;
cd* g_addr[128] = {};

// Device address of g_trace_scratch on the current device, looked up once.
int scratch_address(cd** p)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return ysg_cuda_fail_at(e, "k_ifft_noalloc.cu", __LINE__);
    if (dev < 0 || dev >= 128) return YSG_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_trace_scratch);
        if (e != cudaSuccess) return ysg_cuda_fail_at(e, "k_ifft_noalloc.cu", __LINE__);
        if (!ptr) return YSG_ERR_CUDA;
        g_addr[dev] = static_cast<cd*>(ptr);
    }
    *p = g_addr[dev];
    return YSG_OK;
}

}  // namespace

extern "C" int ysg_traces_noalloc(const ysg_time* tm, const double* d_ur, const double* d_ut,
                                  const double* d_up, const double* d_azep, double* d_out,
                                  int* nout, void* stream)
{
    if (!tm) return YSG_ERR_ARG;
    const int n = tm->nt, nr = tm->nr;
    // the same argument rules as the allocating time-series stage (k_ifft.cu)
    if (n < 8 || (n & (n - 1)) || tm->i1 < 1 || tm->i2 < tm->i1 || tm->i2 > n || nr < 0)
        return YSG_ERR_ARG;
    if (nr > 0 && (!d_ur || !d_ut || !d_up || !d_azep || !d_out)) return YSG_ERR_ARG;
    if ((size_t)3 * n > kScratchComplex) return YSG_ERR_LIMIT;   // one receiver must fit
    const int rows_out = ysg_trace_rows(tm);
    if (nout) *nout = rows_out;
    if (nr == 0) return YSG_OK;
    // an error left pending by earlier work on this thread is cleared here,
    // so the check after the launches reports this call's own failures
    (void)cudaGetLastError();
    cd* scr = nullptr;
    int rc = scratch_address(&scr);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    int p = 0;
    while ((1 << p) < n) p++;
    Noalloc a{};
    a.nt = n;
    a.i1 = tm->i1;
    a.i2 = tm->i2;
    a.nw = tm->i2 - tm->i1 + 1;
    a.nr = nr;
    a.nout = rows_out;
    a.log2n = p;
    a.b1 = 1 << ((p + 1) / 2);
    a.df = tm->df;
    a.dt = tm->dt;
    a.ep = tm->ep;
    a.scale = tm->dt * (double)n;
    a.t_norm = tm->t_norm;
    a.amp_norm = tm->amp_norm;
    a.w1 = tm->f11;
    a.w2 = tm->f12;
    a.w3 = tm->f21;
    a.w4 = tm->f22;
    a.filter = !(a.w1 == 0.0 && a.w2 == 0.0 && a.w3 == 0.0 && a.w4 == 0.0);
    int per_chunk = (int)(kScratchComplex / ((size_t)3 * n));   // receivers per chunk
    if (per_chunk > kMaxRowsY / 3) per_chunk = kMaxRowsY / 3;
    const int tile = n < kTile ? n : kTile;
    const int B2 = n / a.b1;
    int G = 512 / B2;
    if (G < 1) G = 1;
    if (G > a.b1) G = a.b1;
    int threads = G * B2 / 2;
    if (threads > 256) threads = 256;
    if (threads < 32) threads = 32;
    const cd* ur = reinterpret_cast<const cd*>(d_ur);
    const cd* ut = reinterpret_cast<const cd*>(d_ut);
    const cd* up = reinterpret_cast<const cd*>(d_up);
    for (int k0 = 0; k0 < nr; k0 += per_chunk) {
        const int nk = nr - k0 < per_chunk ? nr - k0 : per_chunk;
        a.k0 = k0;
        k_noalloc_a<<<dim3(n / tile, 3 * nk), tile / 2, 0, st>>>(a, ur, ut, up, scr);
        k_noalloc_b<<<dim3(a.b1 / G, 3 * nk), threads, (size_t)G * B2 * sizeof(cd), st>>>(a, G, scr, d_out);
        k_noalloc_rotate<<<dim3((rows_out + 255) / 256, nk), 256, 0, st>>>(a, nk, d_azep, d_out);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return ysg_cuda_fail_at(e, "k_ifft_noalloc.cu", __LINE__);
    }
    return YSG_OK;
}
