// k_schedule.cu -- cost model and ordering of the pair schedule.
//
// The batched solver can take its work as (event, l, 32 consecutive
// frequencies) tiles, or as lists of 32 pairs of near-equal cost and the
// same code path.  The second needs every pair's cost before the solve:
// k_pair_cost runs each pair's driver (yspec.f90:259-400) in the
// count-only build of the solver code, where yint makes every integer
// decision a real solve makes (start level, layers, steps per layer,
// module_int.f90:1847-1968) but steps no state, so the counts are exact.
// The steps across a whole knot interval depend only on omega: k_step_prefix
// sums them per frequency first, and the count-only yint reads its whole
// intervals from those sums, computing only its two end intervals.
// A pair with l >= 2 gives two list entries, its spheroidal part (with the
// radial mode for l = 0) and its toroidal part (yspec.f90:301-316), which
// are independent solves writing disjoint coefficients; so a warp runs one
// kind of system.  The cost of an entry is its counted FP64 work, sum over
// systems of steps x flops per step; the path class is the set of systems
// it integrates.  Entries are then sorted (CUB radix sort, descending) by
//   key = spheroidal first | log-cost bucket (1.1% wide) | path class | entry index,
// so a warp's 32 lanes take the same yint sequence with nearly the same
// number of steps, the persistent kernel takes the costliest first, and
// the spheroidal and toroidal stepping code do not compete for an SM's
// instruction cache except where the two parts meet.
// Entry value: event << 48 | part << 47 | l index << 24 | j - 1 (part 1 =
// toroidal).
#define YSG_COUNT_ONLY 1
#include "ysg_kernels.h"
#include "ysg_solvers.cuh"

#include <cub/device/device_radix_sort.cuh>

namespace ysg {

namespace {

__device__ __forceinline__ int event_of(const long long* __restrict__ off, int nev, long long p)
{
    int lo = 0, hi = nev;                  // off[lo] <= p < off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= p) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Step counts of the whole knot intervals at every frequency of every
// event, summed: row r = poff[e] + j - 1 (frequency j of event e) holds
// pfx[r (nknot + 1) + k] = sum over intervals 1 .. k-1 of the steps yint
// takes across the interval (zero for a zero-length one), the same
// arithmetic as yint's.  The count-only yint then needs only its two end
// intervals.  One warp per row: 32 intervals at a time, prefix-summed by
// shuffles.
__global__ void __launch_bounds__(128) k_step_prefix(const Knot* __restrict__ kn, const ModelHdr* __restrict__ mh,
                                                     const EventDev* __restrict__ evs,
                                                     const long long* __restrict__ poff, int nev,
                                                     int* __restrict__ pfx)
{
    const long long nrow = poff[nev];
    const int n = mh->nknot;
    const int lane = threadIdx.x & 31;
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long r = w0; r < nrow; r += nwarp) {        // uniform across the warp
        const int e = event_of(poff, nev, r);
        const EventDev& ev = evs[e];
        const int j = (int)(r - poff[e]) + 1;
        Ctx c;
        c.kn = kn;
        c.mh = mh;
        c.pfx = nullptr;
        set_omega(c, omega_of(ev, j));
        int* row = pfx + (size_t)r * (n + 1);
        if (lane == 0) row[0] = row[1] = 0;
        int carry = 0;
        for (int base = 1; base <= n - 1; base += 32) {
            const int i = base + lane;
            int cnt = 0;
            if (i <= n - 1) {
                const double h = kn[i + 1].r - kn[i].r;
                if (h != 0.0) cnt = 1 + (int)fmin(floor(fabs(h) / steps(c, i)), 4194304.0);
            }
            int incl = cnt;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += v;
            }
            if (i <= n - 1) row[i + 1] = carry + incl;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
}

__global__ void __launch_bounds__(128) k_pair_cost(const Knot* __restrict__ kn, const Seg* __restrict__ sg,
                                                   const ModelHdr* __restrict__ mh,
                                                   const EventDev* __restrict__ evs,
                                                   const long long* __restrict__ off, int nev,
                                                   const long long* __restrict__ poff,
                                                   const int* __restrict__ pfx, StepCost sc,
                                                   unsigned long long* __restrict__ keys,
                                                   unsigned long long* __restrict__ vals)
{
    const long long np = off[nev];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < 2 * np;
         q += (long long)gridDim.x * blockDim.x) {
        const long long p = q >> 1;
        const int part = (int)(q & 1);
        const int e = event_of(off, nev, p);
        const EventDev& ev = evs[e];
        const long long local = p - off[e];
        const int li = (int)(local / ev.nw);
        const int j = (int)(local - (long long)li * ev.nw) + 1;
        const int l = ev.lmin + li;
        Ctx c;
        c.kn = kn;
        c.mh = mh;
        c.pib = mh->pibigg;
        c.sg = sg;
        c.kb = nullptr;
        c.ats = (double)ev.ats;
        c.pfx = pfx + (size_t)(poff[e] + j - 1) * (mh->nknot + 1);
        for (int q = 0; q < NSYS; q++) c.nst[q] = 0;
        cd out[NCOEF];
        if (part == 1) {
            if (l > 1) pair_toroidal(c, ev, l, j, out + 10);
        } else if (l == 0) {
            pair_radial(c, ev, j, out);
        } else {
            pair_spheroidal(c, ev, l, j, out, out + 5);
        }
        double cost = sc.base;
        unsigned cls = 0;
        for (int s = 0; s < NSYS; s++) {
            cost += (double)c.nst[s] * sc.flops[s];
            if (c.nst[s]) cls |= 1u << s;
        }
        // an l < 2 pair has no toroidal part: its entry sorts last and is skipped
        const bool none = part == 1 && l < 2;
        unsigned bucket = none ? 0u : (unsigned)fmax(1.0, fmin(4095.0, 64.0 * log2(cost)));
        keys[q] = ((unsigned long long)(part == 0) << 63) | ((unsigned long long)bucket << 51) |
                  ((unsigned long long)cls << 43) | ((unsigned long long)q & ((1ull << 43) - 1));
        vals[q] = none ? ~0ull
                       : ((unsigned long long)e << 48) | ((unsigned long long)part << 47) |
                             ((unsigned long long)li << 24) | (unsigned long long)(j - 1);
    }
}

// The sort orders the key from bit 43 up (part, cost bucket, path class);
// the entry index below it is a tie-break, and a stable radix sort keeps
// equal keys in their input order, which is event-major already.
constexpr int kSortBegin = 43;

}  // namespace

size_t pair_sort_tmp_bytes(long long npairs)
{
    size_t bytes = 0;
    cub::DoubleBuffer<unsigned long long> k(nullptr, nullptr), v(nullptr, nullptr);
    cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, k, v, (int)(2 * npairs), kSortBegin, 64);
    return bytes;
}

cudaError_t launch_pair_schedule(const Knot* kn, const Seg* sg, const ModelHdr* mh,
                                 const EventDev* evs, const long long* off, int nev, long long npairs,
                                 const long long* poff, long long nrows, int* pfx,
                                 const StepCost& sc, unsigned long long* keys[2],
                                 unsigned long long* vals[2], void* tmp, size_t tmp_bytes,
                                 unsigned long long** sorted, cudaStream_t st)
{
    if (npairs <= 0) return cudaSuccess;
    if (2 * npairs >= (1ll << 31)) return cudaErrorInvalidValue;
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    long long pblocks = (nrows + 3) / 4;          // four rows (warps) per block
    if (pblocks > (long long)nsm * 16) pblocks = (long long)nsm * 16;
    if (pblocks < 1) pblocks = 1;
    k_step_prefix<<<(unsigned)pblocks, 128, 0, st>>>(kn, mh, evs, poff, nev, pfx);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    long long blocks = (2 * npairs + 127) / 128;
    if (blocks > (long long)nsm * 16) blocks = (long long)nsm * 16;
    k_pair_cost<<<(unsigned)blocks, 128, 0, st>>>(kn, sg, mh, evs, off, nev, poff, pfx, sc, keys[0], vals[0]);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cub::DoubleBuffer<unsigned long long> k(keys[0], keys[1]), v(vals[0], vals[1]);
    e = cub::DeviceRadixSort::SortPairsDescending(tmp, tmp_bytes, k, v, (int)(2 * npairs), kSortBegin, 64, st);
    if (e != cudaSuccess) return e;
    *sorted = v.Current();
    return cudaSuccess;
}

}  // namespace ysg
