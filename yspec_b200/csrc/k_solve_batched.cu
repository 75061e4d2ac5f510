// k_solve_batched.cu -- batched persistent solve stage.
//
// Same per-pair work as the plain form (yspec.f90:259-400 for one
// (omega_j, l)), organised for the B200:
//   * one thread per pair, but the Cash-Karp stage vectors of the
//     14-component minor / b-vector systems live in a per-thread slab of
//     shared memory: four slots of 14 complex values (896 bytes), the stages
//     folded into partial sums as they are produced (ysg_ode.cuh
//     rkck_step_loop), interleaved across the lanes of a warp so accesses
//     are bank-conflict free and every offset is a constant; y and the
//     stage input stay in registers.  Four 64-thread blocks (57 KB each)
//     fill an SM's 228 KB of shared memory -- two warps on every SMSP --
//     once the kernel asks for the largest shared-memory carveout.  The
//     plain form keeps all stage vectors in local memory, which spills
//     through L1 into L2.
//   * a persistent grid (resident blocks only) pulls work items from an
//     atomic counter, one item per warp.  Schedule 0: an item is (event, l,
//     32 consecutive frequencies); the lanes share l and step through
//     nearly identical radial grids; items are ordered by a cost estimate,
//     most expensive first (longest-processing-time first), so the tail is
//     short.  Schedule 1: an item is 32 pairs of equal code path and
//     near-equal exact cost from the sorted list of k_schedule.cu, so the
//     lanes of a warp finish together.
//   * items may come from several events (different frequency grids,
//     degrees, sources, switches) sharing one model: one launch serves a
//     whole batch.
#define YSG_SMEM_STAGES 1
#include "ysg_kernels.h"
#include "ysg_solvers.cuh"

namespace ysg {

constexpr int SLAB = 4 * 14;     // complex entries per thread (four stage slots)

// Four 64-thread blocks per SM (shared memory admits four), each thread
// with the full 255 registers.
template <int SCHED>
__global__ void __launch_bounds__(64, 4) k_solve_batched(const Knot* __restrict__ kn,
                                                      const Seg* __restrict__ sg,
                                                      const ModelHdr* __restrict__ mh,
                                                      const EventDev* __restrict__ evs,
                                                      cd* const* __restrict__ coefs,
                                                      const int4* __restrict__ items,
                                                      const unsigned long long* __restrict__ pairs,
                                                      long long npairs, int nitems, int* counter,
                                                      unsigned long long* __restrict__ work)
{
    // the slab is all the shared memory a block has: four blocks fill the SM
    extern __shared__ cd slab[];
    const int lane = threadIdx.x & 31;
    Ctx c;
    c.kn = kn;
    c.mh = mh;
    c.pib = mh->pibigg;
    c.sg = sg;
    c.kb = slab + (threadIdx.x >> 5) * (SLAB * KS) + lane;
    for (int q = 0; q < NSYS; q++) c.nst[q] = 0;
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= nitems) break;
        int e, li, j, part = 2;             // part: 0 spheroidal, 1 toroidal, 2 both
        if (SCHED == 0) {
            const int4 w = items[it];
            e = w.x;
            li = w.y;
            j = w.z + lane + 1;
            if (j > evs[e].nw) continue;
        } else {
            const long long p = (long long)it * 32 + lane;
            if (p >= 2 * npairs) continue;
            const unsigned long long v = pairs[p];
            if (v == ~0ull) continue;           // l < 2 has no toroidal entry
            e = (int)(v >> 48);
            part = (int)((v >> 47) & 1u);
            li = (int)((v >> 24) & 0x7fffffu);
            j = (int)(v & 0xffffffu) + 1;
        }
        const EventDev& ev = evs[e];
        const int l = ev.lmin + li;
        c.ats = (double)ev.ats;
        cd out[NCOEF];
        int q0 = 0, q1 = NCOEF;             // coefficients this entry writes
        if (part == 1) {
            pair_toroidal(c, ev, l, j, out + 10);
            q0 = 10;
        } else if (l == 0) {
            pair_radial(c, ev, j, out);
        } else {
            if (part == 2 && l > 1) pair_toroidal(c, ev, l, j, out + 10);
            else
                for (int q = 10; q < 15; q++) out[q] = mk(0.0);
            pair_spheroidal(c, ev, l, j, out, out + 5);
            if (part == 0 && l > 1) q1 = 10;
        }
        cd* dst = coefs[e] + (size_t)li * NCOEF * ev.nw + (j - 1);
        for (int q = q0; q < q1; q++) dst[(size_t)q * ev.nw] = out[q];
    }
    for (int q = 0; q < NSYS; q++) {
        unsigned long long v = c.nst[q];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0 && v) atomicAdd(&work[q], v);
    }
}

namespace {

constexpr int kBlock = 64;

using SolveFn = void (*)(const Knot*, const Seg*, const ModelHdr*, const EventDev*, cd* const*,
                         const int4*, const unsigned long long*, long long, int, int*,
                         unsigned long long*);

SolveFn solve_fn(int sched) { return sched == 1 ? k_solve_batched<1> : k_solve_batched<0>; }

size_t solve_smem() { return (size_t)kBlock * SLAB * sizeof(cd); }

}  // namespace

int solve_batched_blocks(int variant)
{
    int dev = 0, nsm = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 0;
    SolveFn f = solve_fn(variant);
    // the largest carveout: four slabs need all 228 KB of the SM's shared memory
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem()) !=
            cudaSuccess ||
        cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, f, kBlock, solve_smem()) != cudaSuccess)
        return 0;
    if (per < 1) per = 1;
    return nsm * per;
}

cudaError_t launch_solve_batched(int variant, const Knot* kn, const Seg* sg, const ModelHdr* mh,
                                 const EventDev* evs_dev, cd* const* coefs_dev, const int4* items,
                                 const unsigned long long* pairs, long long npairs, int nitems,
                                 int* counter, unsigned long long* work, int nblocks, cudaStream_t st)
{
    if (nitems <= 0) return cudaSuccess;
    SolveFn f = solve_fn(variant);
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem());
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    f<<<nblocks, kBlock, solve_smem(), st>>>(kn, sg, mh, evs_dev, coefs_dev, items, pairs, npairs,
                                             nitems, counter, work);
    return cudaGetLastError();
}

}  // namespace ysg
