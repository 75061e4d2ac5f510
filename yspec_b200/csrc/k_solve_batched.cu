// k_solve_batched.cu -- batched persistent solve stage.
//
// Same per-pair work as the plain form (yspec.f90:259-400 for one
// (omega_j, l)), organised for the B200:
//   * one thread per pair, but the five Cash-Karp stage vectors of the
//     14-component minor / b-vector systems live in a per-thread slab of
//     shared memory (70 complex entries, interleaved across the lanes of a
//     warp so accesses are bank-conflict free and every offset is a
//     constant); y and the stage input stay in registers.  The plain form
//     keeps them in local memory, which spills through L1 into L2.
//   * a persistent grid (resident blocks only) pulls work items from an
//     atomic counter.  An item is (event, l, 32 consecutive frequencies):
//     the lanes of a warp share l and step through nearly identical radial
//     grids.  Items are ordered by predicted cost, most expensive first
//     (longest-processing-time first), so the tail is short.
//   * items may come from several events (different frequency grids,
//     degrees, sources, switches) sharing one model: one launch serves a
//     whole batch.
#define YSG_SMEM_STAGES 1
#include "ysg_kernels.h"
#include "ysg_solvers.cuh"

namespace ysg {

constexpr int SLAB = 5 * 14;     // complex entries per thread

__global__ void __launch_bounds__(64) k_solve_batched(const Knot* __restrict__ kn,
                                                      const Seg* __restrict__ sg, ModelHdr mh_in,
                                                      const EventDev* __restrict__ evs,
                                                      cd* const* __restrict__ coefs,
                                                      const int4* __restrict__ items, int nitems,
                                                      int* counter,
                                                      unsigned long long* __restrict__ work)
{
    extern __shared__ cd slab[];
    __shared__ ModelHdr mh;
    if (threadIdx.x == 0) mh = mh_in;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    Ctx c;
    c.kn = kn;
    c.mh = &mh;
    c.sg = sg;
    c.kb = slab + (threadIdx.x >> 5) * (SLAB * KS) + lane;
    for (int q = 0; q < NSYS; q++) c.nst[q] = 0;
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= nitems) break;
        const int4 w = items[it];
        const EventDev& ev = evs[w.x];
        const int li = w.y;
        const int j = w.z + lane + 1;
        if (j > ev.nw) continue;
        const int l = ev.lmin + li;
        c.ats = (double)ev.ats;
        cd out[NCOEF];
        if (l == 0) {
            pair_radial(c, ev, j, out);
        } else {
            if (l > 1) pair_toroidal(c, ev, l, j, out + 10);
            else
                for (int q = 10; q < 15; q++) out[q] = mk(0.0);
            pair_spheroidal(c, ev, l, j, out, out + 5);
        }
        cd* dst = coefs[w.x] + (size_t)li * NCOEF * ev.nw + (j - 1);
        for (int q = 0; q < NCOEF; q++) dst[(size_t)q * ev.nw] = out[q];
    }
    for (int q = 0; q < NSYS; q++) {
        unsigned long long v = c.nst[q];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0 && v) atomicAdd(&work[q], v);
    }
}

size_t solve_batched_smem(int block) { return (size_t)block * SLAB * sizeof(cd); }

int solve_batched_blocks(int block)
{
    int dev = 0, nsm = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_solve_batched, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)solve_batched_smem(block));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_solve_batched, block,
                                                  solve_batched_smem(block));
    if (per < 1) per = 1;
    return nsm * per;
}

cudaError_t launch_solve_batched(const Knot* kn, const Seg* sg, const ModelHdr& mh,
                                 const EventDev* evs_dev,
                                 cd* const* coefs_dev, const int4* items, int nitems, int* counter,
                                 unsigned long long* work, int nblocks, int block, cudaStream_t st)
{
    if (nitems <= 0) return cudaSuccess;
    size_t smem = solve_batched_smem(block);
    cudaError_t e = cudaFuncSetAttribute(k_solve_batched, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    k_solve_batched<<<nblocks, block, smem, st>>>(kn, sg, mh, evs_dev, coefs_dev, items, nitems,
                                                 counter, work);
    return cudaGetLastError();
}

}  // namespace ysg
