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
//     lanes of a warp finish together.  Schedule 2: the same list run by two
//     kernels, one for the spheroidal / radial entries and one for the
//     toroidal entries, whose 2-component system needs an eighth of the slab
//     and fewer registers, so more warps share an SM.
//   * items may come from several events (different frequency grids,
//     degrees, sources, switches) sharing one model: one launch serves a
//     whole batch.
#define YSG_SMEM_STAGES 1
#include "ysg_kernels.h"
#include "ysg_solvers.cuh"

namespace ysg {

// Launch shape per PART (which entries a kernel runs: 2 = every part of
// every pair, 0 = spheroidal / radial entries only, 1 = toroidal entries
// only).  The kernels that run 14-component systems need four slots of 14
// complex values per thread: four 64-thread blocks fill the SM's shared
// memory, each thread with the full 255 registers.  The toroidal-only
// kernel steps a 2-component system: a small slab and a register budget of
// 96 let twenty warps share an SM.  Its few hundred bytes of spills cost
// less than the occupancy gains: on c2 it beat 168 registers without spills
// (twelve warps) and 128 registers (sixteen warps).
template <int PART>
struct SolveCfg {
    static constexpr int BLOCK = 64, MINB = 4, SLAB = 4 * 14;
};
template <>
struct SolveCfg<1> {
    static constexpr int BLOCK = 128, MINB = 5, SLAB = 4 * 2;
};

template <int SCHED, int PART>
__global__ void __launch_bounds__(SolveCfg<PART>::BLOCK, SolveCfg<PART>::MINB)
    k_solve_batched(const Knot* __restrict__ kn, const Seg* __restrict__ sg,
                    const ModelHdr* __restrict__ mh, const EventDev* __restrict__ evs,
                    cd* const* __restrict__ coefs, const int4* __restrict__ items,
                    const unsigned long long* __restrict__ pairs, long long plo, long long phi,
                    int item0, int item_end, int* counter, unsigned long long* __restrict__ work)
{
    constexpr int SLAB = SolveCfg<PART>::SLAB;
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
        if (lane == 0) it = item0 + atomicAdd(counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= item_end) break;
        int e, li, j, part = 2;             // part: 0 spheroidal, 1 toroidal, 2 both
        if (SCHED == 0) {
            const int4 w = items[it];
            e = w.x;
            li = w.y;
            j = w.z + lane + 1;
            if (j > evs[e].nw) continue;
        } else {
            const long long p = (long long)it * 32 + lane;
            if (p < plo || p >= phi) continue;
            const unsigned long long v = pairs[p];
            if (v == ~0ull) continue;           // l < 2 has no toroidal entry
            e = (int)(v >> 48);
            part = (int)((v >> 47) & 1u);
            li = (int)((v >> 24) & 0x7fffffu);
            j = (int)(v & 0xffffffu) + 1;
            if (PART != 2 && part != PART) continue;
        }
        const EventDev& ev = evs[e];
        const int l = ev.lmin + li;
        c.ats = (double)ev.ats;
        cd out[NCOEF];
        int q0 = 0, q1 = NCOEF;             // coefficients this entry writes
        if constexpr (PART == 1) {
            pair_toroidal(c, ev, l, j, out + 10);
            q0 = 10;
        } else {
            if (PART == 2 && part == 1) {
                pair_toroidal(c, ev, l, j, out + 10);
                q0 = 10;
            } else if (l == 0) {
                pair_radial(c, ev, j, out);
            } else {
                if (PART == 2 && part == 2 && l > 1) pair_toroidal(c, ev, l, j, out + 10);
                else
                    for (int q = 10; q < 15; q++) out[q] = mk(0.0);
                pair_spheroidal(c, ev, l, j, out, out + 5);
                if (part == 0 && l > 1) q1 = 10;
            }
        }
        cd* dst = coefs[e] + (size_t)li * NCOEF * ev.nw + (j - 1);
        // streaming stores: the coefficients are not read again in this
        // launch, so they should not push the threads' stack frames out of L2
        for (int q = q0; q < q1; q++)
            __stcs(reinterpret_cast<double2*>(dst + (size_t)q * ev.nw), make_double2(out[q].x, out[q].y));
    }
    for (int q = 0; q < NSYS; q++) {
        unsigned long long v = c.nst[q];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0 && v) atomicAdd(&work[q], v);
    }
}

namespace {

using SolveFn = void (*)(const Knot*, const Seg*, const ModelHdr*, const EventDev*, cd* const*,
                         const int4*, const unsigned long long*, long long, long long, int, int,
                         int*, unsigned long long*);

struct KernelDesc {
    SolveFn f;
    int block;
    size_t smem;
};

template <int SCHED, int PART>
KernelDesc desc()
{
    return {k_solve_batched<SCHED, PART>, SolveCfg<PART>::BLOCK,
            (size_t)SolveCfg<PART>::BLOCK * SolveCfg<PART>::SLAB * sizeof(cd)};
}

KernelDesc kernel(int kid)
{
    switch (kid) {
        case 1: return desc<1, 2>();
        case 2: return desc<1, 0>();
        case 3: return desc<1, 1>();
        default: return desc<0, 2>();
    }
}

}  // namespace

int solve_kernel_blocks(int kid)
{
    int dev = 0, nsm = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 0;
    const KernelDesc k = kernel(kid);
    // the largest carveout: the 14-component kernels need all 228 KB of shared memory
    if (cudaFuncSetAttribute(k.f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k.f, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k.f, k.block, k.smem) != cudaSuccess)
        return 0;
    if (per < 1) per = 1;
    return nsm * per;
}

cudaError_t launch_solve_kernel(int kid, const Knot* kn, const Seg* sg, const ModelHdr* mh,
                                const EventDev* evs_dev, cd* const* coefs_dev, const int4* items,
                                const unsigned long long* pairs, long long plo, long long phi,
                                int item0, int item_end, int* counter, unsigned long long* work,
                                int nblocks, cudaStream_t st)
{
    if (item_end <= item0) return cudaSuccess;
    const KernelDesc k = kernel(kid);
    cudaError_t e = cudaFuncSetAttribute(k.f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    k.f<<<nblocks, k.block, k.smem, st>>>(kn, sg, mh, evs_dev, coefs_dev, items, pairs, plo, phi, item0,
                                          item_end, counter, work);
    return cudaGetLastError();
}

}  // namespace ysg
