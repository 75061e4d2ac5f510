// k_solve_plain.cu -- plain solve stage: one thread per (omega_j, l) pair,
// one event per launch.  The (omega,l) double loop of yspec.f90:250-426
// with the pairs laid out l-major; each thread runs the whole pair (radial
// or toroidal + spheroidal) and writes uu(1:5), vv(1:5), ww(1:5).
#include "ysg_kernels.h"
#include "ysg_solvers.cuh"
#include "ysg_tma.cuh"

namespace ysg {

__global__ void __launch_bounds__(128) k_solve_plain(const Knot* __restrict__ kn_g,
                                                     const Seg* __restrict__ sg, ModelHdr mh,
                                                     EventDev ev, cd* __restrict__ coef,
                                                     unsigned long long* __restrict__ work,
                                                     int* status)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int nrec = mh.nknot + 2;                       // records 0..nknot+1
    Knot* kn = reinterpret_cast<Knot*>(smem_raw);
    ModelHdr* mhs = reinterpret_cast<ModelHdr*>(smem_raw + (size_t)nrec * sizeof(Knot));
    uint64_t* mbar = reinterpret_cast<uint64_t*>(mhs + 1);
    if (threadIdx.x == 0) *mhs = mh;
    if (!stage_to_smem(kn, kn_g, (uint32_t)(nrec * sizeof(Knot)), mbar, status)) return;

    const int L = ev.lmax - ev.lmin + 1;
    const long long total = (long long)L * ev.nw;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    Ctx c;
    c.kn = kn;
    c.mh = mhs;
    c.pib = mh.pibigg;
    c.ats = (double)ev.ats;
    c.sg = sg;
    c.kb = nullptr;
    for (int q = 0; q < NSYS; q++) c.nst[q] = 0;
    if (gid < total) {
        const int li = (int)(gid / ev.nw);
        const int j = (int)(gid - (long long)li * ev.nw) + 1;
        const int l = ev.lmin + li;
        cd out[NCOEF];
        if (l == 0) {
            pair_radial(c, ev, j, out);
        } else {
            if (l > 1) pair_toroidal(c, ev, l, j, out + 10);
            else
                for (int q = 10; q < 15; q++) out[q] = mk(0.0);
            pair_spheroidal(c, ev, l, j, out, out + 5);
        }
        cd* dst = coef + (size_t)li * NCOEF * ev.nw + (j - 1);
        for (int q = 0; q < NCOEF; q++) dst[(size_t)q * ev.nw] = out[q];
    }
    // step counters: warp reduction then one atomic per warp
    for (int q = 0; q < NSYS; q++) {
        unsigned long long v = c.nst[q];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&work[q], v);
    }
}

size_t solve_plain_smem(int nknot)
{
    return (size_t)(nknot + 2) * sizeof(Knot) + sizeof(ModelHdr) + 16;
}

cudaError_t launch_solve_plain(const Knot* kn, const Seg* sg, const ModelHdr& mh, const EventDev& ev,
                               cd* coef,
                               unsigned long long* work, int* status, cudaStream_t st)
{
    const long long total = (long long)(ev.lmax - ev.lmin + 1) * ev.nw;
    if (total <= 0) return cudaSuccess;
    const int bs = 128;
    const long long nb = (total + bs - 1) / bs;
    size_t smem = solve_plain_smem(mh.nknot);
    cudaError_t e = cudaFuncSetAttribute(k_solve_plain, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    k_solve_plain<<<(unsigned)nb, bs, smem, st>>>(kn, sg, mh, ev, coef, work, status);
    return cudaGetLastError();
}

}  // namespace ysg
