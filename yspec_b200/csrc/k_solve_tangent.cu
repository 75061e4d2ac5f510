// k_solve_tangent.cu -- tangent-linear solve stage.
//
// The per-pair solve of yspec.f90:259-400 compiled with dual numbers
// (YSG_TANGENT, ysg_dual.cuh): every model value the solver reads comes with
// its derivative along one direction of the earth model (the tangent knot
// and segment tables), and each pair returns its uu / vv / ww coefficients
// together with their derivatives.  The start levels, step counts and
// rescaling decisions come from the value part, as in the primal solve.
//
// The l-sum, the filter, the inverse FFT and the post-processing that follow
// are linear in the coefficients, so running them on the derivative
// coefficients gives the derivative of the traces.  The kernel writes the
// derivative coefficients in the layout of the primal ones.
//
// The stage vectors live in local memory (the dual solve needs twice the
// state of the primal one).  One launch serves every slot of a batch, and
// slot s takes model direction s (or direction 0 when a single direction is
// loaded), so many directions of one event run as one batch of copies of it.
// One thread per entry of the cost-sorted list of the batched solver
// (k_schedule.cu: the spheroidal and the toroidal part of every pair of
// every slot, costliest first, equal paths side by side).  The cost of a
// solve is that of its value part, so the primal order serves the tangent
// solve.
#define YSG_TANGENT 1
#include "ysg_kernels.h"
#include "ysg_solvers.cuh"

namespace ysg {

__global__ void __launch_bounds__(128) k_solve_tangent(const Knot* __restrict__ kn,
                                                       const Seg* __restrict__ sg,
                                                       const Knot* __restrict__ dkn,
                                                       const Seg* __restrict__ dsg, int ndir,
                                                       const ModelHdr* __restrict__ mh,
                                                       const EventDev* __restrict__ evs,
                                                       cd* const* __restrict__ coefs,
                                                       const unsigned long long* __restrict__ pairs,
                                                       long long nentries,
                                                       unsigned long long* __restrict__ work)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned long long v = gid < nentries ? pairs[gid] : ~0ull;
    const bool active = v != ~0ull;           // l < 2 has no toroidal entry
    const int slot = active ? (int)(v >> 48) : 0;
    const int part = (int)((v >> 47) & 1u);   // 0 spheroidal / radial, 1 toroidal
    const int li = (int)((v >> 24) & 0x7fffffu);
    const int j = (int)(v & 0xffffffu) + 1;
    const int dir = ndir == 1 ? 0 : slot;
    const EventDev& ev = evs[slot];
    cd* const dcoef = coefs[slot];
    const int nknot = mh->nknot;
    Ctx c;
    c.kn = kn;
    c.mh = mh;
    c.pib = mh->pibigg;
    c.ats = (double)ev.ats;
    c.sg = sg;
    c.kb = nullptr;
    c.dkn = dkn + (size_t)dir * (nknot + 2);     // knot records 0..nknot+1
    c.dsg = dsg + (size_t)dir * (nknot + 1);     // segment records 0..nknot
    for (int q = 0; q < NSYS; q++) c.nst[q] = 0;
    if (active) {
        const int l = ev.lmin + li;
        mcplx out[NCOEF];
        int q0 = 0, q1 = NCOEF;               // coefficients this thread writes
        if (part == 1) {
            pair_toroidal(c, ev, l, j, out + 10);
            q0 = 10;
        } else if (l == 0) {
            pair_radial(c, ev, j, out);
        } else {
            for (int q = 10; q < 15; q++) out[q] = mk(0.0);
            pair_spheroidal(c, ev, l, j, out, out + 5);
            if (l > 1) q1 = 10;               // ww comes from the toroidal entry
        }
        const size_t o = (size_t)li * NCOEF * ev.nw + (j - 1);
        for (int q = q0; q < q1; q++) dcoef[o + (size_t)q * ev.nw] = out[q].d;
    }
    for (int q = 0; q < NSYS; q++) {
        unsigned long long v = c.nst[q];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&work[q], v);
    }
}

cudaError_t launch_solve_tangent(const Knot* kn, const Seg* sg, const Knot* dkn, const Seg* dsg,
                                 int ndir, const ModelHdr* mh, const EventDev* evs_dev,
                                 cd* const* coefs_dev, const unsigned long long* pairs,
                                 long long nentries, unsigned long long* work, cudaStream_t st)
{
    const int bs = 128;
    if (nentries <= 0) return cudaSuccess;
    const long long nb = (nentries + bs - 1) / bs;
    if (nb > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    k_solve_tangent<<<(unsigned)nb, bs, 0, st>>>(kn, sg, dkn, dsg, ndir, mh, evs_dev, coefs_dev, pairs,
                                                 nentries, work);
    return cudaGetLastError();
}

}  // namespace ysg
