// k_solve_adjoint.cu -- reverse mode of the synthetics of one event: the
// gradient of L = sum_t,k,c gout[t, c, k] traces[t, c, k] with respect to
// the uploaded earth model.  No reference counterpart: the reference has no
// derivatives.
//
// The stages after the solves are linear, so their transposes carry the
// trace adjoint back to the adjoints of the uu / vv / ww coefficients of
// every (omega, l) pair; the reverse sweep of each pair's solve
// (ysg_pair_adjoint.cuh) then adds its contribution to dL/dc[i][p][k], the
// gradient with respect to the power-form spline segments of the model.
//
//   k_basis, then the time stage (launch_ifft) on the basis: the time
//       stage's response to a unit real / imaginary spectrum at every
//       frequency (its matrix, from the forward code itself);
//   k_spec_adjoint: time stage and rotation to Z/N/E transposed, with that
//       response: trace adjoint -> spectrum adjoint;
//   k_lsum_adjoint: the l-sum (k_lsum.cu) transposed: spectrum adjoint ->
//       coefficient adjoint;
//   k_solve_adjoint: one reverse sweep per entry of the pair schedule's
//       cost-sorted list (k_schedule.cu), persistent, a warp fetching 32
//       consecutive entries at a time.
//
// Complex adjoints follow one convention throughout: for a real L and a
// complex z, zb = dL/dRe z - i dL/dIm z, so dL = Re(sum zb dz) and a
// complex-linear map is transposed without conjugation.
// The primal solves of the sweep take the looped Cash-Karp step: the kernel
// holds every system's replay, reverse step and tangent start / source
// evaluations, and its instruction footprint, not its registers, limits it.
#define YSG_LOOPED_STEP 1
#include "ysg_kernels.h"
#include "ysg_pair_adjoint.cuh"

namespace ysg {

// Basis spectra: row b < nw is the unit at frequency b, row nw + b is i
// times it ((nw, 2 nw) complex, frequency fastest).
__global__ void k_basis(int nw, cd* __restrict__ spec)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = 2LL * nw * nw;
    if (e >= n) return;
    const int b = (int)(e / nw), j = (int)(e - (long long)b * nw);
    spec[e] = b == j ? mk(1.0) : (b == j + nw ? mk(0.0, 1.0) : mk(0.0));
}

// Spectrum adjoints of receiver k = blockIdx.y at frequency j.  bout is the
// time stage's output on the basis with azimuth 0 ((nout, 4, 2 nw): Z =
// T_r, N = -T_t, E = T_p of the unit spectrum); gout (nout, 4, nr) the
// trace adjoint; cs the receivers' cos / sin of azep.  With
// N = -t1 ca + t2 sa, E = t1 sa + t2 ca (t1 from ut, t2 from up):
//   sb_c[j] = sum_t g_c(t) T_c(e_j)(t) - i sum_t g_c(t) T_c(i e_j)(t).
__global__ void k_spec_adjoint(int nw, int nr, int nout, const double* __restrict__ bout,
                               const double* __restrict__ gout, const double* __restrict__ cs,
                               cd* __restrict__ sbar)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (j >= nw || k >= nr) return;
    const double ca = cs[2 * k], sa = cs[2 * k + 1];
    const double* g = gout + (size_t)nout * 4 * k;
    const double* bre = bout + (size_t)nout * 4 * j;
    const double* bim = bout + (size_t)nout * 4 * (nw + j);
    double xr = 0.0, yr = 0.0, xt = 0.0, yt = 0.0, xp = 0.0, yp = 0.0;
    for (int t = 0; t < nout; t++) {
        const double gz = g[nout + t], gn = g[2 * nout + t], ge = g[3 * nout + t];
        const double g1 = ge * sa - gn * ca, g2 = gn * sa + ge * ca;
        xr += gz * bre[nout + t];
        yr += gz * bim[nout + t];
        xt -= g1 * bre[2 * nout + t];
        yt -= g1 * bim[2 * nout + t];
        xp += g2 * bre[3 * nout + t];
        yp += g2 * bim[3 * nout + t];
    }
    const size_t nspec = (size_t)nw * nr, o = (size_t)k * nw + j;
    sbar[o] = mk(xr, -yr);
    sbar[nspec + o] = mk(xt, -yt);
    sbar[2 * nspec + o] = mk(xp, -yp);
}

// Coefficient adjoints of pair (l index blockIdx.y, frequency j): the
// transpose of k_lsum's sums, term for term.
__global__ void k_lsum_adjoint(int nw, int nr, int lmin, const double* __restrict__ T,
                               const cd* __restrict__ E, const cd* __restrict__ sbar, cd* __restrict__ coefb)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int li = blockIdx.y;
    if (j >= nw) return;
    cd acc[NCOEF];
    for (int q = 0; q < NCOEF; q++) acc[q] = mk(0.0);
    const size_t nspec = (size_t)nw * nr;
    for (int k = 0; k < nr; k++) {
        const double* x = T + ((size_t)(li + lmin) * nr + k) * 8;
        const size_t o = (size_t)k * nw + j;
        const cd sr = sbar[o], st = sbar[nspec + o], sp = sbar[2 * nspec + o];
        // m = 0: ur += uu_0 X_0, ut += vv_0 dX_0
        acc[2] += sr * x[0];
        acc[7] += st * x[3];
#pragma unroll
        for (int a = 1; a <= 2; a++) {
            const double X = x[a], XP = x[3 + a], XC = x[5 + a];
            const double sgn = (a & 1) ? -1.0 : 1.0;
#pragma unroll
            for (int sm = -1; sm <= 1; sm += 2) {
                const int m = sm * a;
                const int slot = m + 2;
                const double s = sm < 0 ? sgn : 1.0;
                const cd e = E[(size_t)k * 5 + slot];
                const cd er = e * sr, et = e * st, ep = e * sp;
                // ur += e uu s X; ut += e (vv s XP + i m s X ww); up += e (i m s XC vv - s XP ww)
                acc[slot] += er * (s * X);
                acc[5 + slot] += et * (s * XP) + imul(ep) * ((double)m * s * XC);
                acc[10 + slot] += imul(et) * ((double)m * s * X) - ep * (s * XP);
            }
        }
    }
    for (int q = 0; q < NCOEF; q++) coefb[((size_t)li * NCOEF + q) * nw + j] = acc[q];
}

// Thread tid's view of an interleaved step log.
__device__ __forceinline__ StepLog step_log(const AdjStepArrays& a, int tid, int nthreads)
{
    return StepLog{a.y + tid, a.x + tid, a.h + tid, a.il + tid, a.f + tid, a.n, nthreads};
}

__device__ __forceinline__ void adj_ctx(primal::Ctx& c, const Knot* kn, const Seg* sg, const ModelHdr* mh,
                                        const EventDev& ev)
{
    c.kn = kn;
    c.mh = mh;
    c.sg = sg;
    c.pib = mh->pibigg;
    c.ats = (double)ev.ats;
    c.kb = nullptr;
    for (int q = 0; q < primal::NSYS; q++) c.nst[q] = 0;
}

// Reverse sweeps of the l >= 1 entries (the l = 0 pairs go to
// k_radial_adjoint).  Thread tid owns scratch and chain step logs tid of
// the interleaved work space; the grid holds exactly w.nthreads threads.
// status bit 0: a sweep exceeded its logs.
__global__ void __launch_bounds__(ADJ_THREADS) k_solve_adjoint(
    const Knot* __restrict__ kn, const Seg* __restrict__ sg, const ModelHdr* __restrict__ mh,
    const EventDev* __restrict__ evp, UnitDirs u, const cd* __restrict__ coefb,
    const unsigned long long* __restrict__ pairs, long long nentries, AdjLogs w, double* __restrict__ grad,
    unsigned long long* __restrict__ counter, int* __restrict__ status)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    StepLog L = step_log(w.s, tid, w.nthreads), CL = step_log(w.c, tid, w.nthreads);
    const EventDev ev = *evp;
    SegGrad G;
    G.init(grad);
    primal::Ctx c;                               // the plain form of the solver code
    adj_ctx(c, kn, sg, mh, ev);
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(counter, 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= (unsigned long long)nentries) break;
        const unsigned long long e = base + (unsigned long long)lane;
        const unsigned long long v = e < (unsigned long long)nentries ? pairs[e] : ~0ull;
        if (v == ~0ull) continue;                 // l < 2 has no toroidal entry
        const int part = (int)((v >> 47) & 1u);   // 0 spheroidal / radial, 1 toroidal
        const int li = (int)((v >> 24) & 0x7fffffu);
        const int j = (int)(v & 0xffffffu) + 1;
        const int l = ev.lmin + li;
        if (l == 0) continue;
        const size_t o = (size_t)li * NCOEF * ev.nw + (j - 1);
        const int q0 = part == 1 ? 10 : 0, q1 = part == 1 ? NCOEF : 10;
        cd wb[NCOEF];
        bool any = false;
        for (int q = 0; q < NCOEF; q++) {
            wb[q] = (q >= q0 && q < q1) ? coefb[o + (size_t)q * ev.nw] : mk(0.0);
            any = any || wb[q].x != 0.0 || wb[q].y != 0.0;
        }
        if (!any) continue;                       // the pair does not reach L
        const bool ok = part == 1 ? pair_toroidal_adj(c, u, ev, l, j, wb + 10, L, CL, G)
                                  : pair_spheroidal_adj(c, u, ev, l, j, wb, wb + 5, L, CL, G);
        if (!ok) atomicOr(status, 1);
    }
    G.flush();
}

// Reverse sweeps of the l = 0 pairs (rad_solver_wg with its grid, or
// rad_solver_ng without gravity), one thread per frequency; thread tid owns
// scratch, chain and grid logs tid.
__global__ void __launch_bounds__(ADJ_THREADS) k_radial_adjoint(
    const Knot* __restrict__ kn, const Seg* __restrict__ sg, const ModelHdr* __restrict__ mh,
    const EventDev* __restrict__ evp, UnitDirs u, const cd* __restrict__ coefb, AdjLogs w,
    double* __restrict__ grad, int* __restrict__ status)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const EventDev ev = *evp;
    if (ev.lmin != 0) return;
    StepLog L = step_log(w.s, tid, w.nthreads), CL = step_log(w.c, tid, w.nthreads);
    GridLog GL{w.gy + tid, w.gr + tid, w.gi + tid, w.gmax, w.nthreads};
    SegGrad G;
    G.init(grad);
    primal::Ctx c;
    adj_ctx(c, kn, sg, mh, ev);
    for (int j = tid + 1; j <= ev.nw; j += w.nthreads) {
        cd wb[NCOEF];
        for (int q = 0; q < NCOEF; q++) wb[q] = coefb[(size_t)q * ev.nw + (j - 1)];
        if (wb[2].x == 0.0 && wb[2].y == 0.0) continue;   // only uu(3) comes from the radial solve
        if (!pair_radial_adj(c, u, ev, j, wb, L, CL, GL, G)) atomicOr(status, 1);
    }
    G.flush();
}

int solve_adjoint_blocks()
{
    int dev = 0, nsm = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_solve_adjoint, ADJ_THREADS, 0) != cudaSuccess)
        return 0;
    return nsm * std::max(per, 1);
}

cudaError_t launch_time_basis(const TraceDev& td, cd* basis, const double* filt, const cd* tw,
                              const double* expt, const double* cs0, cd* scratch, double* bout, cudaStream_t st)
{
    const long long n = 2LL * td.nw * td.nw;
    if (n <= 0) return cudaSuccess;
    k_basis<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(td.nw, basis);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    TraceDev tb = td;
    tb.nr = 2 * td.nw;
    return launch_ifft(tb, basis, basis, basis, filt, tw, expt, cs0, scratch, bout, st);
}

cudaError_t launch_spec_adjoint(int nw, int nr, int nout, const double* bout, const double* gout, const double* cs,
                                cd* sbar, cudaStream_t st)
{
    if (nr <= 0 || nw <= 0) return cudaSuccess;
    if (nr > 65535) return cudaErrorInvalidConfiguration;
    dim3 g((unsigned)((nw + 127) / 128), (unsigned)nr);
    k_spec_adjoint<<<g, 128, 0, st>>>(nw, nr, nout, bout, gout, cs, sbar);
    return cudaGetLastError();
}

cudaError_t launch_lsum_adjoint(int nw, int nr, int lmin, int lmax, const double* T, const cd* E, const cd* sbar,
                                cd* coefb, cudaStream_t st)
{
    const int L = lmax - lmin + 1;
    if (L <= 0 || nw <= 0) return cudaSuccess;
    if (L > 65535) return cudaErrorInvalidConfiguration;
    dim3 g((unsigned)((nw + 127) / 128), (unsigned)L);
    k_lsum_adjoint<<<g, 128, 0, st>>>(nw, nr, lmin, T, E, sbar, coefb);
    return cudaGetLastError();
}

cudaError_t launch_radial_adjoint(const Knot* kn, const Seg* sg, const ModelHdr* mh, const EventDev* ev,
                                  const UnitDirs& u, const cd* coefb, const AdjLogs& w, double* grad, int* status,
                                  cudaStream_t st)
{
    if (w.nthreads <= 0 || w.nthreads % ADJ_THREADS) return cudaErrorInvalidValue;
    k_radial_adjoint<<<(unsigned)(w.nthreads / ADJ_THREADS), ADJ_THREADS, 0, st>>>(kn, sg, mh, ev, u, coefb, w, grad,
                                                                                  status);
    return cudaGetLastError();
}

cudaError_t launch_solve_adjoint(const Knot* kn, const Seg* sg, const ModelHdr* mh, const EventDev* ev,
                                 const UnitDirs& u, const cd* coefb, const unsigned long long* pairs,
                                 long long nentries, const AdjLogs& w, double* grad,
                                 unsigned long long* counter, int* status, cudaStream_t st)
{
    if (nentries <= 0) return cudaSuccess;
    if (w.nthreads <= 0 || w.nthreads % ADJ_THREADS) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    k_solve_adjoint<<<(unsigned)(w.nthreads / ADJ_THREADS), ADJ_THREADS, 0, st>>>(
        kn, sg, mh, ev, u, coefb, pairs, nentries, w, grad, counter, status);
    return cudaGetLastError();
}

}  // namespace ysg
