// ysg_kernels.h -- launchers of the device stages, used by the C-ABI layer.
#pragma once
#include <cuda_runtime.h>
#include "ysg_model.cuh"

namespace ysg {

// step-counter classes of the solve stage (see ysg_ode.cuh)
constexpr int NSYS_COUNT = 8;

// K1 plain: one thread per (omega,l) pair of one event.
size_t solve_plain_smem(int nknot);
cudaError_t launch_solve_plain(const Knot* kn, const Seg* sg, const ModelHdr& mh, const EventDev& ev,
                               cd* coef, unsigned long long* work, int* status, cudaStream_t st);

// K1 tangent-linear: dual numbers, one launch over slots 0..nslot-1 (their
// EventDev records and coefficient buffers in device arrays); slot s takes
// direction s of the ndir derivative tables (nknot + 2 knot records and
// nknot + 1 segments each), or direction 0 when ndir is 1, and receives the
// derivative coefficients.  One thread per entry of `pairs`, the nentries
// sorted entries of launch_pair_schedule over the same slots.
cudaError_t launch_solve_tangent(const Knot* kn, const Seg* sg, const Knot* dkn, const Seg* dsg,
                                 int ndir, const ModelHdr* mh, const EventDev* evs_dev,
                                 cd* const* coefs_dev, const unsigned long long* pairs,
                                 long long nentries, unsigned long long* work, cudaStream_t st);

// K1 batched persistent: work items (event, l index, first frequency - 1)
// of one or more events, one thread per (omega,l) pair, stage vectors in
// shared memory.  counter must be device memory (reset by the launcher).
// Schedules of the batched solver: 0 = tiles of (event, l, 32 consecutive
// frequencies) from `items`; 1 = lists of 32 entries from `pairs` (2 npairs
// entries, the spheroidal and toroidal part of each pair, packed event << 48
// | part << 47 | l index << 24 | j - 1, sorted by launch_pair_schedule with
// every spheroidal entry first); 2 = the same list as two concurrent
// launches, the spheroidal entries [0, npairs) and the toroidal ones
// [npairs, 2 npairs) with a small-slab kernel on a side stream.
// Kernels (k_solve_batched.cu): kid 0 tiles, 1 pair lists (all parts),
// 2 pair lists (spheroidal part), 3 pair lists (toroidal part).  A kernel
// takes work items item0 .. item_end-1 (entries p = item 32 + lane in
// [plo, phi) for the lists) from the device counter, which it resets.
constexpr int NSCHED = 3;
constexpr int NSOLVE_KERNELS = 4;
int solve_kernel_blocks(int kid);
cudaError_t launch_solve_kernel(int kid, const Knot* kn, const Seg* sg, const ModelHdr* mh,
                                const EventDev* evs_dev, cd* const* coefs_dev, const int4* items,
                                const unsigned long long* pairs, long long plo, long long phi,
                                int item0, int item_end, int* counter, unsigned long long* work,
                                int nblocks, cudaStream_t st);

// Pair cost model and ordering for schedule 1 (k_schedule.cu).  off[e] is
// the flat index of event e's first pair (off[nev] = npairs); keys and vals
// are two pairs of npairs-element buffers; *sorted receives the buffer
// holding the packed pairs in schedule order.
struct StepCost {
    double flops[NSYS_COUNT];    // FP64 work per Cash-Karp step, per system class
    double base;                 // per-pair work outside the stepping
};
size_t pair_sort_tmp_bytes(long long npairs);
// poff[e] is the first row of event e in the per-frequency step table pfx
// (poff[nev] = nrows = sum of the events' nw; pfx holds nrows x (nknot + 1)
// ints, filled here).
cudaError_t launch_pair_schedule(const Knot* kn, const Seg* sg, const ModelHdr* mh,
                                 const EventDev* evs, const long long* off, int nev, long long npairs,
                                 const long long* poff, long long nrows, int* pfx,
                                 const StepCost& sc, unsigned long long* keys[2],
                                 unsigned long long* vals[2], void* tmp, size_t tmp_bytes,
                                 unsigned long long** sorted, cudaStream_t st);

// K2: Legendre table, T[((l * nr) + k) * 8 + q].
cudaError_t launch_legendre(int nr, int lmax, const double* delta, const double* ct,
                            const double* st, double* T, cudaStream_t s);

// K3: receiver l-sum.  coef (nw, 15, L) complex; T as above; E (5, nr)
// complex powers e^{i m azst}, m = -2..2; outputs (nw, nr) complex.
cudaError_t launch_lsum(int nw, int nr, int lmin, int lmax, const cd* coef, const double* T,
                        const cd* E, cd* ur, cd* ut, cd* up, cudaStream_t s);

// K4: filter + Hermitian extension + inverse FFT + post-processing.
struct TraceDev {
    int nt, i1, i2, nw, nr, nout, log2n, b1;
    double dt, scale, t_norm, amp_norm;
};
size_t ifft_scratch_bytes(int nt, int nr);
cudaError_t launch_ifft(const TraceDev& td, const cd* ur, const cd* ut, const cd* up,
                        const double* filt, const cd* tw, const double* expt,
                        const double* cs_azep, cd* scratch, double* out, cudaStream_t s);

// Reverse mode (k_solve_adjoint.cu).  Work space of the reverse sweeps,
// interleaved over threads: thread t's scratch step log (nmax steps: the
// replayed integrations), chain step log (ncmax steps: the minor chain from
// the start level to the source, logged in the forward pass) and grid log
// (gmax points of the l = 0 gravity solve), entry e of an array at
// e * nthreads + t.
constexpr int ADJ_THREADS = 128;
struct AdjStepArrays {
    cd* y;             // n x 14 states
    double* x;         // n radii
    double* h;         // n step sizes
    int* il;           // n intervals
    double* f;         // n rescaling factors
    int n;
};
struct AdjLogs {
    AdjStepArrays s, c;  // scratch and chain step logs
    cd* gy;            // gmax x 4 states
    double* gr;        // gmax radii
    int* gi;           // gmax intervals
    int gmax;
    int nthreads;      // a multiple of ADJ_THREADS
};
inline size_t adj_step_bytes(int n) { return (size_t)n * (14 * sizeof(cd) + 3 * sizeof(double) + sizeof(int)); }
inline size_t adj_log_bytes(int nmax, int ncmax, int gmax)
{
    return adj_step_bytes(nmax) + adj_step_bytes(ncmax) + (size_t)gmax * (4 * sizeof(cd) + sizeof(double) + sizeof(int));
}
// resident blocks of k_solve_adjoint over the device (0 on failure)
int solve_adjoint_blocks();
// Time stage on the 2 nw basis spectra (k_basis) with azimuth 0: bout
// (nout, 4, 2 nw); basis holds 2 nw * nw complex, scratch
// ifft_scratch_bytes(nt, 2 nw) bytes, cs0 2 nw (cos, sin) = (1, 0) pairs.
cudaError_t launch_time_basis(const TraceDev& td, cd* basis, const double* filt, const cd* tw,
                              const double* expt, const double* cs0, cd* scratch, double* bout, cudaStream_t st);
// Trace adjoint gout (nout, 4, nr) -> spectrum adjoints sbar (3 x (nw, nr)).
cudaError_t launch_spec_adjoint(int nw, int nr, int nout, const double* bout, const double* gout, const double* cs,
                                cd* sbar, cudaStream_t st);
// Spectrum adjoints -> coefficient adjoints coefb ((nw, 15, L) complex).
cudaError_t launch_lsum_adjoint(int nw, int nr, int lmin, int lmax, const double* T, const cd* E, const cd* sbar,
                                cd* coefb, cudaStream_t st);
// Reverse sweeps of the l >= 1 entries of `pairs` (one event,
// launch_pair_schedule's list; w needs no grid log): grad ((nknot + 1) x
// NPARAM x 4 doubles, zeroed by the caller) receives dL/dc[i][p][k]; status
// bit 0 is set if a sweep failed.  launch_radial_adjoint: the l = 0 pairs,
// one thread per frequency (w with grid logs).
cudaError_t launch_radial_adjoint(const Knot* kn, const Seg* sg, const ModelHdr* mh, const EventDev* ev,
                                  const UnitDirs& u, const cd* coefb, const AdjLogs& w, double* grad, int* status,
                                  cudaStream_t st);
cudaError_t launch_solve_adjoint(const Knot* kn, const Seg* sg, const ModelHdr* mh, const EventDev* ev,
                                 const UnitDirs& u, const cd* coefb, const unsigned long long* pairs,
                                 long long nentries, const AdjLogs& w, double* grad,
                                 unsigned long long* counter, int* status, cudaStream_t st);

}  // namespace ysg
