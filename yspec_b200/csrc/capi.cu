// capi.cu -- the ysg_* C-ABI (include/yspec_gpu.h).
//
// Orchestrates the device stages of one event on the handle's stream:
//   K2 Legendre table -> K1 (omega,l) solves -> K3 receiver l-sum
//   -> K4 filter + inverse FFT + post-processing
// with CUDA events between stages for the per-stage device times.  Small
// host-side tables (cos/sin of the epicentral angles, e^{i m azst} powers,
// the taper, FFT twiddles, e^{eps t}) are formed here on the host, in FP64,
// as the reference forms them, and uploaded with each event.
//
// Internally every call is upload (host -> device, synchronous) followed by
// enqueue (kernels only, asynchronous) and finish (device -> host, counters).
// ysg_event_prepare / _execute / _fetch expose the three phases so a caller
// can time the device work alone.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <vector>

#include "yspec_gpu.h"
#include "ysg_kernels.h"

using namespace ysg;

namespace {

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes)
    {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess) cap = bytes;
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// Algorithmic FP64 flops of one Cash-Karp step per system class (index =
// Sys::CLS in ysg_ode.cuh): six right-hand sides plus the stage
// combinations (88 flops per complex component).  The per-RHS counts are
// hand tallies of the coefficient-matrix and derivative expressions.
const double kStepFlops[NSYS_COUNT] = {
    6 * 88.0 + 88.0 * 2,     // toroidal
    6 * 177.0 + 88.0 * 2,    // radial
    6 * 100.0 + 88.0 * 2,    // fluid minors, no gravity / Cowling
    6 * 290.0 + 88.0 * 4,    // b-vector, no gravity / Cowling
    6 * 300.0 + 88.0 * 5,    // solid minors, no gravity / Cowling
    6 * 240.0 + 88.0 * 5,    // fluid minors, self-gravitation
    6 * 666.0 + 88.0 * 14,   // solid minors, self-gravitation
    6 * 666.0 + 88.0 * 14,   // b-vector, self-gravitation
};

// Work of a pair outside the stepping (start level, start vectors, minor
// algebra, source vectors), for the scheduler's cost model only.
constexpr double kPairBaseFlops = 2.0e4;

// Workload signature of the autotuner: events, pairs (to 1%), largest
// degree and band, gravity switch of the first event, knots.
using Signature = std::array<long long, 6>;

// Device buffers and uploaded state of one event.  Slot 0 serves the
// single-event calls; a batch uses slots 0..nev-1.
struct Slot {
    DevBuf coef, leg, E, delta, ct, stv, spec, filt, tw, expt, cs, out;
    EventDev pev{};
    TraceDev ptd{};
    int nr = 0, lmax = 0;
    bool ev_ready = false, tm_ready = false;
    void release()
    {
        for (DevBuf* b : {&coef, &leg, &E, &delta, &ct, &stv, &spec, &filt, &tw, &expt, &cs, &out})
            b->release();
        ev_ready = tm_ready = false;
    }
};

}  // namespace

struct ysg_handle {
    int device = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev[6] = {};          // stage boundaries 0..4; 5 = end of an overlapped K2
    bool leg_overlap = false;        // K2 of the last single event ran beside K1
    int solver = 1;
    int pot_mode = 0;                // events uploaded in potential mode (ysg_event_potential)
    // model
    DevBuf kn, sg, hdr_dev;
    ModelHdr hdr{};
    std::vector<double> grav_host;   // knot gravity for the tilt correction
    std::vector<double> r_host;      // knot radii of the uploaded model
    std::vector<double> alpha_host;  // knot alpha (step counts) of the uploaded model
    bool has_model = false;
    DevBuf dkn, dsg;                 // model derivatives (directions) for the tangent solver
    int ndir = 0;                    // directions loaded; 0 = none
    // reverse mode: unit directions of the model (built on first use after
    // an upload), time-stage basis, adjoint buffers and sweep work space
    DevBuf ukn, usg;
    bool has_units = false;
    DevBuf abasis, about, ascr, acs0, agout, asbar, acoefb, agrad, alogs;
    // events
    std::vector<Slot> slots;
    int nactive = 0;                 // slots of the last prepare / batch
    // Side streams for the per-event kernels of a batch (K2, K3, K4 of
    // different events are independent); fork/join events order them with
    // the handle's stream, also under graph capture.  Each side stream has
    // its own inverse-FFT scratch rows.
    static constexpr int NSIDE = 4;
    cudaStream_t side[NSIDE] = {};
    cudaEvent_t fork_ev = nullptr, join_ev[NSIDE] = {};
    // A batch's trace copies run on their own stream: the copy of event e
    // waits only for the end of e's l-sum and time series (done_ev[e], an
    // event-record node of the batch graph), so it overlaps the later
    // events' stages.
    cudaStream_t copy_st = nullptr;
    cudaEvent_t copy_ev = nullptr;
    std::vector<cudaEvent_t> done_ev;
    DevBuf scratch[NSIDE];
    DevBuf work, status, items, counter, evdev, coefptr;
    int nitems = 0;                  // schedule-0 tiles
    bool tiles_ready = false;        // the tiles of the active slots are on the device
    long long npairs = 0;            // pairs of the active slots
    int nev_items = 0;               // slots the items were built for
    DevBuf offs, keys0, keys1, vals0, vals1, sort_tmp;
    DevBuf poff, pfx;                // per-frequency step table of the cost model (rows, table)
    long long nrows = 0;             // frequencies of the active slots
    int sched = -1;                  // batched-solver schedule; -1 = autotuned
    int cur_sched = 0;               // schedule of the next solve launch
    std::map<Signature, int> tuned;  // autotuner choices
    float tune_ms[NSCHED] = {};      // solve times of the last tuning run (per schedule)
    bool tune_warm = false;          // every schedule's kernels have been launched once
    long long launches = 0;          // this library's kernels enqueued since the last prepare
    int solve_blocks[NSOLVE_KERNELS] = {};   // resident grid per solve kernel
    bool has_spectra = false;
    // CUDA graph of the last batch (updated in place when the shape repeats)
    cudaGraphExec_t gexec = nullptr;
    bool capturing = false;          // enqueue_* run under stream capture
    float ms[4] = {0, 0, 0, 0};
    double h2d = 0.0, d2h = 0.0;     // bytes moved since the last prepare
    double pairs = 0.0, flops = 0.0;
};

// CUDA failures return YSG_ERR_CUDA and leave the runtime's error name and
// the failing call's source line for ysg_last_cuda_error().
thread_local char g_cuda_err[160] = "";

int ysg_cuda_fail_at(cudaError_t e, const char* file, int line)
{
    std::snprintf(g_cuda_err, sizeof g_cuda_err, "%s (%s) at %s:%d", cudaGetErrorName(e),
                  cudaGetErrorString(e), file, line);
    return YSG_ERR_CUDA;
}

int cuda_fail(cudaError_t e, int line) { return ysg_cuda_fail_at(e, "capi.cu", line); }

#define CK(x)                                                  \
    do {                                                       \
        cudaError_t e_ = (x);                                  \
        if (e_ != cudaSuccess) return cuda_fail(e_, __LINE__); \
    } while (0)

namespace {

// Stage timing event i.  Under stream capture a plain record only orders the
// captured work; cudaEventRecordExternal makes it an event-record node of the
// graph, so the stage times of a batch are measured like a single event's.
cudaError_t record(ysg_handle* h, int i)
{
    return cudaEventRecordWithFlags(h->ev[i], h->st,
                                    h->capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
}

int check_event(const ysg_handle* h, const ysg_event* ev)
{
    if (!h || !ev) return YSG_ERR_ARG;
    if (!h->has_model) return YSG_ERR_NO_MODEL;
    if (ev->lmin < 0 || ev->lmax < ev->lmin || ev->nw < 1 || ev->nr < 0) return YSG_ERR_ARG;
    if (ev->is < 1 || ev->ir < 1 || ev->is >= h->hdr.nknot || ev->ir >= h->hdr.nknot) return YSG_ERR_ARG;
    if (ev->nr > 0 && (!ev->delta || !ev->azst)) return YSG_ERR_ARG;
    if (ev->grav < 0 || ev->grav > 2 || ev->out < 0 || ev->out > 2) return YSG_ERR_ARG;
    if (!(ev->dw > 0.0) || !(ev->wmin > 0.0) || !(ev->ep > 0.0)) return YSG_ERR_ARG;
    if (ev->jofs < 0 || ev->jstride < 1) return YSG_ERR_ARG;
    return YSG_OK;
}

EventDev make_event(const ysg_handle* h, const ysg_event* ev)
{
    EventDev d{};
    d.lmin = ev->lmin;
    d.lmax = ev->lmax;
    d.nw = ev->nw;
    d.is = ev->is;
    d.ir = ev->ir;
    d.ats = ev->ats;
    d.grav = ev->grav;
    d.out = ev->out;
    d.cor = ev->cor;
    d.nr = ev->nr;
    d.jofs = ev->jofs;
    d.jstride = ev->jstride;
    d.rs = ev->rs;
    d.rr = ev->rr;
    d.ep = ev->ep;
    d.wmin = ev->wmin;
    d.dw = ev->dw;
    d.grav_ir = h->grav_host[(size_t)ev->ir - 1];
    d.pot = h->pot_mode;
    for (int i = 0; i < 6; i++) d.mm[i] = ev->mm[i];
    return d;
}

// integer power of a complex number as libgfortran's pow_c8_i4 forms it
cd cpowi(cd a, int m)
{
    cd pw = mk(1.0), x = a;
    if (m == 0) return pw;
    unsigned u;
    if (m < 0) {
        u = (unsigned)(-m);
        x = pw / x;
    } else {
        u = (unsigned)m;
    }
    for (;;) {
        if (u & 1) pw = pw * x;
        u >>= 1;
        if (u) x = x * x;
        else break;
    }
    return pw;
}

// Predicted relative cost of the pairs (l, omega_j .. omega_j+31) of an
// event: Cash-Karp steps grow with omega times the radial path integrated
// (start level below the turning radius up to the source, then the minor
// continuation and four b-vector passes from source to receiver) plus a
// per-interval floor.  Used only to order the work (longest first).
double item_cost(const EventDev& ev, int li, int j0)
{
    const int l = ev.lmin + li;
    const double w = ev.wmin + (ev.jofs + (j0 + 16) * ev.jstride) * ev.dw;
    const double vref = 1.0;                       // normalised wave speed scale
    double rturn = (l + 0.5) * vref / w;
    if (rturn > 1.0) rturn = 1.0;
    double below = ev.rs - 0.6 * rturn;
    if (below < 0.0) below = 0.0;
    double above = std::fabs(ev.rr - ev.rs);
    return 32.0 + w * (below + 5.0 * above) * 200.0;
}

struct Item {
    int ev, li, j0;
    double cost;
};

void build_items(std::vector<Item>& out, int e, const EventDev& ev)
{
    const int L = ev.lmax - ev.lmin + 1;
    for (int li = 0; li < L; li++)
        for (int j0 = 0; j0 < ev.nw; j0 += 32) out.push_back({e, li, j0, item_cost(ev, li, j0)});
}

// The schedule-0 tiles of slots 0..nev-1, longest first, built and uploaded
// only when a schedule-0 solve is about to run (a fixed or tuned schedule
// 0, or the autotuner's trial of it): the cost-sorted schedules 1 and 2
// never read them, and at c5 sizes the list has a million entries to sort.
int ensure_tiles(ysg_handle* h, int nev)
{
    if (h->tiles_ready) return YSG_OK;
    std::vector<Item> items;
    for (int e = 0; e < nev; e++) build_items(items, e, h->slots[(size_t)e].pev);
    std::stable_sort(items.begin(), items.end(),
                     [](const Item& a, const Item& b) { return a.cost > b.cost; });
    std::vector<int4> packed(items.size());
    for (size_t i = 0; i < items.size(); i++) packed[i] = make_int4(items[i].ev, items[i].li, items[i].j0, 0);
    CK(h->items.ensure(std::max<size_t>(packed.size(), 1) * sizeof(int4)));
    if (!packed.empty())
        CK(cudaMemcpyAsync(h->items.p, packed.data(), packed.size() * sizeof(int4), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));    // the host list goes out of scope
    h->h2d += (double)(packed.size() * sizeof(int4));
    h->nitems = (int)packed.size();
    h->tiles_ready = true;
    return YSG_OK;
}

int upload_items(ysg_handle* h, const std::vector<EventDev>& evs, const std::vector<cd*>& coefs)
{
    h->tiles_ready = false;
    h->nitems = 0;
    CK(h->items.ensure(sizeof(int4)));
    CK(h->evdev.ensure(std::max<size_t>(evs.size(), 1) * sizeof(EventDev)));
    CK(h->coefptr.ensure(std::max<size_t>(coefs.size(), 1) * sizeof(cd*)));
    CK(h->counter.ensure(2 * sizeof(int)));
    CK(cudaMemcpyAsync(h->evdev.p, evs.data(), evs.size() * sizeof(EventDev), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->coefptr.p, coefs.data(), coefs.size() * sizeof(cd*), cudaMemcpyHostToDevice, h->st));
    // flat pair offsets of the events and buffers of the pair schedule
    std::vector<long long> off(evs.size() + 1, 0);
    for (size_t e = 0; e < evs.size(); e++)
        off[e + 1] = off[e] + (long long)(evs[e].lmax - evs[e].lmin + 1) * evs[e].nw;
    const long long np = off.back();
    CK(h->offs.ensure(off.size() * sizeof(long long)));
    CK(cudaMemcpyAsync(h->offs.p, off.data(), off.size() * sizeof(long long), cudaMemcpyHostToDevice, h->st));
    // rows of the cost model's per-frequency step table
    std::vector<long long> poff(evs.size() + 1, 0);
    for (size_t e = 0; e < evs.size(); e++) poff[e + 1] = poff[e] + evs[e].nw;
    CK(h->poff.ensure(poff.size() * sizeof(long long)));
    CK(cudaMemcpyAsync(h->poff.p, poff.data(), poff.size() * sizeof(long long), cudaMemcpyHostToDevice, h->st));
    CK(h->pfx.ensure(std::max<size_t>((size_t)poff.back() * ((size_t)h->hdr.nknot + 1) * sizeof(int), 16)));
    h->nrows = poff.back();
    const size_t pb = (size_t)std::max<long long>(2 * np, 1) * sizeof(unsigned long long);
    CK(h->keys0.ensure(pb));
    CK(h->keys1.ensure(pb));
    CK(h->vals0.ensure(pb));
    CK(h->vals1.ensure(pb));
    CK(h->sort_tmp.ensure(std::max<size_t>(pair_sort_tmp_bytes(np), 16)));
    CK(cudaStreamSynchronize(h->st));
    h->h2d += (double)(evs.size() * sizeof(EventDev) + coefs.size() * sizeof(cd*) +
                       (off.size() + poff.size()) * sizeof(long long));
    h->npairs = np;
    h->nev_items = (int)evs.size();
    for (int v = 0; v < NSOLVE_KERNELS; v++) {
        if (h->solve_blocks[v] == 0) h->solve_blocks[v] = solve_kernel_blocks(v);
        if (h->solve_blocks[v] == 0) return YSG_ERR_CUDA;
    }
    return YSG_OK;
}

// Work items of the batched solver for slots 0..nev-1, longest first.
int upload_batch_items(ysg_handle* h, int nev)
{
    std::vector<EventDev> evs((size_t)nev);
    std::vector<cd*> coefs((size_t)nev);
    for (int e = 0; e < nev; e++) {
        evs[(size_t)e] = h->slots[(size_t)e].pev;
        coefs[(size_t)e] = h->slots[(size_t)e].coef.as<cd>();
    }
    return upload_items(h, evs, coefs);
}

// Event inputs to the device: cos/sin of delta and e^{i m azst}
// (yspec.f90:173-174, :331, :414); buffers sized.  No kernel runs.
int upload_event(ysg_handle* h, Slot& s, const ysg_event* ev)
{
    const int nr = ev->nr, nw = ev->nw, n1 = std::max(nr, 1);
    std::vector<double> ct(n1), stv(n1);
    std::vector<cd> E((size_t)n1 * 5);
    for (int k = 0; k < nr; k++) {
        ct[k] = std::cos(ev->delta[k]);
        stv[k] = std::sin(ev->delta[k]);
        cd eia = mk(std::cos(ev->azst[k]), std::sin(ev->azst[k]));
        for (int m = -2; m <= 2; m++) E[(size_t)k * 5 + (m + 2)] = cpowi(eia, m);
    }
    const int L = ev->lmax - ev->lmin + 1;
    s.ev_ready = s.tm_ready = false;
    CK(s.coef.ensure((size_t)L * NCOEF * nw * sizeof(cd)));
    CK(s.spec.ensure(3 * (size_t)nw * n1 * sizeof(cd)));
    CK(s.delta.ensure((size_t)n1 * sizeof(double)));
    CK(s.ct.ensure((size_t)n1 * sizeof(double)));
    CK(s.stv.ensure((size_t)n1 * sizeof(double)));
    CK(s.E.ensure((size_t)n1 * 5 * sizeof(cd)));
    CK(s.leg.ensure((size_t)(ev->lmax + 1) * n1 * 8 * sizeof(double)));
    if (nr > 0) {
        CK(cudaMemcpyAsync(s.delta.p, ev->delta, (size_t)nr * sizeof(double), cudaMemcpyHostToDevice, h->st));
        CK(cudaMemcpyAsync(s.ct.p, ct.data(), (size_t)nr * sizeof(double), cudaMemcpyHostToDevice, h->st));
        CK(cudaMemcpyAsync(s.stv.p, stv.data(), (size_t)nr * sizeof(double), cudaMemcpyHostToDevice, h->st));
        CK(cudaMemcpyAsync(s.E.p, E.data(), (size_t)nr * 5 * sizeof(cd), cudaMemcpyHostToDevice, h->st));
        h->h2d += (double)nr * (3 * sizeof(double) + 5 * sizeof(cd));
    }
    CK(cudaStreamSynchronize(h->st));   // the host vectors go out of scope
    s.pev = make_event(h, ev);
    s.nr = nr;
    s.lmax = ev->lmax;
    s.ev_ready = true;
    return YSG_OK;
}

// Time-stage inputs: taper (module_fourier.f90:96-116), twiddles with pi_d,
// e^{eps t} (yspec.f90:439-444), cos/sin of azep (:466-473).
int upload_time(ysg_handle* h, Slot& s, const ysg_time* tm, int nw)
{
    const int n = tm->nt, nr = tm->nr;
    if (n < 4 || (n & (n - 1)) || n > (1 << 20)) return YSG_ERR_ARG;
    if (tm->i2 - tm->i1 + 1 != nw || tm->i1 < 1 || tm->i2 > n) return YSG_ERR_ARG;
    if (nr > 0 && !tm->azep) return YSG_ERR_ARG;
    const int nout = ysg_trace_rows(tm);
    int p = 0;
    while ((1 << p) < n) p++;
    const double pi_d = (double)3.14159265358979323846f;
    std::vector<double> filt((size_t)n / 2 + 1, 1.0), expt(nout), cs(2 * (size_t)std::max(nr, 1));
    const double w1 = tm->f11, w2 = tm->f12, w3 = tm->f21, w4 = tm->f22;
    if (!(w1 == 0.0 && w2 == 0.0 && w3 == 0.0 && w4 == 0.0)) {
        double f = 0.0;
        for (int i = 1; i <= n / 2 + 1; i++) {
            double w = (double)(i - 1) * tm->df;
            if (w < w1) f = 0.0;
            else if (w >= w1 && w < w2) f = 0.5 * (1.0 - std::cos(pi_d * (w - w1) / (w2 - w1)));
            else if (w >= w2 && w < w3) f = 1.0;
            else if (w >= w3 && w < w4) f = 0.5 * (1.0 - std::cos(pi_d * (w4 - w) / (w4 - w3)));
            else if (w >= w4) f = 0.0;
            filt[(size_t)i - 1] = f;
        }
    }
    std::vector<cd> tw((size_t)n / 2);
    const double dth = pi_d / (double)(n / 2);     // exact: n/2 is a power of two
    for (int m = 0; m < n / 2; m++) {
        double a = (double)m * dth;
        tw[(size_t)m] = mk(std::cos(a), std::sin(a));
    }
    for (int i = 0; i < nout; i++) expt[(size_t)i] = std::exp(tm->ep * ((double)i * tm->dt));
    for (int k = 0; k < nr; k++) {
        cs[2 * (size_t)k] = std::cos(tm->azep[k]);
        cs[2 * (size_t)k + 1] = std::sin(tm->azep[k]);
    }
    s.tm_ready = false;
    CK(s.filt.ensure(filt.size() * sizeof(double)));
    CK(s.tw.ensure(tw.size() * sizeof(cd)));
    CK(s.expt.ensure(expt.size() * sizeof(double)));
    CK(s.cs.ensure(cs.size() * sizeof(double)));
    CK(h->scratch[0].ensure(std::max<size_t>(ifft_scratch_bytes(n, nr), 16)));
    CK(s.out.ensure(std::max<size_t>((size_t)nout * 4 * nr * sizeof(double), 16)));
    CK(cudaMemcpyAsync(s.filt.p, filt.data(), filt.size() * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(s.tw.p, tw.data(), tw.size() * sizeof(cd), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(s.expt.p, expt.data(), expt.size() * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(s.cs.p, cs.data(), cs.size() * sizeof(double), cudaMemcpyHostToDevice, h->st));
    h->h2d += (double)((filt.size() + expt.size() + cs.size()) * sizeof(double) + tw.size() * sizeof(cd));
    CK(cudaStreamSynchronize(h->st));
    TraceDev& td = s.ptd;
    td = TraceDev{};
    td.nt = n;
    td.i1 = tm->i1;
    td.i2 = tm->i2;
    td.nw = nw;
    td.nr = nr;
    td.nout = nout;
    td.log2n = p;
    td.b1 = 1 << ((p + 1) / 2);
    td.dt = tm->dt;
    td.scale = tm->dt * (double)n;
    td.t_norm = tm->t_norm;
    td.amp_norm = tm->amp_norm;
    s.tm_ready = true;
    return YSG_OK;
}

// K1 for slots 0..nev-1: one batched launch over all their items, or one
// plain launch per event.
int fork_side(ysg_handle* h, int nside);
int join_side(ysg_handle* h, int nside);

int enqueue_solve(ysg_handle* h, int nev)
{
    CK(cudaMemsetAsync(h->work.p, 0, NSYS_COUNT * sizeof(unsigned long long), h->st));
    CK(cudaMemsetAsync(h->status.p, 0, sizeof(int), h->st));
    if (h->solver == 0) {
        for (int e = 0; e < nev; e++) {
            const Slot& s = h->slots[(size_t)e];
            h->launches += 1;
            CK(launch_solve_plain(h->kn.as<Knot>(), h->sg.as<Seg>(), h->hdr, s.pev, s.coef.as<cd>(),
                                  h->work.as<unsigned long long>(), h->status.as<int>(), h->st));
        }
    } else if (h->solver == 2) {
        // slot s takes direction s, or the one direction loaded
        if (h->ndir == 0 || (h->ndir != 1 && h->ndir != nev)) return YSG_ERR_ARG;
        // the batched solver's cost-sorted entry list of the same slots
        // (its packing: slot < 2^16, l index < 2^23, frequency < 2^24)
        bool packable = nev <= 65535 && h->nev_items == nev;
        for (int e = 0; e < nev && packable; e++) {
            const EventDev& d = h->slots[(size_t)e].pev;
            packable = d.lmax - d.lmin + 1 < (1 << 23) && d.nw < (1 << 24);
        }
        if (!packable) return YSG_ERR_LIMIT;
        StepCost sc;
        for (int q = 0; q < NSYS_COUNT; q++) sc.flops[q] = kStepFlops[q];
        sc.base = kPairBaseFlops;
        unsigned long long* keys[2] = {h->keys0.as<unsigned long long>(), h->keys1.as<unsigned long long>()};
        unsigned long long* vals[2] = {h->vals0.as<unsigned long long>(), h->vals1.as<unsigned long long>()};
        unsigned long long* sorted = nullptr;
        h->launches += 3;            // k_step_prefix, k_pair_cost and the tangent solve (the radix sort is CUB's)
        CK(launch_pair_schedule(h->kn.as<Knot>(), h->sg.as<Seg>(), h->hdr_dev.as<ModelHdr>(),
                                h->evdev.as<EventDev>(), h->offs.as<long long>(), nev, h->npairs,
                                h->poff.as<long long>(), h->nrows, h->pfx.as<int>(), sc, keys, vals,
                                h->sort_tmp.p, h->sort_tmp.cap, &sorted, h->st));
        CK(launch_solve_tangent(h->kn.as<Knot>(), h->sg.as<Seg>(), h->dkn.as<Knot>(), h->dsg.as<Seg>(),
                                h->ndir, h->hdr_dev.as<ModelHdr>(), h->evdev.as<EventDev>(),
                                h->coefptr.as<cd*>(), sorted, 2 * h->npairs,
                                h->work.as<unsigned long long>(), h->st));
    } else {
        const int s = h->cur_sched;
        const unsigned long long* pairs = nullptr;
        if (s >= 1) {
            StepCost sc;
            for (int q = 0; q < NSYS_COUNT; q++) sc.flops[q] = kStepFlops[q];
            sc.base = kPairBaseFlops;
            unsigned long long* keys[2] = {h->keys0.as<unsigned long long>(), h->keys1.as<unsigned long long>()};
            unsigned long long* vals[2] = {h->vals0.as<unsigned long long>(), h->vals1.as<unsigned long long>()};
            unsigned long long* sorted = nullptr;
            h->launches += 2;        // k_step_prefix and k_pair_cost (the radix sort is CUB's)
            CK(launch_pair_schedule(h->kn.as<Knot>(), h->sg.as<Seg>(), h->hdr_dev.as<ModelHdr>(),
                                    h->evdev.as<EventDev>(), h->offs.as<long long>(), h->nev_items,
                                    h->npairs, h->poff.as<long long>(), h->nrows, h->pfx.as<int>(), sc, keys,
                                    vals, h->sort_tmp.p, h->sort_tmp.cap, &sorted, h->st));
            pairs = sorted;
        }
        const long long np = h->npairs;
        int* ctr = h->counter.as<int>();
        auto launch = [&](int kid, long long plo, long long phi, int i0, int i1, int* cnt) {
            h->launches += 1;
            return launch_solve_kernel(kid, h->kn.as<Knot>(), h->sg.as<Seg>(), h->hdr_dev.as<ModelHdr>(),
                                       h->evdev.as<EventDev>(), h->coefptr.as<cd*>(), h->items.as<int4>(),
                                       pairs, plo, phi, i0, i1, cnt, h->work.as<unsigned long long>(),
                                       h->solve_blocks[kid], h->st);
        };
        if (s == 0) {
            CK(launch(0, 0, 0, 0, h->nitems, ctr));
        } else if (s == 1) {
            CK(launch(1, 0, 2 * np, 0, (int)((2 * np + 31) / 32), ctr));
        } else {
            // Spheroidal entries sort first (k_schedule.cu): [0, np), then the
            // toroidal ones.  The two parts write disjoint coefficients: the
            // toroidal launch runs on a side stream and takes SMs as the
            // spheroidal kernel drains.
            int rc = fork_side(h, 1);
            if (rc) return rc;
            CK(launch(2, 0, np, 0, (int)((np + 31) / 32), ctr));
            cudaStream_t main = h->st;
            h->st = h->side[0];
            const cudaError_t e2 = launch(3, np, 2 * np, (int)(np / 32), (int)((2 * np + 31) / 32), ctr + 1);
            h->st = main;
            CK(e2);
            if ((rc = join_side(h, 1))) return rc;
        }
    }
    return YSG_OK;
}

// Choose the batched solver's schedule for the active slots.  A fixed
// schedule (ysg_set_schedule) is used as is; otherwise the autotuner looks
// up the workload signature and, the first time it is seen, runs the solve
// stage once with each schedule (timed with CUDA events on the stream) and
// keeps the faster.  Every schedule computes every pair with the same
// per-thread arithmetic, so the coefficients do not depend on the choice.
int resolve_schedule(ysg_handle* h, int nev)
{
    if (h->solver != 1) return YSG_OK;
    // schedule 1 packs an entry as event (16 bits) | part | l index (23) | j - 1 (24)
    bool packable = nev <= 65535;
    for (int e = 0; e < nev && packable; e++) {
        const EventDev& d = h->slots[(size_t)e].pev;
        packable = d.lmax - d.lmin + 1 < (1 << 23) && d.nw < (1 << 24);
    }
    if (!packable) {
        h->cur_sched = 0;
        return ensure_tiles(h, nev);
    }
    if (h->sched >= 0) {
        h->cur_sched = h->sched;
        return h->sched == 0 ? ensure_tiles(h, nev) : YSG_OK;
    }
    long long maxl = 0, maxw = 0;
    for (int e = 0; e < nev; e++) {
        maxl = std::max<long long>(maxl, h->slots[(size_t)e].pev.lmax);
        maxw = std::max<long long>(maxw, h->slots[(size_t)e].pev.nw);
    }
    long long q = h->npairs;                   // two significant digits
    long long scale = 1;
    while (q >= 100) {
        q /= 10;
        scale *= 10;
    }
    const Signature sig = {nev, q * scale, maxl, maxw, h->slots[0].pev.grav, h->hdr.nknot};
    auto it = h->tuned.find(sig);
    if (it != h->tuned.end()) {
        h->cur_sched = it->second;
        return it->second == 0 ? ensure_tiles(h, nev) : YSG_OK;
    }
    int rc0 = ensure_tiles(h, nev);     // the trials include schedule 0
    if (rc0) return rc0;
    // The first tuning of a handle runs each schedule once untimed: with lazy
    // module loading a kernel's first launch also loads its module on the
    // host, which would be charged to whichever schedule launches it first.
    if (!h->tune_warm) {
        for (int s = 0; s < NSCHED; s++) {
            h->cur_sched = s;
            int rc = enqueue_solve(h, nev);
            if (rc) return rc;
        }
        CK(cudaStreamSynchronize(h->st));
        h->tune_warm = true;
    }
    int best = 0;
    for (int s = 0; s < NSCHED; s++) {
        h->cur_sched = s;
        CK(record(h, 1));
        int rc = enqueue_solve(h, nev);
        if (rc) return rc;
        CK(record(h, 2));
        CK(cudaStreamSynchronize(h->st));
        CK(cudaEventElapsedTime(&h->tune_ms[s], h->ev[1], h->ev[2]));
        if (h->tune_ms[s] < h->tune_ms[best]) best = s;
    }
    h->tuned[sig] = best;
    h->cur_sched = best;
    return YSG_OK;
}

// Streams of a stage group over nev slots: the handle's stream alone for one
// event, else `nside` side streams forked from it (slot e on side e % nside).
int fork_side(ysg_handle* h, int nside)
{
    CK(cudaEventRecord(h->fork_ev, h->st));
    for (int i = 0; i < nside; i++) CK(cudaStreamWaitEvent(h->side[i], h->fork_ev, 0));
    return YSG_OK;
}

int join_side(ysg_handle* h, int nside)
{
    for (int i = 0; i < nside; i++) {
        CK(cudaEventRecord(h->join_ev[i], h->side[i]));
        CK(cudaStreamWaitEvent(h->st, h->join_ev[i], 0));
    }
    return YSG_OK;
}

int side_count(int nev) { return nev > 1 ? std::min(nev, (int)ysg_handle::NSIDE) : 0; }

cudaStream_t stream_of(ysg_handle* h, int nside, int e) { return nside ? h->side[e % nside] : h->st; }

// K2 (all slots) -> K1 -> K3 (all slots), with timing events between the
// stage groups; no host synchronisation.  The per-event kernels of a group
// run on the side streams.
int enqueue_spectra(ysg_handle* h, int nev, bool lsum = true)
{
    const int ns = side_count(nev);
    CK(record(h, 0));
    int rc = YSG_OK;
    // One event outside stream capture: the Legendre table, which only the
    // l-sum reads, runs on side stream 1 beside the cost model and the
    // solves (schedule 2 uses side stream 0); the l-sum waits for it.
    h->leg_overlap = ns == 0 && !h->capturing;
    if (h->leg_overlap) {
        Slot& s = h->slots[0];
        CK(cudaEventRecord(h->fork_ev, h->st));
        CK(cudaStreamWaitEvent(h->side[1], h->fork_ev, 0));
        h->launches += s.nr > 0 ? 1 : 0;
        CK(launch_legendre(s.nr, s.lmax, s.delta.as<double>(), s.ct.as<double>(), s.stv.as<double>(),
                           s.leg.as<double>(), h->side[1]));
        CK(cudaEventRecord(h->ev[5], h->side[1]));
        CK(cudaEventRecord(h->join_ev[1], h->side[1]));
    } else {
        rc = ns ? fork_side(h, ns) : YSG_OK;
        if (rc) return rc;
        for (int e = 0; e < nev; e++) {
            Slot& s = h->slots[(size_t)e];
            h->launches += s.nr > 0 ? 1 : 0;
            CK(launch_legendre(s.nr, s.lmax, s.delta.as<double>(), s.ct.as<double>(), s.stv.as<double>(),
                               s.leg.as<double>(), stream_of(h, ns, e)));
        }
        if (ns && (rc = join_side(h, ns))) return rc;
    }
    CK(record(h, 1));
    rc = enqueue_solve(h, nev);
    if (rc) return rc;
    CK(record(h, 2));
    if (!lsum) return YSG_OK;        // the l-sums follow per event (enqueue_chains)
    if (h->leg_overlap) CK(cudaStreamWaitEvent(h->st, h->join_ev[1], 0));
    if (ns && (rc = fork_side(h, ns))) return rc;
    for (int e = 0; e < nev; e++) {
        Slot& s = h->slots[(size_t)e];
        const EventDev& d = s.pev;
        const size_t nspec = (size_t)d.nw * std::max(s.nr, 1);
        cd* d_ur = s.spec.as<cd>();
        h->launches += s.nr > 0 ? 1 : 0;
        CK(launch_lsum(d.nw, s.nr, d.lmin, d.lmax, s.coef.as<cd>(), s.leg.as<double>(), s.E.as<cd>(),
                       d_ur, d_ur + nspec, d_ur + 2 * nspec, stream_of(h, ns, e)));
    }
    if (ns && (rc = join_side(h, ns))) return rc;
    CK(record(h, 3));
    return YSG_OK;
}

// Scratch rows for the K4 group of slots 0..nev-1: one buffer per side
// stream while they fit a 4 GiB budget, else fewer streams.
int ensure_ifft_scratch(ysg_handle* h, int nev, int* nside)
{
    size_t need = 16;
    for (int e = 0; e < nev; e++) {
        const TraceDev& td = h->slots[(size_t)e].ptd;
        need = std::max(need, ifft_scratch_bytes(td.nt, td.nr));
    }
    int ns = side_count(nev);
    const size_t budget = (size_t)4 << 30;
    while (ns > 1 && need * (size_t)ns > budget) ns--;
    if (ns == 1) ns = 0;                 // one buffer: the group runs in order on the handle's stream
    for (int i = 0; i < std::max(ns, 1); i++) CK(h->scratch[i].ensure(need));
    *nside = ns;
    return YSG_OK;
}

// K4 for slots 0..nev-1 (scratch sized by ensure_ifft_scratch, or by
// upload_time for one event); `ns` side streams, 0 = the handle's stream.
int enqueue_traces(ysg_handle* h, int nev, int ns)
{
    CK(record(h, 3));
    int rc = ns ? fork_side(h, ns) : YSG_OK;
    if (rc) return rc;
    for (int e = 0; e < nev; e++) {
        Slot& s = h->slots[(size_t)e];
        const TraceDev& td = s.ptd;
        const size_t nspec = (size_t)td.nw * std::max(td.nr, 1);
        const cd* d_ur = s.spec.as<cd>();
        h->launches += td.nr > 0 ? 3 : 0;   // pass A, pass B, rotation
        CK(launch_ifft(td, d_ur, d_ur + nspec, d_ur + 2 * nspec, s.filt.as<double>(), s.tw.as<cd>(),
                       s.expt.as<double>(), s.cs.as<double>(), h->scratch[ns ? e % ns : 0].as<cd>(),
                       s.out.as<double>(), stream_of(h, ns, e)));
    }
    if (ns && (rc = join_side(h, ns))) return rc;
    CK(record(h, 4));
    return YSG_OK;
}

// A batch's K3 and K4 as one chain per event (slot e on side stream e % ns,
// each with its own scratch rows; ns = 0: all on the handle's stream), the
// end of each chain recorded as done_ev[e] for its trace copy.  Timing: the
// two stages share one interval, [2] of ysg_last_timings, and [3] is empty.
int enqueue_chains(ysg_handle* h, int nev, int ns)
{
    int rc = ns ? fork_side(h, ns) : YSG_OK;
    if (rc) return rc;
    for (int e = 0; e < nev; e++) {
        Slot& s = h->slots[(size_t)e];
        const EventDev& d = s.pev;
        const TraceDev& td = s.ptd;
        const size_t nspec = (size_t)d.nw * std::max(s.nr, 1);
        cd* d_ur = s.spec.as<cd>();
        cudaStream_t st = stream_of(h, ns, e);
        h->launches += s.nr > 0 ? 4 : 0;    // l-sum, pass A, pass B, rotation
        CK(launch_lsum(d.nw, s.nr, d.lmin, d.lmax, s.coef.as<cd>(), s.leg.as<double>(), s.E.as<cd>(),
                       d_ur, d_ur + nspec, d_ur + 2 * nspec, st));
        CK(launch_ifft(td, d_ur, d_ur + nspec, d_ur + 2 * nspec, s.filt.as<double>(), s.tw.as<cd>(),
                       s.expt.as<double>(), s.cs.as<double>(), h->scratch[ns ? e % ns : 0].as<cd>(),
                       s.out.as<double>(), st));
        CK(cudaEventRecordWithFlags(h->done_ev[(size_t)e], st, cudaEventRecordExternal));
    }
    if (ns && (rc = join_side(h, ns))) return rc;
    CK(record(h, 3));
    CK(record(h, 4));
    return YSG_OK;
}

// Wait for the stream, read the solve counters and the status word.
int finish(ysg_handle* h, int nev, bool spectra, bool traces)
{
    unsigned long long w[NSYS_COUNT] = {};
    int status = 0;
    if (spectra) {
        CK(cudaMemcpyAsync(w, h->work.p, sizeof w, cudaMemcpyDeviceToHost, h->st));
        CK(cudaMemcpyAsync(&status, h->status.p, sizeof status, cudaMemcpyDeviceToHost, h->st));
    }
    CK(cudaStreamSynchronize(h->st));
    if (spectra) {
        double fl = 0.0;
        for (int q = 0; q < NSYS_COUNT; q++) fl += (double)w[q] * kStepFlops[q];
        h->flops = fl;
        double pairs = 0.0;
        for (int e = 0; e < nev; e++) {
            const EventDev& d = h->slots[(size_t)e].pev;
            pairs += (double)(d.lmax - d.lmin + 1) * d.nw;
        }
        h->pairs = pairs;
        // K2's time: to the end of the table, on its own stream when overlapped
        CK(cudaEventElapsedTime(&h->ms[0], h->ev[0], h->ev[h->leg_overlap ? 5 : 1]));
        CK(cudaEventElapsedTime(&h->ms[1], h->ev[1], h->ev[2]));
        CK(cudaEventElapsedTime(&h->ms[2], h->ev[2], h->ev[3]));
        h->has_spectra = status == 0;
    }
    if (traces) CK(cudaEventElapsedTime(&h->ms[3], h->ev[3], h->ev[4]));
    return status ? YSG_ERR_DEVICE_WAIT : YSG_OK;
}

int copy_out(ysg_handle* h, const Slot& s, double* out, int* nout, cudaStream_t st = nullptr)
{
    const TraceDev& td = s.ptd;
    if (nout) *nout = td.nout;
    if (out && td.nr > 0) {
        CK(cudaMemcpyAsync(out, s.out.p, (size_t)td.nout * 4 * td.nr * sizeof(double),
                           cudaMemcpyDeviceToHost, st ? st : h->st));
        h->d2h += (double)td.nout * 4 * td.nr * sizeof(double);
    }
    return YSG_OK;
}

Slot& slot0(ysg_handle* h)
{
    if (h->slots.empty()) h->slots.resize(1);
    return h->slots[0];
}

// Upload one event into slot 0 (and its work items for the batched solver).
int prepare_single(ysg_handle* h, const ysg_event* ev)
{
    Slot& s = slot0(h);
    int rc = upload_event(h, s, ev);
    if (rc) return rc;
    h->nactive = 1;
    if (h->solver == 1) {
        rc = upload_batch_items(h, 1);
        if (!rc) rc = resolve_schedule(h, 1);
        return rc;
    }
    if (h->solver == 2) return upload_batch_items(h, 1);
    return YSG_OK;
}

// Capture the whole batch (K2, K1, K3, K4 of slots 0..nev-1) into a CUDA
// graph and launch it.  A graph of the same shape as the previous batch
// updates the instantiated one in place.
int launch_batch_graph(ysg_handle* h, int nev)
{
    int ns4 = 0;
    int rc0 = ensure_ifft_scratch(h, nev, &ns4);
    if (rc0) return rc0;
    // several events: K3 and K4 chained per event, so that each event's
    // trace copy can start while the others are still in their stages
    const bool chain = nev > 1;
    while (chain && h->done_ev.size() < (size_t)nev) {
        cudaEvent_t e = nullptr;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        h->done_ev.push_back(e);
    }
    CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeRelaxed));
    h->capturing = true;
    int rc = enqueue_spectra(h, nev, !chain);
    if (!rc) rc = chain ? enqueue_chains(h, nev, ns4) : enqueue_traces(h, nev, ns4);
    h->capturing = false;
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(h->st, &g);
    if (rc || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return rc ? rc : YSG_ERR_CUDA;
    }
    bool updated = false;
    if (h->gexec) {
        cudaGraphExecUpdateResultInfo info;
        updated = cudaGraphExecUpdate(h->gexec, g, &info) == cudaSuccess;
        if (!updated) {
            cudaGetLastError();
            cudaGraphExecDestroy(h->gexec);
            h->gexec = nullptr;
        }
    }
    if (!updated) {
        ce = cudaGraphInstantiate(&h->gexec, g, 0);
        if (ce != cudaSuccess) {
            h->gexec = nullptr;
            cudaGraphDestroy(g);
            return YSG_ERR_CUDA;
        }
    }
    cudaGraphDestroy(g);
    CK(cudaGraphLaunch(h->gexec, h->st));
    return YSG_OK;
}

// Knot records and power-form segments (ysg_model.cuh) of the 13 spline
// parameters on radii r.  The segment coefficients are linear in the knot
// values and second derivatives, so the same construction applied to their
// derivatives gives the derivative tables of the tangent solver.
void build_tables(int n, const double* r, const double* const* val, const double* const* cs,
                  const double* alpha, const double* beta, std::vector<Knot>& rec, std::vector<Seg>& seg)
{
    rec.assign((size_t)n + 2, Knot{});
    std::memset(rec.data(), 0, rec.size() * sizeof(Knot));
    for (int i = 0; i < n; i++) {
        Knot& k = rec[(size_t)i + 1];
        k.r = r[i];
        k.alpha = alpha ? alpha[i] : 0.0;
        k.beta = beta ? beta[i] : 0.0;
        for (int p = 0; p < NPARAM; p++) {
            k.v[p][0] = val[p][i];
            k.v[p][1] = cs[p][i];
        }
        knot_derive(k);
    }
    seg.assign((size_t)n + 1, Seg{});
    std::memset(seg.data(), 0, seg.size() * sizeof(Seg));
    for (int i = 1; i < n; i++) {
        Seg& s = seg[(size_t)i];
        const Knot &a = rec[(size_t)i], &b = rec[(size_t)i + 1];
        const double hh = b.r - a.r;
        s.r0 = a.r;
        for (int p = 0; p < NPARAM; p++) {
            s.c[p][0] = a.v[p][0];
            if (hh == 0.0) continue;
            s.c[p][1] = (b.v[p][0] - a.v[p][0]) / hh - hh * (2.0 * a.v[p][1] + b.v[p][1]) / 6.0;
            s.c[p][2] = 0.5 * a.v[p][1];
            s.c[p][3] = (b.v[p][1] - a.v[p][1]) / (6.0 * hh);
        }
    }
    seg[(size_t)n].r0 = rec[(size_t)n].r;
    for (int p = 0; p < NPARAM; p++) seg[(size_t)n].c[p][0] = rec[(size_t)n].v[p][0];
}

// Unit model directions of the reverse sweep (UnitDirs), one knot and one
// segment table per parameter, built once per uploaded model.
int ensure_units(ysg_handle* h)
{
    if (h->has_units) return YSG_OK;
    const int n = h->hdr.nknot;
    const size_t nk = (size_t)n + 2, ns = (size_t)n + 1;
    std::vector<Knot> rec_all(nk * NPARAM);
    std::vector<Seg> seg_all(ns * NPARAM);
    const std::vector<double> one((size_t)n, 1.0), zero((size_t)n, 0.0);
    for (int p = 0; p < NPARAM; p++) {
        const double* val[NPARAM];
        const double* cs[NPARAM];
        for (int q = 0; q < NPARAM; q++) {
            val[q] = q == p ? one.data() : zero.data();
            cs[q] = zero.data();
        }
        std::vector<Knot> rec;
        std::vector<Seg> seg;
        build_tables(n, h->r_host.data(), val, cs, nullptr, nullptr, rec, seg);
        std::copy(rec.begin(), rec.end(), rec_all.begin() + (ptrdiff_t)(nk * p));
        std::copy(seg.begin(), seg.end(), seg_all.begin() + (ptrdiff_t)(ns * p));
    }
    CK(h->ukn.ensure(rec_all.size() * sizeof(Knot)));
    CK(h->usg.ensure(seg_all.size() * sizeof(Seg)));
    CK(cudaMemcpyAsync(h->ukn.p, rec_all.data(), rec_all.size() * sizeof(Knot), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->usg.p, seg_all.data(), seg_all.size() * sizeof(Seg), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->has_units = true;
    return YSG_OK;
}

// Capacities of the reverse sweep's logs for an event.  Steps: a yint takes
// 2 + floor(length / drr) - 1 steps on each interval it crosses, with
// drr = max(alpha_i, alpha_i+1) / (4 Re omega) (module_int.f90:2121-2138),
// never more than on the whole interval at the band's largest frequency;
// one more per interval covers rounding.  The supported solves integrate
// within one region at a time (inner core, outer core, mantle: the start
// levels, the solid / fluid hand-overs at nic and noc, source and receiver
// in the mantle), so the longest region bounds a yint.  Grid points of the
// l = 0 gravity solve: floor(length / dr) + 2 per piece, at most three
// pieces per interval (split at the source and the receiver),
// dr = alpha_min / (4 Re omega) or 1/4 at omega = 0 (module_model.f90:578-787
// with module_int.f90:1145-1166).
void adj_bounds(const ysg_handle* h, const EventDev& d, int* nmax, int* ncmax, int* gmax)
{
    const int n = h->hdr.nknot;
    const double* r = h->r_host.data();
    const double* al = h->alpha_host.data();
    const double w = d.wmin + (double)(d.jofs + (d.nw - 1) * d.jstride) * d.dw;
    const double amin = al[h->hdr.imin_alpha - 1];
    const double dr = w > 0.0 ? std::min(0.25, amin / (4.0 * w)) : 0.25;
    double steps[3] = {0.0, 0.0, 0.0}, pts = 0.0;
    for (int i = 1; i <= n - 1; i++) {
        const double hh = r[i] - r[i - 1];
        if (hh == 0.0) continue;
        const double drr = std::max(al[i - 1], al[i]) / (4.0 * w);
        const int reg = i < h->hdr.nic ? 0 : (i < h->hdr.noc ? 1 : 2);
        steps[reg] += 2.0 + std::floor(hh / drr);
        pts += 8.0 + std::floor(hh / dr);
    }
    const double smax = std::max(steps[0], std::max(steps[1], steps[2]));
    *nmax = (int)std::min(smax + 2.0, 1.0e8);
    // the chain from the start level to the source crosses at most all three
    *ncmax = (int)std::min(steps[0] + steps[1] + steps[2] + 2.0, 1.0e8);
    *gmax = (int)std::min(pts + 4.0, 1.0e8);
}

}  // namespace

extern "C" {

const char* ysg_last_cuda_error(void) { return g_cuda_err; }

const char* ysg_status_string(int s)
{
    switch (s) {
        case YSG_OK: return "ok";
        case YSG_ERR_ARG: return "bad argument";
        case YSG_ERR_CUDA: return "CUDA runtime error";
        case YSG_ERR_NO_MODEL: return "no model uploaded";
        case YSG_ERR_NO_SPECTRA: return "traces requested before spectra";
        case YSG_ERR_DEVICE_WAIT: return "a bounded device-side wait gave up";
        case YSG_ERR_NO_DEVICE: return "no CUDA device";
        case YSG_ERR_LIMIT: return "size beyond a fixed capacity";
        case YSG_ERR_UNSUPPORTED: return "path not covered by the reverse-mode solver";
        default: return "unknown status";
    }
}

int ysg_create(ysg_handle** out, int device)
{
    if (!out) return YSG_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return YSG_ERR_NO_DEVICE;
    if (device < 0 || device >= n) return YSG_ERR_ARG;
    ysg_handle* h = new ysg_handle;
    h->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return YSG_ERR_CUDA;
    }
    for (auto& e : h->ev) cudaEventCreate(&e);
    bool ok = cudaEventCreateWithFlags(&h->fork_ev, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < ysg_handle::NSIDE; i++)
        ok = ok && cudaStreamCreateWithFlags(&h->side[i], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&h->join_ev[i], cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaStreamCreateWithFlags(&h->copy_st, cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&h->copy_ev, cudaEventDisableTiming) == cudaSuccess;
    if (!ok || h->status.ensure(sizeof(int)) != cudaSuccess ||
        h->work.ensure(NSYS_COUNT * sizeof(unsigned long long)) != cudaSuccess) {
        ysg_destroy(h);
        return YSG_ERR_CUDA;
    }
    *out = h;
    return YSG_OK;
}

void ysg_destroy(ysg_handle* h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    for (Slot& s : h->slots) s.release();
    for (DevBuf* b : {&h->kn, &h->sg, &h->hdr_dev, &h->offs, &h->keys0, &h->keys1, &h->vals0,
                      &h->vals1, &h->sort_tmp, &h->poff, &h->pfx, &h->work, &h->status, &h->items, &h->counter,
                      &h->evdev, &h->coefptr, &h->dkn, &h->dsg, &h->ukn, &h->usg, &h->abasis,
                      &h->about, &h->ascr, &h->acs0, &h->agout, &h->asbar, &h->acoefb, &h->agrad, &h->alogs})
        b->release();
    for (DevBuf& b : h->scratch) b.release();
    for (auto& e : h->ev)
        if (e) cudaEventDestroy(e);
    for (int i = 0; i < ysg_handle::NSIDE; i++) {
        if (h->side[i]) {
            cudaStreamSynchronize(h->side[i]);
            cudaStreamDestroy(h->side[i]);
        }
        if (h->join_ev[i]) cudaEventDestroy(h->join_ev[i]);
    }
    if (h->fork_ev) cudaEventDestroy(h->fork_ev);
    if (h->copy_st) {
        cudaStreamSynchronize(h->copy_st);
        cudaStreamDestroy(h->copy_st);
    }
    if (h->copy_ev) cudaEventDestroy(h->copy_ev);
    for (cudaEvent_t e : h->done_ev)
        if (e) cudaEventDestroy(e);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

int ysg_set_solver(ysg_handle* h, int which)
{
    if (!h || which < 0 || which > 2) return YSG_ERR_ARG;
    h->solver = which;
    h->nactive = 0;          // work items depend on the solver: prepare again
    h->has_spectra = false;
    return YSG_OK;
}

int ysg_set_schedule(ysg_handle* h, int sched)
{
    if (!h || sched < -1 || sched >= NSCHED) return YSG_ERR_ARG;
    h->sched = sched;
    h->nactive = 0;          // prepare again
    h->has_spectra = false;
    return YSG_OK;
}

static_assert(NSCHED == 3, "ysg_last_schedule's tune_ms[] holds 3 entries (yspec_gpu.h)");

int ysg_last_schedule(ysg_handle* h, int* sched, float* tune_ms)
{
    if (!h || !sched) return YSG_ERR_ARG;
    *sched = h->cur_sched;
    if (tune_ms)
        for (int s = 0; s < NSCHED; s++) tune_ms[s] = h->tune_ms[s];
    return YSG_OK;
}

int ysg_get_stream(ysg_handle* h, void** stream)
{
    if (!h || !stream) return YSG_ERR_ARG;
    *stream = (void*)h->st;
    return YSG_OK;
}

int ysg_model_upload(ysg_handle* h, const ysg_model* m)
{
    if (!h || !m || m->nknot < 2 || !m->r || !m->alpha || !m->beta) return YSG_ERR_ARG;
    for (int p = 0; p < NPARAM; p++)
        if (!m->val[p] || !m->cs[p]) return YSG_ERR_ARG;
    const int n = m->nknot;
    if ((size_t)(n + 2) * sizeof(Knot) > 200 * 1024) return YSG_ERR_LIMIT;   // fits shared memory
    if (m->nic < 1 || m->noc <= m->nic || m->nsl <= m->noc || m->nsl > n) return YSG_ERR_ARG;
    std::vector<Knot> rec;
    std::vector<Seg> seg;
    build_tables(n, m->r, m->val, m->cs, m->alpha, m->beta, rec, seg);
    ModelHdr hd{};
    hd.nknot = n;
    hd.nic = m->nic;
    hd.noc = m->noc;
    hd.nsl = m->nsl;
    hd.ocean = m->ocean;
    hd.fic = m->fic;
    // iminloc: first index of the minimum (nrutil.f90:392-399)
    int ia = 1;
    for (int i = 2; i <= n; i++)
        if (m->alpha[i - 1] < m->alpha[ia - 1]) ia = i;
    int ib = m->noc + 1;
    for (int i = m->noc + 2; i <= m->nsl; i++)
        if (m->beta[i - 1] < m->beta[ib - 1]) ib = i;
    hd.imin_alpha = ia;
    hd.imin_beta = ib;
    hd.tref = m->tref;
    hd.pibigg = m->pibigg;
    hd.fre_norm = m->fre_norm;
    cudaSetDevice(h->device);
    CK(h->kn.ensure(rec.size() * sizeof(Knot)));
    CK(cudaMemcpyAsync(h->kn.p, rec.data(), rec.size() * sizeof(Knot), cudaMemcpyHostToDevice, h->st));
    CK(h->sg.ensure(seg.size() * sizeof(Seg)));
    CK(cudaMemcpyAsync(h->sg.p, seg.data(), seg.size() * sizeof(Seg), cudaMemcpyHostToDevice, h->st));
    CK(h->hdr_dev.ensure(sizeof(ModelHdr)));
    CK(cudaMemcpyAsync(h->hdr_dev.p, &hd, sizeof(ModelHdr), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->hdr = hd;
    h->grav_host.assign(m->val[P_GRAV], m->val[P_GRAV] + n);
    h->r_host.assign(m->r, m->r + n);
    h->alpha_host.assign(m->alpha, m->alpha + n);
    h->has_model = true;
    h->ndir = 0;
    h->has_units = false;
    h->has_spectra = false;
    for (Slot& s : h->slots) s.ev_ready = s.tm_ready = false;
    return YSG_OK;
}

int ysg_model_tangents_upload(ysg_handle* h, int ndir, const ysg_model* dms)
{
    if (!h || !dms || ndir < 1 || ndir > 65535) return YSG_ERR_ARG;
    if (!h->has_model) return YSG_ERR_NO_MODEL;
    const int n = h->hdr.nknot;
    for (int d = 0; d < ndir; d++) {
        if (dms[d].nknot != n) return YSG_ERR_ARG;
        for (int p = 0; p < NPARAM; p++)
            if (!dms[d].val[p] || !dms[d].cs[p]) return YSG_ERR_ARG;
    }
    const size_t nk = (size_t)n + 2, ns = (size_t)n + 1;
    std::vector<Knot> rec_all(nk * ndir);
    std::vector<Seg> seg_all(ns * ndir);
    for (int d = 0; d < ndir; d++) {
        std::vector<Knot> rec;
        std::vector<Seg> seg;
        build_tables(n, h->r_host.data(), dms[d].val, dms[d].cs, nullptr, nullptr, rec, seg);
        // the tables hold derivatives, except the radii the segments are based on
        for (size_t i = 0; i < seg.size(); i++) seg[i].r0 = 0.0;
        std::copy(rec.begin(), rec.end(), rec_all.begin() + (ptrdiff_t)(nk * d));
        std::copy(seg.begin(), seg.end(), seg_all.begin() + (ptrdiff_t)(ns * d));
    }
    cudaSetDevice(h->device);
    h->ndir = 0;
    CK(h->dkn.ensure(rec_all.size() * sizeof(Knot)));
    CK(cudaMemcpyAsync(h->dkn.p, rec_all.data(), rec_all.size() * sizeof(Knot), cudaMemcpyHostToDevice, h->st));
    CK(h->dsg.ensure(seg_all.size() * sizeof(Seg)));
    CK(cudaMemcpyAsync(h->dsg.p, seg_all.data(), seg_all.size() * sizeof(Seg), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->ndir = ndir;
    h->has_spectra = false;
    return YSG_OK;
}

int ysg_model_tangent_upload(ysg_handle* h, const ysg_model* dm)
{
    return ysg_model_tangents_upload(h, 1, dm);
}

int ysg_trace_rows(const ysg_time* tm)
{
    if (!tm) return 0;
    int nout = tm->nt;
    for (int i = 1; i <= tm->nt; i++)
        if ((double)(i - 1) * tm->dt > tm->tout) {
            nout = i;
            break;
        }
    return nout;
}

int ysg_event_coef(ysg_handle* h, const ysg_event* ev, double* coef)
{
    int rc = check_event(h, ev);
    if (rc) return rc;
    cudaSetDevice(h->device);
    h->has_spectra = false;
    rc = prepare_single(h, ev);
    if (rc) return rc;
    h->leg_overlap = false;          // no Legendre stage here
    CK(record(h, 0));
    CK(record(h, 1));
    rc = enqueue_solve(h, 1);
    if (rc) return rc;
    CK(record(h, 2));
    CK(record(h, 3));
    const size_t n = (size_t)(ev->lmax - ev->lmin + 1) * NCOEF * ev->nw;
    if (coef) CK(cudaMemcpyAsync(coef, slot0(h).coef.p, n * sizeof(cd), cudaMemcpyDeviceToHost, h->st));
    rc = finish(h, 1, true, false);
    h->has_spectra = false;
    return rc;
}

int ysg_event_potential(ysg_handle* h, const ysg_event* ev, const ysg_time* tm, double* out, int* nout)
{
    int rc = check_event(h, ev);
    if (rc) return rc;
    if (!tm || tm->nr != ev->nr) return YSG_ERR_ARG;
    cudaSetDevice(h->device);
    h->has_spectra = false;
    h->h2d = h->d2h = 0.0;
    h->pot_mode = 1;
    rc = prepare_single(h, ev);
    h->launches = 0;          // count this call's kernels only (not autotuning)
    if (!rc) rc = upload_time(h, slot0(h), tm, ev->nw);
    h->pot_mode = 0;
    if (rc) return rc;
    rc = enqueue_spectra(h, 1);
    if (!rc) rc = enqueue_traces(h, 1, 0);
    if (rc) return rc;
    const Slot& s = slot0(h);
    const TraceDev& td = s.ptd;
    if (nout) *nout = td.nout;
    if (out && td.nr > 0) {
        // columns 0 (time) and 1 (the potential, in the Z position) of each receiver
        CK(cudaMemcpy2DAsync(out, (size_t)2 * td.nout * sizeof(double), s.out.p, (size_t)4 * td.nout * sizeof(double),
                             (size_t)2 * td.nout * sizeof(double), (size_t)td.nr, cudaMemcpyDeviceToHost, h->st));
        h->d2h += (double)td.nout * 2 * td.nr * sizeof(double);
    }
    rc = finish(h, 1, true, true);
    h->has_spectra = false;            // the device spectra hold the potential, not displacements
    return rc;
}

int ysg_event_gradient(ysg_handle* h, const ysg_event* ev, const ysg_time* tm, const double* gout, double* gval,
                       double* gcs)
{
    int rc = check_event(h, ev);
    if (rc) return rc;
    if (!tm || !gval || !gcs || tm->nr != ev->nr || (ev->nr > 0 && !gout)) return YSG_ERR_ARG;
    // the source and the receivers in the solid above the outer core
    if (ev->is <= h->hdr.noc || ev->ir <= h->hdr.noc) return YSG_ERR_UNSUPPORTED;
    const int L = ev->lmax - ev->lmin + 1;
    if (L >= (1 << 23) || L > 65535 || ev->nw >= (1 << 24) || ev->nr > 65535) return YSG_ERR_LIMIT;
    cudaSetDevice(h->device);
    h->has_spectra = false;
    h->launches = 0;
    h->h2d = h->d2h = 0.0;
    Slot& s = slot0(h);
    rc = upload_event(h, s, ev);
    if (!rc) rc = upload_time(h, s, tm, ev->nw);
    if (!rc) rc = upload_batch_items(h, 1);
    if (!rc) rc = ensure_units(h);
    if (rc) return rc;
    h->nactive = 1;
    const int n = h->hdr.nknot, nw = ev->nw, nr = ev->nr;
    const TraceDev& td = s.ptd;
    const int nout = td.nout;
    int nmax = 0, ncmax = 0, gmax = 0;
    adj_bounds(h, s.pev, &nmax, &ncmax, &gmax);
    // sweep work space: every resident thread of the l >= 1 sweeps (step
    // logs only) and one thread per frequency of the l = 0 sweeps (step and
    // grid logs), within a quarter of the free memory
    int nblk = solve_adjoint_blocks();
    if (nblk <= 0) return YSG_ERR_CUDA;
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    const size_t per = adj_log_bytes(nmax, ncmax, 0), per_r = adj_log_bytes(nmax, ncmax, gmax);
    const size_t Tr = ev->lmin == 0 ? (size_t)(nw + ADJ_THREADS - 1) / ADJ_THREADS * ADJ_THREADS : 0;
    const size_t budget = (free_b + h->alogs.cap) / 4;
    // no more threads than entries
    nblk = (int)std::min<long long>(nblk, (2 * h->npairs + ADJ_THREADS - 1) / ADJ_THREADS);
    while (nblk > 1 && (size_t)nblk * ADJ_THREADS * per + Tr * per_r > budget) nblk--;
    if ((size_t)nblk * ADJ_THREADS * per + Tr * per_r > budget) return YSG_ERR_LIMIT;
    const size_t T = (size_t)nblk * ADJ_THREADS;
    const size_t nspec = (size_t)nw * std::max(nr, 1);
    const size_t ngrad = (size_t)(n + 1) * NPARAM * 4;
    CK(h->abasis.ensure((size_t)2 * nw * nw * sizeof(cd)));
    CK(h->about.ensure((size_t)nout * 4 * 2 * nw * sizeof(double)));
    CK(h->ascr.ensure(std::max<size_t>(ifft_scratch_bytes(td.nt, 2 * nw), 16)));
    CK(h->acs0.ensure((size_t)2 * 2 * nw * sizeof(double)));
    CK(h->agout.ensure(std::max<size_t>((size_t)nout * 4 * nr * sizeof(double), 16)));
    CK(h->asbar.ensure(3 * nspec * sizeof(cd)));
    CK(h->acoefb.ensure((size_t)L * NCOEF * nw * sizeof(cd)));
    CK(h->agrad.ensure(ngrad * sizeof(double)));
    CK(h->alogs.ensure(T * per + Tr * per_r));
    std::vector<double> cs0((size_t)4 * nw);
    for (int b = 0; b < 2 * nw; b++) {
        cs0[2 * (size_t)b] = 1.0;
        cs0[2 * (size_t)b + 1] = 0.0;
    }
    CK(cudaMemcpyAsync(h->acs0.p, cs0.data(), cs0.size() * sizeof(double), cudaMemcpyHostToDevice, h->st));
    if (nr > 0)
        CK(cudaMemcpyAsync(h->agout.p, gout, (size_t)nout * 4 * nr * sizeof(double), cudaMemcpyHostToDevice, h->st));
    h->h2d += (double)(cs0.size() * sizeof(double) + (size_t)nout * 4 * nr * sizeof(double));
    // work space: each log's arrays in turn (every size a multiple of 512
    // bytes, as the thread counts are multiples of 128)
    unsigned char* base = h->alogs.as<unsigned char>();
    auto take = [&](size_t bytes) {
        unsigned char* q = base;
        base += bytes;
        return q;
    };
    auto steps_of = [&](size_t nt, int n) {
        AdjStepArrays a{};
        a.n = n;
        a.y = reinterpret_cast<cd*>(take((size_t)n * 14 * nt * sizeof(cd)));
        a.x = reinterpret_cast<double*>(take((size_t)n * nt * sizeof(double)));
        a.h = reinterpret_cast<double*>(take((size_t)n * nt * sizeof(double)));
        a.f = reinterpret_cast<double*>(take((size_t)n * nt * sizeof(double)));
        a.il = reinterpret_cast<int*>(take((size_t)n * nt * sizeof(int)));
        return a;
    };
    auto carve = [&](size_t nt, int nc, int ng) {
        AdjLogs w{};
        w.nthreads = (int)nt;
        w.s = steps_of(nt, nmax);
        w.c = steps_of(nt, nc);
        w.gmax = ng;
        w.gy = reinterpret_cast<cd*>(take((size_t)ng * 4 * nt * sizeof(cd)));
        w.gr = reinterpret_cast<double*>(take((size_t)ng * nt * sizeof(double)));
        w.gi = reinterpret_cast<int*>(take((size_t)ng * nt * sizeof(int)));
        return w;
    };
    const AdjLogs w = carve(T, ncmax, 0);
    const AdjLogs wr = Tr ? carve(Tr, ncmax, gmax) : AdjLogs{};
    UnitDirs u;
    for (int p = 0; p < NPARAM; p++) {
        u.kn[p] = h->ukn.as<Knot>() + (size_t)p * (n + 2);
        u.sg[p] = h->usg.as<Seg>() + (size_t)p * (n + 1);
    }
    h->leg_overlap = false;
    CK(record(h, 0));
    if (nr > 0) {
        h->launches += 1;
        CK(launch_legendre(nr, s.lmax, s.delta.as<double>(), s.ct.as<double>(), s.stv.as<double>(),
                           s.leg.as<double>(), h->st));
    }
    CK(record(h, 1));
    // time stage on the basis, then its transpose and the l-sum's
    h->launches += nr > 0 ? 6 : 0;   // basis, pass A, pass B, rotation, spectrum and l-sum transposes
    if (nr > 0) {
        CK(launch_time_basis(td, h->abasis.as<cd>(), s.filt.as<double>(), s.tw.as<cd>(), s.expt.as<double>(),
                             h->acs0.as<double>(), h->ascr.as<cd>(), h->about.as<double>(), h->st));
        CK(launch_spec_adjoint(nw, nr, nout, h->about.as<double>(), h->agout.as<double>(), s.cs.as<double>(),
                               h->asbar.as<cd>(), h->st));
    }
    CK(record(h, 2));
    if (nr > 0)
        CK(launch_lsum_adjoint(nw, nr, ev->lmin, ev->lmax, s.leg.as<double>(), s.E.as<cd>(), h->asbar.as<cd>(),
                               h->acoefb.as<cd>(), h->st));
    else
        CK(cudaMemsetAsync(h->acoefb.p, 0, (size_t)L * NCOEF * nw * sizeof(cd), h->st));
    CK(record(h, 3));
    // the pair schedule's cost-sorted entries, then the reverse sweeps
    StepCost sc;
    for (int q = 0; q < NSYS_COUNT; q++) sc.flops[q] = kStepFlops[q];
    sc.base = kPairBaseFlops;
    unsigned long long* keys[2] = {h->keys0.as<unsigned long long>(), h->keys1.as<unsigned long long>()};
    unsigned long long* vals[2] = {h->vals0.as<unsigned long long>(), h->vals1.as<unsigned long long>()};
    unsigned long long* sorted = nullptr;
    h->launches += 3;                // k_step_prefix, k_pair_cost and the sweeps (the radix sort is CUB's)
    CK(launch_pair_schedule(h->kn.as<Knot>(), h->sg.as<Seg>(), h->hdr_dev.as<ModelHdr>(), h->evdev.as<EventDev>(),
                            h->offs.as<long long>(), 1, h->npairs, h->poff.as<long long>(), h->nrows,
                            h->pfx.as<int>(), sc, keys, vals, h->sort_tmp.p, h->sort_tmp.cap, &sorted, h->st));
    CK(cudaMemsetAsync(h->agrad.p, 0, ngrad * sizeof(double), h->st));
    CK(cudaMemsetAsync(h->status.p, 0, sizeof(int), h->st));
    // the l = 0 sweeps (few, long) beside the others on a side stream
    if (Tr) {
        rc = fork_side(h, 1);
        if (rc) return rc;
        h->launches += 1;
        CK(launch_radial_adjoint(h->kn.as<Knot>(), h->sg.as<Seg>(), h->hdr_dev.as<ModelHdr>(),
                                 h->evdev.as<EventDev>(), u, h->acoefb.as<cd>(), wr, h->agrad.as<double>(),
                                 h->status.as<int>(), h->side[0]));
    }
    CK(launch_solve_adjoint(h->kn.as<Knot>(), h->sg.as<Seg>(), h->hdr_dev.as<ModelHdr>(), h->evdev.as<EventDev>(), u,
                            h->acoefb.as<cd>(), sorted, 2 * h->npairs, w, h->agrad.as<double>(),
                            reinterpret_cast<unsigned long long*>(h->counter.p), h->status.as<int>(), h->st));
    if (Tr && (rc = join_side(h, 1))) return rc;
    CK(record(h, 4));
    std::vector<double> g(ngrad);
    int status = 0;
    CK(cudaMemcpyAsync(g.data(), h->agrad.p, ngrad * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(&status, h->status.p, sizeof status, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->d2h += (double)(ngrad * sizeof(double) + sizeof status);
    float t[4];
    CK(cudaEventElapsedTime(&t[0], h->ev[0], h->ev[1]));
    CK(cudaEventElapsedTime(&t[3], h->ev[1], h->ev[2]));
    CK(cudaEventElapsedTime(&t[2], h->ev[2], h->ev[3]));
    CK(cudaEventElapsedTime(&t[1], h->ev[3], h->ev[4]));
    for (int i = 0; i < 4; i++) h->ms[i] = t[i];
    h->pairs = (double)L * nw;
    h->flops = 0.0;
    if (status) return YSG_ERR_LIMIT;
    // dL/dc[i][p][k] -> knot values and spline second derivatives, through
    // the segment formulas of build_tables
    std::fill(gval, gval + (size_t)NPARAM * n, 0.0);
    std::fill(gcs, gcs + (size_t)NPARAM * n, 0.0);
    const double* r = h->r_host.data();
    for (int i = 1; i <= n; i++)
        for (int p = 0; p < NPARAM; p++) {
            const double* c = &g[((size_t)i * NPARAM + p) * 4];
            double* gv = gval + (size_t)p * n;
            double* gc = gcs + (size_t)p * n;
            gv[i - 1] += c[0];
            if (i == n) continue;
            const double hh = r[i] - r[i - 1];
            if (hh == 0.0) continue;
            gv[i] += c[1] / hh;
            gv[i - 1] -= c[1] / hh;
            gc[i - 1] += -c[1] * hh / 3.0 + 0.5 * c[2] - c[3] / (6.0 * hh);
            gc[i] += -c[1] * hh / 6.0 + c[3] / (6.0 * hh);
        }
    return YSG_OK;
}

int ysg_legendre_table(ysg_handle* h, int nr, int lmax, const double* delta, const double* ct,
                       const double* st, double* table)
{
    if (!h || nr < 0 || lmax < 0 || (nr > 0 && (!delta || !ct || !st || !table))) return YSG_ERR_ARG;
    if (nr == 0) return YSG_OK;
    cudaSetDevice(h->device);
    Slot& s = slot0(h);
    s.ev_ready = s.tm_ready = false;
    h->has_spectra = false;
    CK(s.delta.ensure((size_t)nr * sizeof(double)));
    CK(s.ct.ensure((size_t)nr * sizeof(double)));
    CK(s.stv.ensure((size_t)nr * sizeof(double)));
    const size_t nt = (size_t)(lmax + 1) * nr * 8;
    CK(s.leg.ensure(nt * sizeof(double)));
    CK(cudaMemcpyAsync(s.delta.p, delta, (size_t)nr * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(s.ct.p, ct, (size_t)nr * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(s.stv.p, st, (size_t)nr * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(launch_legendre(nr, lmax, s.delta.as<double>(), s.ct.as<double>(), s.stv.as<double>(),
                       s.leg.as<double>(), h->st));
    CK(cudaMemcpyAsync(table, s.leg.p, nt * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return YSG_OK;
}

int ysg_event_spectra(ysg_handle* h, const ysg_event* ev, double* ur, double* ut, double* up)
{
    int rc = check_event(h, ev);
    if (rc) return rc;
    cudaSetDevice(h->device);
    h->has_spectra = false;
    rc = prepare_single(h, ev);
    if (rc) return rc;
    rc = enqueue_spectra(h, 1);
    if (rc) return rc;
    const int nr = ev->nr, nw = ev->nw;
    const size_t nspec = (size_t)nw * std::max(nr, 1);
    const cd* d_ur = slot0(h).spec.as<cd>();
    const size_t nb = (size_t)nw * nr * sizeof(cd);
    if (ur && nr > 0) CK(cudaMemcpyAsync(ur, d_ur, nb, cudaMemcpyDeviceToHost, h->st));
    if (ut && nr > 0) CK(cudaMemcpyAsync(ut, d_ur + nspec, nb, cudaMemcpyDeviceToHost, h->st));
    if (up && nr > 0) CK(cudaMemcpyAsync(up, d_ur + 2 * nspec, nb, cudaMemcpyDeviceToHost, h->st));
    return finish(h, 1, true, false);
}

int ysg_event_spectra_device(ysg_handle* h, const ysg_event* ev, void* d_ur, void* d_ut, void* d_up)
{
    int rc = check_event(h, ev);
    if (rc) return rc;
    cudaSetDevice(h->device);
    h->has_spectra = false;
    rc = prepare_single(h, ev);
    if (rc) return rc;
    rc = enqueue_spectra(h, 1);
    if (rc) return rc;
    const int nr = ev->nr, nw = ev->nw;
    const size_t nspec = (size_t)nw * std::max(nr, 1);
    const cd* d_spec = slot0(h).spec.as<cd>();
    const size_t nb = (size_t)nw * nr * sizeof(cd);
    if (d_ur && nr > 0) CK(cudaMemcpyAsync(d_ur, d_spec, nb, cudaMemcpyDeviceToDevice, h->st));
    if (d_ut && nr > 0) CK(cudaMemcpyAsync(d_ut, d_spec + nspec, nb, cudaMemcpyDeviceToDevice, h->st));
    if (d_up && nr > 0) CK(cudaMemcpyAsync(d_up, d_spec + 2 * nspec, nb, cudaMemcpyDeviceToDevice, h->st));
    return finish(h, 1, true, false);
}

int ysg_event_traces(ysg_handle* h, const ysg_time* tm, double* out, int* nout)
{
    if (!h || !tm) return YSG_ERR_ARG;
    if (!h->has_spectra || h->nactive != 1 || !slot0(h).ev_ready) return YSG_ERR_NO_SPECTRA;
    Slot& s = slot0(h);
    if (tm->nr != s.nr) return YSG_ERR_ARG;
    if (tm->nr > 0 && !out) return YSG_ERR_ARG;
    cudaSetDevice(h->device);
    int rc = upload_time(h, s, tm, s.pev.nw);
    if (rc) return rc;
    rc = enqueue_traces(h, 1, 0);
    if (rc) return rc;
    rc = copy_out(h, s, out, nout);
    if (rc) return rc;
    return finish(h, 1, false, true);
}

int ysg_event_prepare(ysg_handle* h, const ysg_event* ev, const ysg_time* tm)
{
    int rc = check_event(h, ev);
    if (rc) return rc;
    if (!tm || tm->nr != ev->nr) return YSG_ERR_ARG;
    cudaSetDevice(h->device);
    h->has_spectra = false;
    h->h2d = h->d2h = 0.0;
    rc = prepare_single(h, ev);
    h->launches = 0;          // count the execute's kernels only (not autotuning)
    if (rc) return rc;
    return upload_time(h, slot0(h), tm, ev->nw);
}

int ysg_event_execute(ysg_handle* h)
{
    if (!h) return YSG_ERR_ARG;
    if (h->nactive != 1 || !slot0(h).ev_ready || !slot0(h).tm_ready) return YSG_ERR_NO_SPECTRA;
    cudaSetDevice(h->device);
    int rc = enqueue_spectra(h, 1);
    if (rc) return rc;
    return enqueue_traces(h, 1, 0);
}

int ysg_event_fetch(ysg_handle* h, double* out, int* nout)
{
    if (!h) return YSG_ERR_ARG;
    if (h->nactive != 1 || !slot0(h).ev_ready || !slot0(h).tm_ready) return YSG_ERR_NO_SPECTRA;
    cudaSetDevice(h->device);
    int rc = copy_out(h, slot0(h), out, nout);
    if (rc) return rc;
    return finish(h, 1, true, true);
}

int ysg_event_run(ysg_handle* h, const ysg_event* ev, const ysg_time* tm, double* out, int* nout)
{
    int rc = ysg_event_prepare(h, ev, tm);
    if (rc) return rc;
    if (tm->nr > 0 && !out) return YSG_ERR_ARG;
    rc = ysg_event_execute(h);
    if (rc) return rc;
    return ysg_event_fetch(h, out, nout);
}

int ysg_batch_run(ysg_handle* h, int nev, const ysg_event* evs, const ysg_time* tms, double** outs,
                  int* nouts)
{
    if (!h || nev < 0 || (nev > 0 && (!evs || !tms || !outs))) return YSG_ERR_ARG;
    for (int e = 0; e < nev; e++) {
        int rc = check_event(h, &evs[e]);
        if (rc) return rc;
        if (tms[e].nr != evs[e].nr || (evs[e].nr > 0 && !outs[e])) return YSG_ERR_ARG;
    }
    if (nev == 0) return YSG_OK;
    cudaSetDevice(h->device);
    h->has_spectra = false;
    h->nactive = 0;
    h->h2d = h->d2h = 0.0;
    if (h->slots.size() < (size_t)nev) h->slots.resize((size_t)nev);
    for (int e = 0; e < nev; e++) {
        Slot& s = h->slots[(size_t)e];
        int rc = upload_event(h, s, &evs[e]);
        if (!rc) rc = upload_time(h, s, &tms[e], evs[e].nw);
        if (rc) return rc;
    }
    if (h->solver == 1) {
        int rc = upload_batch_items(h, nev);
        if (!rc) rc = resolve_schedule(h, nev);
        if (rc) return rc;
    } else if (h->solver == 2) {
        int rc = upload_batch_items(h, nev);
        if (rc) return rc;
    }
    h->nactive = nev;
    h->launches = 0;
    int rc = launch_batch_graph(h, nev);
    if (rc) return rc;
    if (nev > 1) {
        // each copy waits for its own event's chain (enqueue_chains); the
        // handle's stream then waits for the copies
        for (int e = 0; e < nev; e++) {
            CK(cudaStreamWaitEvent(h->copy_st, h->done_ev[(size_t)e], 0));
            rc = copy_out(h, h->slots[(size_t)e], outs[e], nouts ? &nouts[e] : nullptr, h->copy_st);
            if (rc) return rc;
        }
        CK(cudaEventRecord(h->copy_ev, h->copy_st));
        CK(cudaStreamWaitEvent(h->st, h->copy_ev, 0));
    } else {
        rc = copy_out(h, h->slots[0], outs[0], nouts ? &nouts[0] : nullptr);
        if (rc) return rc;
    }
    return finish(h, nev, true, true);
}

int ysg_last_launches(ysg_handle* h, long long* n)
{
    if (!h || !n) return YSG_ERR_ARG;
    *n = h->launches;
    return YSG_OK;
}

int ysg_last_bytes(ysg_handle* h, double* h2d, double* d2h)
{
    if (!h) return YSG_ERR_ARG;
    if (h2d) *h2d = h->h2d;
    if (d2h) *d2h = h->d2h;
    return YSG_OK;
}

int ysg_last_timings(ysg_handle* h, float ms[4])
{
    if (!h || !ms) return YSG_ERR_ARG;
    for (int i = 0; i < 4; i++) ms[i] = h->ms[i];
    return YSG_OK;
}

int ysg_last_work(ysg_handle* h, double* pairs, double* flops)
{
    if (!h) return YSG_ERR_ARG;
    if (pairs) *pairs = h->pairs;
    if (flops) *flops = h->flops;
    return YSG_OK;
}

}  // extern "C"
