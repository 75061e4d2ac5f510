// capi.cu -- the ysg_* C-ABI (include/yspec_gpu.h).
//
// Orchestrates the device stages of one event on the handle's stream:
//   K2 Legendre table -> K1 (omega,l) solves -> K3 receiver l-sum
//   -> K4 filter + inverse FFT + post-processing
// with CUDA events between stages for the per-stage device times.  Small
// host-side tables (cos/sin of the epicentral angles, e^{i m azst} powers,
// the taper, FFT twiddles, e^{eps t}) are formed here on the host, in FP64,
// as the reference forms them, and uploaded with each event.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
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
// Sys::CLS in ysg_ode.cuh): 6 right-hand sides plus the stage
// combinations (88 flops per complex component).  The per-RHS counts are
// hand tallies of the coefficient matrix and derivative expressions.
const double kStepFlops[8] = {
    6 * 88.0 + 88.0 * 2,     // toroidal
    6 * 177.0 + 88.0 * 2,    // radial
    6 * 100.0 + 88.0 * 2,    // fluid minors, no gravity / Cowling
    6 * 290.0 + 88.0 * 4,    // b-vector, no gravity / Cowling
    6 * 300.0 + 88.0 * 5,    // solid minors, no gravity / Cowling
    6 * 240.0 + 88.0 * 5,    // fluid minors, self-gravitation
    6 * 700.0 + 88.0 * 14,   // solid minors, self-gravitation
    6 * 700.0 + 88.0 * 14,   // b-vector, self-gravitation
};

}  // namespace

struct ysg_handle {
    int device = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev[5] = {};
    int solver = 0;
    // model
    DevBuf kn;
    ModelHdr hdr{};
    std::vector<double> grav_host;   // knot gravity for the tilt correction
    bool has_model = false;
    // event buffers
    DevBuf coef, leg, E, delta, ct, stv, spec, filt, tw, expt, cs, scratch, out;
    DevBuf work, status;
    bool has_spectra = false;
    int last_nw = 0, last_nr = 0;
    float ms[4] = {0, 0, 0, 0};
    double pairs = 0.0, flops = 0.0;
};

#define CK(x)                                   \
    do {                                        \
        cudaError_t e_ = (x);                   \
        if (e_ != cudaSuccess) return YSG_ERR_CUDA; \
    } while (0)

extern "C" {

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
    if (h->status.ensure(sizeof(int)) != cudaSuccess || h->work.ensure(8 * sizeof(unsigned long long)) != cudaSuccess) {
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
    for (DevBuf* b : {&h->kn, &h->coef, &h->leg, &h->E, &h->delta, &h->ct, &h->stv, &h->spec,
                      &h->filt, &h->tw, &h->expt, &h->cs, &h->scratch, &h->out, &h->work,
                      &h->status})
        b->release();
    for (auto& e : h->ev)
        if (e) cudaEventDestroy(e);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

int ysg_set_solver(ysg_handle* h, int which)
{
    if (!h || which < 0 || which > 1) return YSG_ERR_ARG;
    h->solver = which;
    return YSG_OK;
}

int ysg_model_upload(ysg_handle* h, const ysg_model* m)
{
    if (!h || !m || m->nknot < 2 || !m->r || !m->alpha || !m->beta) return YSG_ERR_ARG;
    for (int p = 0; p < NPARAM; p++)
        if (!m->val[p] || !m->cs[p]) return YSG_ERR_ARG;
    const int n = m->nknot;
    if ((size_t)(n + 2) * sizeof(Knot) > 200 * 1024) return YSG_ERR_LIMIT;   // fits shared memory
    std::vector<Knot> rec((size_t)n + 2);
    std::memset(rec.data(), 0, rec.size() * sizeof(Knot));
    for (int i = 0; i < n; i++) {
        Knot& k = rec[(size_t)i + 1];
        k.r = m->r[i];
        k.alpha = m->alpha[i];
        k.beta = m->beta[i];
        for (int p = 0; p < NPARAM; p++) {
            k.v[p][0] = m->val[p][i];
            k.v[p][1] = m->cs[p][i];
        }
    }
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
    CK(cudaStreamSynchronize(h->st));
    h->hdr = hd;
    h->grav_host.assign(m->val[P_GRAV], m->val[P_GRAV] + n);
    h->has_model = true;
    h->has_spectra = false;
    return YSG_OK;
}

}  // extern "C"

namespace {

int check_event(const ysg_handle* h, const ysg_event* ev)
{
    if (!h || !ev) return YSG_ERR_ARG;
    if (!h->has_model) return YSG_ERR_NO_MODEL;
    if (ev->lmin < 0 || ev->lmax < ev->lmin || ev->nw < 1 || ev->nr < 0) return YSG_ERR_ARG;
    if (ev->is < 1 || ev->ir < 1 || ev->is >= h->hdr.nknot || ev->ir >= h->hdr.nknot) return YSG_ERR_ARG;
    if (ev->nr > 0 && (!ev->delta || !ev->azst)) return YSG_ERR_ARG;
    if (ev->grav < 0 || ev->grav > 2 || ev->out < 0 || ev->out > 2) return YSG_ERR_ARG;
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
    d.rs = ev->rs;
    d.rr = ev->rr;
    d.ep = ev->ep;
    d.wmin = ev->wmin;
    d.dw = ev->dw;
    d.grav_ir = h->grav_host[(size_t)ev->ir - 1];
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

int run_solve_stage(ysg_handle* h, const EventDev& d)
{
    const int L = d.lmax - d.lmin + 1;
    const size_t ncoef = (size_t)L * NCOEF * d.nw;
    CK(h->coef.ensure(ncoef * sizeof(cd)));
    CK(cudaMemsetAsync(h->work.p, 0, 8 * sizeof(unsigned long long), h->st));
    CK(cudaMemsetAsync(h->status.p, 0, sizeof(int), h->st));
    CK(launch_solve_plain(h->kn.as<Knot>(), h->hdr, d, h->coef.as<cd>(),
                          h->work.as<unsigned long long>(), h->status.as<int>(), h->st));
    return YSG_OK;
}

int finish_solve_stage(ysg_handle* h, const EventDev& d)
{
    unsigned long long w[8];
    int status = 0;
    CK(cudaMemcpyAsync(w, h->work.p, sizeof w, cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(&status, h->status.p, sizeof status, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    double fl = 0.0;
    for (int q = 0; q < 8; q++) fl += (double)w[q] * kStepFlops[q];
    h->flops = fl;
    h->pairs = (double)(d.lmax - d.lmin + 1) * d.nw;
    return status ? YSG_ERR_DEVICE_WAIT : YSG_OK;
}

}  // namespace

extern "C" {

int ysg_event_coef(ysg_handle* h, const ysg_event* ev, double* coef)
{
    int rc = check_event(h, ev);
    if (rc) return rc;
    cudaSetDevice(h->device);
    EventDev d = make_event(h, ev);
    CK(cudaEventRecord(h->ev[0], h->st));
    rc = run_solve_stage(h, d);
    if (rc) return rc;
    CK(cudaEventRecord(h->ev[1], h->st));
    const size_t n = (size_t)(d.lmax - d.lmin + 1) * NCOEF * d.nw;
    if (coef) CK(cudaMemcpyAsync(coef, h->coef.p, n * sizeof(cd), cudaMemcpyDeviceToHost, h->st));
    rc = finish_solve_stage(h, d);
    cudaEventElapsedTime(&h->ms[1], h->ev[0], h->ev[1]);
    return rc;
}

int ysg_legendre_table(ysg_handle* h, int nr, int lmax, const double* delta, const double* ct,
                       const double* st, double* table)
{
    if (!h || nr < 0 || lmax < 0 || (nr > 0 && (!delta || !ct || !st || !table))) return YSG_ERR_ARG;
    if (nr == 0) return YSG_OK;
    cudaSetDevice(h->device);
    CK(h->delta.ensure((size_t)nr * sizeof(double)));
    CK(h->ct.ensure((size_t)nr * sizeof(double)));
    CK(h->stv.ensure((size_t)nr * sizeof(double)));
    const size_t nt = (size_t)(lmax + 1) * nr * 8;
    CK(h->leg.ensure(nt * sizeof(double)));
    CK(cudaMemcpyAsync(h->delta.p, delta, (size_t)nr * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->ct.p, ct, (size_t)nr * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->stv.p, st, (size_t)nr * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(launch_legendre(nr, lmax, h->delta.as<double>(), h->ct.as<double>(), h->stv.as<double>(),
                       h->leg.as<double>(), h->st));
    CK(cudaMemcpyAsync(table, h->leg.p, nt * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return YSG_OK;
}

int ysg_event_spectra(ysg_handle* h, const ysg_event* ev, double* ur, double* ut, double* up)
{
    int rc = check_event(h, ev);
    if (rc) return rc;
    cudaSetDevice(h->device);
    EventDev d = make_event(h, ev);
    const int nr = ev->nr, nw = ev->nw;
    h->has_spectra = false;
    // host tables: cos/sin of delta, e^{i m azst} (yspec.f90:173-174, :331, :414)
    std::vector<double> ct(std::max(nr, 1)), stv(std::max(nr, 1));
    std::vector<cd> E((size_t)std::max(nr, 1) * 5);
    for (int k = 0; k < nr; k++) {
        ct[k] = std::cos(ev->delta[k]);
        stv[k] = std::sin(ev->delta[k]);
        cd eia = mk(std::cos(ev->azst[k]), std::sin(ev->azst[k]));
        for (int m = -2; m <= 2; m++) E[(size_t)k * 5 + (m + 2)] = cpowi(eia, m);
    }
    const size_t nspec = (size_t)nw * std::max(nr, 1);
    CK(h->spec.ensure(3 * nspec * sizeof(cd)));
    cd* d_ur = h->spec.as<cd>();
    cd* d_ut = d_ur + nspec;
    cd* d_up = d_ut + nspec;
    if (nr > 0) {
        CK(h->delta.ensure((size_t)nr * sizeof(double)));
        CK(h->ct.ensure((size_t)nr * sizeof(double)));
        CK(h->stv.ensure((size_t)nr * sizeof(double)));
        CK(h->E.ensure((size_t)nr * 5 * sizeof(cd)));
        CK(h->leg.ensure((size_t)(ev->lmax + 1) * nr * 8 * sizeof(double)));
        CK(cudaMemcpyAsync(h->delta.p, ev->delta, (size_t)nr * sizeof(double), cudaMemcpyHostToDevice, h->st));
        CK(cudaMemcpyAsync(h->ct.p, ct.data(), (size_t)nr * sizeof(double), cudaMemcpyHostToDevice, h->st));
        CK(cudaMemcpyAsync(h->stv.p, stv.data(), (size_t)nr * sizeof(double), cudaMemcpyHostToDevice, h->st));
        CK(cudaMemcpyAsync(h->E.p, E.data(), (size_t)nr * 5 * sizeof(cd), cudaMemcpyHostToDevice, h->st));
    }
    CK(cudaEventRecord(h->ev[0], h->st));
    CK(launch_legendre(nr, ev->lmax, h->delta.as<double>(), h->ct.as<double>(), h->stv.as<double>(),
                       h->leg.as<double>(), h->st));
    CK(cudaEventRecord(h->ev[1], h->st));
    rc = run_solve_stage(h, d);
    if (rc) return rc;
    CK(cudaEventRecord(h->ev[2], h->st));
    CK(launch_lsum(nw, nr, ev->lmin, ev->lmax, h->coef.as<cd>(), h->leg.as<double>(),
                   h->E.as<cd>(), d_ur, d_ut, d_up, h->st));
    CK(cudaEventRecord(h->ev[3], h->st));
    const size_t nb = (size_t)nw * nr * sizeof(cd);
    if (ur && nr > 0) CK(cudaMemcpyAsync(ur, d_ur, nb, cudaMemcpyDeviceToHost, h->st));
    if (ut && nr > 0) CK(cudaMemcpyAsync(ut, d_ut, nb, cudaMemcpyDeviceToHost, h->st));
    if (up && nr > 0) CK(cudaMemcpyAsync(up, d_up, nb, cudaMemcpyDeviceToHost, h->st));
    rc = finish_solve_stage(h, d);
    cudaEventElapsedTime(&h->ms[0], h->ev[0], h->ev[1]);
    cudaEventElapsedTime(&h->ms[1], h->ev[1], h->ev[2]);
    cudaEventElapsedTime(&h->ms[2], h->ev[2], h->ev[3]);
    if (rc) return rc;
    h->has_spectra = true;
    h->last_nw = nw;
    h->last_nr = nr;
    return YSG_OK;
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

int ysg_event_traces(ysg_handle* h, const ysg_time* tm, double* out, int* nout_p)
{
    if (!h || !tm) return YSG_ERR_ARG;
    if (!h->has_spectra) return YSG_ERR_NO_SPECTRA;
    const int n = tm->nt, nr = tm->nr;
    if (n < 4 || (n & (n - 1)) || n > (1 << 20)) return YSG_ERR_ARG;
    if (nr != h->last_nr || tm->i2 - tm->i1 + 1 != h->last_nw || tm->i1 < 1) return YSG_ERR_ARG;
    if (nr > 0 && (!tm->azep || !out)) return YSG_ERR_ARG;
    cudaSetDevice(h->device);
    const int nout = ysg_trace_rows(tm);
    if (nout_p) *nout_p = nout;
    if (nr == 0) return YSG_OK;
    int p = 0;
    while ((1 << p) < n) p++;
    // taper (module_fourier.f90:96-116), twiddles with pi_d, e^{eps t}, rotation
    const double pi_d = (double)3.14159265358979323846f;
    std::vector<double> filt((size_t)n / 2 + 1, 1.0), expt(nout), cs(2 * (size_t)nr);
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
    const double dth = pi_d / (double)(n / 2);
    for (int m = 0; m < n / 2; m++) {
        double a = (double)m * dth;
        tw[(size_t)m] = mk(std::cos(a), std::sin(a));
    }
    for (int i = 0; i < nout; i++) expt[(size_t)i] = std::exp(tm->ep * ((double)i * tm->dt));
    for (int k = 0; k < nr; k++) {
        cs[2 * (size_t)k] = std::cos(tm->azep[k]);
        cs[2 * (size_t)k + 1] = std::sin(tm->azep[k]);
    }
    CK(h->filt.ensure(filt.size() * sizeof(double)));
    CK(h->tw.ensure(tw.size() * sizeof(cd)));
    CK(h->expt.ensure(expt.size() * sizeof(double)));
    CK(h->cs.ensure(cs.size() * sizeof(double)));
    CK(h->scratch.ensure(ifft_scratch_bytes(n, nr)));
    const size_t nout_bytes = (size_t)nout * 4 * nr * sizeof(double);
    CK(h->out.ensure(nout_bytes));
    CK(cudaMemcpyAsync(h->filt.p, filt.data(), filt.size() * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->tw.p, tw.data(), tw.size() * sizeof(cd), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->expt.p, expt.data(), expt.size() * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->cs.p, cs.data(), cs.size() * sizeof(double), cudaMemcpyHostToDevice, h->st));
    TraceDev td{};
    td.nt = n;
    td.i1 = tm->i1;
    td.i2 = tm->i2;
    td.nw = h->last_nw;
    td.nr = nr;
    td.nout = nout;
    td.log2n = p;
    td.b1 = 1 << ((p + 1) / 2);
    td.dt = tm->dt;
    td.scale = tm->dt * (double)n;
    td.t_norm = tm->t_norm;
    td.amp_norm = tm->amp_norm;
    const size_t nspec = (size_t)h->last_nw * nr;
    const cd* d_ur = h->spec.as<cd>();
    CK(cudaEventRecord(h->ev[3], h->st));
    CK(launch_ifft(td, d_ur, d_ur + nspec, d_ur + 2 * nspec, h->filt.as<double>(), h->tw.as<cd>(),
                   h->expt.as<double>(), h->cs.as<double>(), h->scratch.as<cd>(), h->out.as<double>(),
                   h->st));
    CK(cudaEventRecord(h->ev[4], h->st));
    CK(cudaMemcpyAsync(out, h->out.p, nout_bytes, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    cudaEventElapsedTime(&h->ms[3], h->ev[3], h->ev[4]);
    return YSG_OK;
}

int ysg_event_run(ysg_handle* h, const ysg_event* ev, const ysg_time* tm, double* out, int* nout)
{
    int rc = ysg_event_spectra(h, ev, nullptr, nullptr, nullptr);
    if (rc) return rc;
    return ysg_event_traces(h, tm, out, nout);
}

int ysg_batch_run(ysg_handle* h, int nev, const ysg_event* evs, const ysg_time* tms, double** outs,
                  int* nouts)
{
    if (!h || nev < 0 || (nev > 0 && (!evs || !tms || !outs))) return YSG_ERR_ARG;
    for (int e = 0; e < nev; e++) {
        int rc = ysg_event_run(h, &evs[e], &tms[e], outs[e], nouts ? &nouts[e] : nullptr);
        if (rc) return rc;
    }
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
