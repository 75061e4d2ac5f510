/*
 * yspec_gpu.h -- C-ABI of the B200 radial-integration engine.
 *
 * This boundary replaces, in the reference program (da380/YSpec, src/):
 *   yspec.f90:250-426   the (omega,l) double loop: per-pair radial, toroidal
 *                       and spheroidal solves (module_solver.f90:25-1847,
 *                       module_int.f90:134-2138, module_start.f90:14-178)
 *                       and the receiver l-sum with Legendre factors
 *                       (yspec.f90:155-174 table, :291-293, :316-335,
 *                       :396-419 sums)
 *   yspec.f90:432-486   ifft (module_fourier.f90:55-145), e^{eps t},
 *                       dimensionalisation and rotation to Z/N/E.
 * The host keeps everything before (parameter file, read_model with its
 * splines and gravity, delaz, fcal, radius indices) and the ASCII writer.
 *
 * Conventions: plain pointers and sizes only; host buffers are owned by the
 * caller; complex(dp) arrays are interleaved (re, im) doubles; arrays are
 * column-major with the reference's dimension order; knot and interval
 * indices are 1-based exactly as the reference computes them.  Every call
 * returns a status (YSG_OK == 0); nonzero codes replace the reference's
 * `stop` statements and ysg_status_string() gives the message.
 *
 * One handle per host thread; a handle owns one CUDA stream on one device.
 */
#ifndef YSPEC_GPU_H
#define YSPEC_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    YSG_OK = 0,
    YSG_ERR_ARG = 1,          /* bad argument or size */
    YSG_ERR_CUDA = 2,         /* CUDA runtime error */
    YSG_ERR_NO_MODEL = 3,     /* ysg_model_upload not called */
    YSG_ERR_NO_SPECTRA = 4,   /* traces requested before spectra */
    YSG_ERR_DEVICE_WAIT = 5,  /* a bounded device-side wait gave up */
    YSG_ERR_NO_DEVICE = 6,    /* no CUDA device */
    YSG_ERR_LIMIT = 7,        /* size beyond a fixed capacity */
    YSG_ERR_UNSUPPORTED = 8   /* a path the reverse-mode solver does not cover */
};

typedef struct ysg_handle ysg_handle;

/* Earth model after module_model.f90:175-383 (read_model): normalised knot
 * values and per-layer natural-spline second derivatives.  Each pointer is
 * an array of nknot doubles (knot 1 first).  The 13 parameters are, in
 * order: rho, acon, ccon, fcon, lcon, ncon, kappa, mu, qkappa, qmu, grav,
 * xlam, xa2 (module_model.f90:129-160). */
typedef struct {
    int nknot, nic, noc, nsl;        /* module_model.f90:121-125 */
    int ocean, fic;                  /* module_model.f90:119-120 */
    double tref;                     /* normalised 2 pi / T_ref (:195-197) */
    double pibigg;                   /* module_model.f90:490 */
    double fre_norm;                 /* module_model.f90:484 */
    const double *r;
    const double *val[13];
    const double *cs[13];
    const double *alpha, *beta;      /* module_model.f90:276-277 */
} ysg_model;

/* One event's spectral problem (yspec.f90:176-261 after normalisation). */
typedef struct {
    int lmin, lmax;
    int nw;                          /* i2 - i1 + 1 frequencies */
    int is, ir;                      /* find_radius_index of source, receiver */
    int ats, grav, out, cor;         /* switches, yspec.f90:100-103 */
    int nr;                          /* receivers */
    int jofs, jstride;               /* frequency shard: the event's j-th frequency is
                                        omega at index jofs + (j-1) jstride of the full
                                        band (0 and 1 for the whole band) */
    double wmin, dw, ep;             /* omega_k = wmin + k dw - i ep, k = jofs + (j-1) jstride */
    double rs, rr;                   /* normalised source / receiver radius */
    double mm[6];                    /* moment tensor / moment_norm */
    const double *delta;             /* nr epicentral angles (delaz), rad */
    const double *azst;              /* nr azimuths after yspec.f90:150 */
} ysg_event;

/* Time-series stage (fcal outputs, filter, output scaling). */
typedef struct {
    int nt, i1, i2;                  /* module_fourier.f90:362-397 */
    int nr;
    double df, dt, ep, tout;         /* normalised */
    double f11, f12, f21, f22;       /* normalised corners; all 0 = no filter */
    double t_norm;                   /* module_model.f90:485 */
    double amp_norm;                 /* r_norm, vel_norm or acl_norm */
    const double *azep;              /* nr azimuths after yspec.f90:149 */
} ysg_time;

/* Create a handle on CUDA device `device`.  Replaces nothing in the
 * reference (which has no device); allocates the stream and status word. */
int ysg_create(ysg_handle **h, int device);

/* Upload the model (replaces the module_model.f90:118-160 globals that the
 * solver modules read).  Copies the arrays; the caller may free them. */
int ysg_model_upload(ysg_handle *h, const ysg_model *m);

/* Derivative of the uploaded model along one direction of model space, for
 * the tangent-linear solver (ysg_set_solver 2): dm->val[p] and dm->cs[p]
 * are the derivatives of the knot values and of their spline second
 * derivatives.  Only those 26 arrays are read (nknot must match the
 * uploaded model); radii, alpha, beta and the scalar fields are the
 * uploaded model's.  No reference counterpart: the reference has no
 * derivatives.  A new ysg_model_upload discards it. */
int ysg_model_tangent_upload(ysg_handle *h, const ysg_model *dm);

/* ndir directions at once (dms[0..ndir-1], each as above).  With solver 2,
 * slot s of ysg_batch_run takes direction s, so a batch of ndir copies of
 * one event returns the derivatives of its traces along every direction
 * in one solve launch; a single direction serves every slot.  The tangent
 * solve runs the batched solver's cost-sorted entry list: batches of more
 * than 65535 slots, or events of 2^23 degrees or 2^24 frequencies, return
 * YSG_ERR_LIMIT. */
int ysg_model_tangents_upload(ysg_handle *h, int ndir, const ysg_model *dms);

/* Potential traces of one event: the perturbation of the gravitational
 * potential at every receiver, in the event's output type (potential, its
 * first or second time derivative).  Each pair contributes its potential
 * coefficients in place of uu: the spheroidal solution's third component
 * (ysph(3,:), the potential; zero without self-gravitation) combined with
 * the source vectors as uu is in yspec.f90:396-398, and for l = 0 the
 * potential that rad_solver_wg forms and the main program discards
 * (module_solver.f90:534-554); toroidal pairs contribute nothing.  The
 * l-sum and the time stage (module_fourier.f90 ifft4 applied to the
 * potential row, then yspec.f90:432-473) are those of the displacement.
 * out is (nout, 2, nr) column-major: time in seconds, then the potential;
 * tm->amp_norm must be the potential's normalisation for the output type
 * (pot_norm, pot_norm / t_norm or pot_norm / t_norm^2, module_model.f90:489).
 * No reference counterpart as a whole: the reference computes these pieces
 * but never writes potential traces. */
int ysg_event_potential(ysg_handle *h, const ysg_event *ev, const ysg_time *tm, double *out, int *nout);

/* Gradient of the misfit functional L = sum gout * traces of one event
 * with respect to the uploaded model (reverse mode: the discrete adjoint of
 * every (omega, l) solve, after the transposes of the time stage and of the
 * l-sum).  gout is (nout, 4, nr) column-major like ysg_event_run's out
 * (column 0, time, is ignored): dL/d(trace sample).  gval and gcs receive
 * dL/dval[p][i] and dL/dcs[p][i] at gval[p * nknot + i] (13 * nknot
 * doubles each): the gradient with respect to the knot values and spline
 * second derivatives of ysg_model, the arrays read_model forms
 * (module_model.f90:175-383).  As for the tangent-linear solver, start
 * levels, step counts and rescaling are those of the uploaded model (they
 * are piecewise constant in it) and alpha / beta are not differentiated.
 * Covers a source and receivers in the solid above the outer core, the
 * receivers above or below the source, for every gravity setting
 * (self-gravitation, Cowling, none), a solid or a fluid inner core, with or
 * without an ocean; events with the source or the receivers in the core
 * return YSG_ERR_UNSUPPORTED.  No reference counterpart: the reference has no
 * derivatives.  Stage times (ysg_last_timings): Legendre table, reverse
 * sweeps, l-sum transpose, time-stage transpose. */
int ysg_event_gradient(ysg_handle *h, const ysg_event *ev, const ysg_time *tm, const double *gout,
                       double *gval, double *gcs);

/* Spectra of one event: yspec.f90:250-426.  ur, ut, up are complex
 * (nw, nr) column-major host arrays (interleaved re/im), or NULL to keep
 * the spectra on the device only.  Also leaves the spectra on the device
 * for ysg_event_traces. */
int ysg_event_spectra(ysg_handle *h, const ysg_event *ev, double *ur, double *ut, double *up);

/* ysg_event_spectra into device buffers the caller owns (complex (nw, nr)
 * column-major each, on the handle's device), for callers that pass the
 * spectra on without a host round trip (the multi-GPU receiver exchange).
 * Returns when the copies are done. */
int ysg_event_spectra_device(ysg_handle *h, const ysg_event *ev, void *d_ur, void *d_ut,
                             void *d_up);

/* Time series of the last spectra: module_fourier.f90:55-145 and
 * yspec.f90:432-486.  out is (nout, 4, nr) column-major: time in seconds,
 * then Re of the Z, N, E components in SI units, exactly the four columns
 * the reference writes.  *nout receives the row count (yspec.f90:479-486);
 * out must hold nout_max(tm) * 4 * nr doubles. */
int ysg_event_traces(ysg_handle *h, const ysg_time *tm, double *out, int *nout);

/* Rows the trace output will have for tm (yspec.f90:479-486). */
int ysg_trace_rows(const ysg_time *tm);

/* Spectra then traces without copying the spectra to the host
 * (= ysg_event_prepare + ysg_event_execute + ysg_event_fetch). */
int ysg_event_run(ysg_handle *h, const ysg_event *ev, const ysg_time *tm, double *out,
                  int *nout);

/* The three phases of ysg_event_run, for callers that time or overlap the
 * device work.  prepare copies the event's inputs to the device and returns
 * when they are resident; execute enqueues every kernel of the event on the
 * handle's stream and returns at once; fetch copies the traces of the last
 * execute to `out` (if non-NULL), waits, and reports the status. */
int ysg_event_prepare(ysg_handle *h, const ysg_event *ev, const ysg_time *tm);
int ysg_event_execute(ysg_handle *h);
int ysg_event_fetch(ysg_handle *h, double *out, int *nout);

/* The handle's cudaStream_t, as a void pointer. */
int ysg_get_stream(ysg_handle *h, void **stream);

/* Time series from device-resident spectra without any device allocation.
 * No counterpart in the reference: it exists for callers that cannot let
 * the library call cudaMalloc (a host that owns the whole GPU memory
 * through its own pool, or code where an allocation would synchronise the
 * device).  Same result as ysg_event_traces; d_ur/d_ut/d_up are complex
 * (nw, nr) device arrays, d_azep has nr entries, d_out receives
 * (nout, 4, nr); tm->azep is not used.  Work is enqueued on `stream`
 * (a cudaStream_t, or NULL) and the call returns without waiting.
 * Intermediate rows live in one 16 MiB array compiled into the library and
 * held by every GPU that loads it until exit; nt is limited to 262144
 * (YSG_ERR_LIMIT beyond).  All calls share that array: calls that overlap
 * on the GPU race and must be serialised.  The first call on each device
 * looks up the array's device address and should come before any stream
 * capture; the address is cached per device for the primary context, so the
 * entry point is not for use after cudaDeviceReset or from a separate
 * driver-API context.  nt must be a power of two >= 8, as for
 * ysg_event_traces.  An error pending from earlier work on the calling
 * thread is cleared on entry; a failure of this call is described by
 * ysg_last_cuda_error(). */
int ysg_traces_noalloc(const ysg_time *tm, const double *d_ur, const double *d_ut,
                       const double *d_up, const double *d_azep, double *d_out, int *nout,
                       void *stream);

/* Several events through the batched persistent solver: one launch per
 * stage for all events, CUDA-graph captured.  outs[e] receives the traces of
 * event e as ysg_event_traces does; nouts[e] its row count.  Events share
 * the uploaded model.  With more than one event, each event's l-sum and
 * time series run back to back on a side stream and its traces are copied
 * out as soon as they are complete, beside the other events' stages; the
 * call returns when every copy has finished. */
int ysg_batch_run(ysg_handle *h, int nev, const ysg_event *evs, const ysg_time *tms,
                  double **outs, int *nouts);

/* Per-(omega,l) l-sum coefficients uu(1:5), vv(1:5), ww(1:5) of
 * yspec.f90:281-400 for one event: coef is complex (nw, 15, L) with
 * L = lmax - lmin + 1, omega fastest.  Diagnostic entry point used by the
 * parity tests; it runs only the solve stage. */
int ysg_event_coef(ysg_handle *h, const ysg_event *ev, double *coef);

/* Legendre table of yspec.f90:155-170 for nr angles: table is
 * (8, nr, lmax+1) column-major with rows X_l0, X_l1, X_l2, dX_l0, dX_l1,
 * dX_l2, X_l1/sin, X_l2/sin.  ct, st are cos and sin of delta. */
int ysg_legendre_table(ysg_handle *h, int nr, int lmax, const double *delta, const double *ct,
                       const double *st, double *table);

/* Select the solve kernel: 0 = plain (one thread per (omega,l) pair, one
 * event per launch), 1 = batched persistent (default), 2 = tangent-linear:
 * the solve stage returns the derivative of the uu / vv / ww coefficients
 * along the direction given by ysg_model_tangent_upload, with the start
 * levels and step counts of the uploaded model held fixed.  Every later
 * stage is linear in the coefficients, so with solver 2 the spectra and
 * traces of every entry point are the derivatives of the primal ones. */
int ysg_set_solver(ysg_handle *h, int which);

/* Work schedule of the batched solver: 0 = tiles of (event, l, 32
 * consecutive frequencies) ordered by estimated cost; 1 = lists of 32
 * entries (the spheroidal and the toroidal part of each pair) of equal code
 * path and near-equal exact step-count cost (a count-only pass and a sort
 * before the solve); 2 = the same lists in two concurrent launches, the
 * spheroidal parts and the toroidal parts (a small-slab, higher-occupancy
 * kernel on a second stream); -1
 * (default) = autotuned: the first time a workload signature is seen, the
 * solve stage runs once with each schedule and the fastest is kept.
 * Results do not depend on the schedule beyond rounding. */
int ysg_set_schedule(ysg_handle *h, int sched);

/* Schedule of the last batched solve, and the solve-stage times in ms of
 * each schedule from the last autotuning run (tune_ms may be NULL). */
int ysg_last_schedule(ysg_handle *h, int *sched, float tune_ms[3]);

/* Device times in ms of the last event's stages, measured with CUDA events:
 * [0] Legendre table, [1] solves, [2] l-sum, [3] filter + inverse FFT +
 * post-processing.  For a single event (not a batch) the Legendre table is
 * built on a second stream beside the solves, so [0] overlaps [1].  For a
 * batch of more than one event, [2] covers the l-sums and the time series
 * together (they run per event, back to back) and [3] is zero. */
int ysg_last_timings(ysg_handle *h, float ms[4]);

/* Counters of the last solve stage: number of (omega,l) pairs and the
 * algorithmic FP64 flop count of the stepping work actually performed. */
int ysg_last_work(ysg_handle *h, double *pairs, double *flops);

/* Kernels of this library enqueued since the last ysg_event_prepare (or
 * ysg_event_run / ysg_batch_run), autotuning runs excluded. */
int ysg_last_launches(ysg_handle *h, long long *n);

/* Host<->device bytes moved by the last ysg_event_run / prepare+fetch:
 * event inputs and tables copied in, traces copied out. */
int ysg_last_bytes(ysg_handle *h, double *h2d, double *d2h);

/* Measured FP64 fused-multiply-add throughput of `device` in TFLOP/s
 * (roofline denominator of the solve stage). */
int ysg_fp64_peak(int device, double *tflops);

const char *ysg_status_string(int status);

/* The CUDA runtime error behind the calling thread's last YSG_ERR_CUDA
 * (error name, message and the failing call), or "" if there was none. */
const char *ysg_last_cuda_error(void);
void ysg_destroy(ysg_handle *h);

#ifdef __cplusplus
}
#endif
#endif
