/*
 * yo.h -- CPU oracle for the YSpec direct radial integration path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C FP64 restatement of the
 * reference Fortran (da380/YSpec, the Fortran sources under src/) against
 * which the CUDA product path is tested.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs may load it.  It is never part of the
 * product path.
 *
 * Parity status: UNPINNED.  The reference ships no tests, golden outputs or
 * known-answer vectors, and no Fortran compiler exists in the build or GPU
 * images, so the reference itself cannot be executed to pin this
 * restatement.  It is checked instead against internal known-answer tests
 * (spline exactness on cubics, Legendre normalisation, continued fraction vs
 * series overlap, the frequency-grid table, physical sanity checks).
 *
 * Every routine cites the reference file:line it restates.  Arrays follow the
 * reference's 1-based indexing (element 0 unused) so the citations can be
 * checked line by line.
 */
#ifndef YO_H
#define YO_H

#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double _Complex yo_cd;

/* Model arrays, normalised as module_model.f90:251-290 leaves them.
 * All arrays are 1-based with nknot+1 elements. */
typedef struct {
    int ifanis, ocean, fic;
    int nlayer, nknot, nic, noc, nsl;
    int *layer_lo, *layer_hi;        /* layer_index(:,1), layer_index(:,2) */
    double tref;
    double *r;
    double *rho, *rho_cs, *acon, *acon_cs, *ccon, *ccon_cs, *fcon, *fcon_cs;
    double *lcon, *lcon_cs, *ncon, *ncon_cs, *kappa, *kappa_cs, *mu, *mu_cs;
    double *lambda, *qkappa, *qkappa_cs, *qmu, *qmu_cs, *grav, *grav_cs;
    double *beta, *alpha, *rat, *rat_cs, *xlam, *xlam_cs, *xa2, *xa2_cs;
} yo_model;

/* Normalisation constants, module_model.f90:474-492. */
typedef struct {
    double r_norm, rho_norm, vel_norm, acl_norm, fre_norm, t_norm;
    double con_norm, grav_norm, moment_norm, pot_norm, pibigg;
} yo_norms;

/* Everything the parameter file holds (yspec.f90:88-137), raw units. */
typedef struct {
    char pref_out[256];
    char model_file[256];
    int ats, grav, out, cor, lmin, lmax;
    double f1, f2, tout, dt, f11, f12, f21, f22;
    double depth_s, lat_s, lon_s, mm[6];
    double depth_r;
    int nr;
    double *lat_r, *lon_r;          /* 0-based, nr entries */
} yo_params;

/* Derived per-event quantities after normalisation and fcal. */
typedef struct {
    int nt, i1, i2, nw, is, ir;
    double df, ep, dw, wmin, dt, tout, rs, rr;
    double f1, f2, f11, f12, f21, f22;
    double mm[6];
} yo_grid;

/* Counters for the algorithmic work model (RHS evaluations and RK steps per
 * system size).  Index = number of complex components (2, 4, 5, 14). */
typedef struct {
    long long nrhs[16];
    long long nstep[16];
    long long nsolve_tor, nsolve_sph, nsolve_rad;
} yo_counts;

void yo_set_parameters(yo_norms *n);
int  yo_read_model(const char *path, const yo_norms *n, yo_model *m);
void yo_free_model(yo_model *m);
int  yo_read_params(const char *path, yo_params *p);
void yo_free_params(yo_params *p);
int  yo_find_radius_index(const yo_model *m, double rr);
void yo_delaz(double eplati, double eplong, double stlati, double stlong,
              double *delta, double *azep, double *azst);
void yo_legendre(double theta, int l, int m, double *x, double *xp,
                 double *xcosec);
int  yo_fcal(double *f1, double *f2, double dt, double tout, int mex, int qex,
             double *df, double *ep, int *nt, int *i1, int *i2);
void yo_spline(const double *x, const double *y, int n, double yp1,
               double ypn, double *y2);
double yo_splint_dis(const double *xa, const double *ya, const double *y2a,
                     double x, int klo);
void yo_bfs(int l, yo_cd xsq, double eps, yo_cd *fp);

/* Event setup: normalise inputs, fcal, radius indices
 * (yspec.f90:176-215).  Returns 0 or a nonzero stop code. */
int yo_event_setup(const yo_model *m, const yo_norms *n, const yo_params *p,
                   yo_grid *g);

/* One (omega,l) solve giving the l-sum coefficients of yspec.f90:263-400:
 * coef[0..4] = uu(1..5), coef[5..9] = vv(1..5), coef[10..14] = ww(1..5).
 * For l == 0 only uu(3) is set.  Counters are accumulated into cnt if
 * non-NULL. */
void yo_solve_pair(const yo_model *m, const yo_norms *n, const yo_params *p,
                   const yo_grid *g, int l, int j, yo_cd coef[15],
                   yo_counts *cnt);

/* Full spectra: ur/ut/up are (nw, nr) column-major (omega fastest), summed
 * over l exactly as yspec.f90:250-426.
 * lsub_lo/lsub_hi restrict the l range (inclusive) when lsub_hi >= 0.
 * jsub > 0 restricts omega to j <= jsub; jsub < 0 takes every |jsub|-th
 * frequency j = 1, 1+|jsub|, ... (bounded CPU samples across the band).
 * nthreads <= 0 uses every online core. */
int yo_spectra(const yo_model *m, const yo_norms *n, const yo_params *p,
               const yo_grid *g, yo_cd *ur, yo_cd *ut, yo_cd *up,
               int nthreads, int lsub_lo, int lsub_hi, int jsub,
               yo_counts *cnt);

/* Spectra of a frequency shard: column c (0-based, c < count) of the
 * (count, nr) column-major arrays holds omega_j, j = 1 + jofs + c jstride,
 * as the device's jofs/jstride event fields define a shard. */
int yo_spectra_shard(const yo_model *m, const yo_norms *n, const yo_params *p,
                     const yo_grid *g, int jofs, int jstride, int count, yo_cd *ur,
                     yo_cd *ut, yo_cd *up, int nthreads);

/* yo_solve_pair for npair (ls[k], js[k]) pairs; coef is (15, npair)
 * column-major (15 coefficients per pair, pair after pair). */
int yo_coef_list(const yo_model *m, const yo_norms *n, const yo_params *p,
                 const yo_grid *g, int npair, const int *ls, const int *js,
                 yo_cd *coef, int nthreads);

/* The solution of one two-point solver at radius rr (knot index ir) for
 * unit jumps at rs (index is), omega = wr + i wi: kind 0 toroidal (2 x 2),
 * 1 radial without and 2 with gravity (2 x 2), 3 spheroidal with full
 * gravity (6 x 4), 4 without gravity and 5 Cowling (4 x 4); row-major.
 * Used by the reciprocity and gravity-limit checks of the oracle. */
int yo_green(const yo_model *m, const yo_norms *n, int kind, int l, double wr,
             double wi, int ats, double rr, double rs, int ir, int is, yo_cd *out);

/* Oracle-only convergence knob: every knot interval of the Runge-Kutta
 * integration takes refine times the reference's step count (1 restores
 * the reference's rule, module_int.f90:1903-1905).  Process-wide. */
void yo_set_step_refine(int refine);

/* Potential mode: yo_solve_pair and everything built on it (spectra,
 * traces) return the perturbation of the gravitational potential at the
 * receivers in place of the displacement: per pair the spheroidal
 * solution's third component (ysph(3,:)) combined with the source vectors
 * as uu, for l = 0 the potential of rad_solver_wg (module_solver.f90:
 * 534-554), no toroidal part; ur carries the potential, ut and up are zero.
 * The time stage's amplitude factor stays that of the output type (the
 * caller rescales to the potential's normalisation).  Process-wide;
 * 0 restores the reference's outputs. */
void yo_set_potential(int on);

/* Legendre/geometry table used by the l-sum (yspec.f90:144-174):
 * xa/xpa/xca are (lmax+1, 3, nr) column-major; delta/azst/azep are nr. */
void yo_geometry(const yo_params *p, double *delta, double *azep,
                 double *azst);
void yo_legendre_table(const double *delta, int nr, int lmax, double *xa,
                       double *xpa, double *xca);

/* Time series (module_fourier.f90:55-145 + yspec.f90:433-486).
 * ur/ut/up are (nw,nr) spectra; out is (nout,4,nr): t, Z, N, E per row. */
int yo_traces(const yo_norms *n, const yo_params *p, const yo_grid *g,
              const yo_cd *ur, const yo_cd *ut, const yo_cd *up,
              const double *azep, double *out, int *nout);

/* End to end: parameter file -> traces (allocated with malloc; caller
 * frees).  Returns 0 or a nonzero stop code. */
int yo_run(const char *param_file, double **out, int *nout, int *nr,
           int nthreads);

/* Output writer identical in format to yspec.f90:488-503. */
int yo_write_traces(const char *pref_out, const double *out, int nout,
                    int nr);

#ifdef __cplusplus
}
#endif
#endif
