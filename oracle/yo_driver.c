/*
 * yo_driver.c -- oracle restatement of the yspec.f90 driver (event setup,
 * (omega,l) loop, receiver l-sum, post-processing, writer) and of
 * module_fourier.f90 (ifft, fourrow_dp).  TEST INFRASTRUCTURE ONLY.
 */
#include "yo.h"
#include "yo_const.h"
#include "yo_internal.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

#define I_ (_Complex_I)

/* yspec.f90:176-215 */
int yo_event_setup(const yo_model *m, const yo_norms *n, const yo_params *p,
                   yo_grid *g)
{
    memset(g, 0, sizeof *g);
    double f1 = p->f1 * n->t_norm / 1000.0;
    double f2 = p->f2 * n->t_norm / 1000.0;
    g->dt = p->dt / n->t_norm;
    g->rs = m->r[m->nknot] - p->depth_s * 1000.0 / n->r_norm;
    g->rr = m->r[m->nknot] - p->depth_r * 1000.0 / n->r_norm;
    g->tout = p->tout * 60.0 / n->t_norm;
    for (int i = 0; i < 6; i++) g->mm[i] = p->mm[i] / n->moment_norm;
    g->f11 = p->f11 / 1000.0 * n->t_norm;
    g->f12 = p->f12 / 1000.0 * n->t_norm;
    g->f21 = p->f21 / 1000.0 * n->t_norm;
    g->f22 = p->f22 / 1000.0 * n->t_norm;
    int rc = yo_fcal(&f1, &f2, g->dt, g->tout, 5, 1, &g->df, &g->ep, &g->nt,
                     &g->i1, &g->i2);
    if (rc) return rc;
    g->f1 = f1;
    g->f2 = f2;
    g->dw = YO_TWOPI_D * g->df;
    if (g->i1 == g->i2) return YO_ERR_FEW_FREQ;
    g->wmin = (double)(g->i1 - 1) * g->dw;
    g->nw = g->i2 - g->i1 + 1;
    if (g->nw == 1) return YO_ERR_FEW_FREQ;
    g->is = yo_find_radius_index(m, g->rs);
    if (g->is == 0) return YO_ERR_SRC_MODEL;
    if (g->is > m->nsl) return YO_ERR_SRC_OCEAN;
    g->ir = yo_find_radius_index(m, g->rr);
    if (g->ir == 0) return YO_ERR_REC_MODEL;
    if (g->ir > m->nsl) return YO_ERR_REC_OCEAN;
    return 0;
}

/* Potential mode (yo_set_potential): each pair's uu carries its potential */
/* coefficients, vv and ww are zero.  Process-wide.                         */
static int g_potential = 0;

void yo_set_potential(int on) { g_potential = on != 0; }

/* yspec.f90:259-400 for one (omega_j, l) */
void yo_solve_pair(const yo_model *m, const yo_norms *n, const yo_params *p,
                   const yo_grid *g, int l, int j, yo_cd coef[15], yo_counts *cnt)
{
    yo_counts dummy;
    if (!cnt) { memset(&dummy, 0, sizeof dummy); cnt = &dummy; }
    yo_ctx c;
    memset(&c, 0, sizeof c);
    c.M = m;
    c.N = n;
    c.ats = (double)p->ats;
    c.cnt = cnt;
    for (int q = 0; q < 15; q++) coef[q] = 0.0;
    double rr = g->rr, rs = g->rs;
    int ir = g->ir, is = g->is;
    yo_cd w = (g->wmin + (double)(j - 1) * g->dw) - I_ * g->ep;
    double zeta = (double)sqrtf((float)(l * (l + 1)));   /* yspec.f90:255 */
    yo_cd *uu = coef, *vv = coef + 5, *ww = coef + 10;

    if (l == 0) {
        yo_cd sr0[2], yrad[2][2];
        yo_source_vector_rad(&c, w, is, rs, g->mm, sr0);
        if (g_potential) {
            /* the potential of rad_solver_wg (module_solver.f90:534-554) */
            yo_cd ph[2] = {0.0, 0.0};
            if (p->grav != 0) yo_rad_solver_wg(&c, w, rr, rs, ir, is, yrad, ph);
            uu[2] = (sr0[0] * ph[0] + sr0[1] * ph[1]) / rr;
        } else {
            if (p->grav == 0) yo_rad_solver_ng(&c, w, rr, rs, ir, is, yrad);
            else yo_rad_solver_wg(&c, w, rr, rs, ir, is, yrad, NULL);
            uu[2] = (sr0[0] * yrad[0][0] + sr0[1] * yrad[0][1]) / rr;
        }
        if (p->out == 1) uu[2] = I_ * w * uu[2];
        else if (p->out == 2) uu[2] = -(w * w * uu[2]);
        return;
    }
    if (l > 1 && !g_potential) {
        yo_cd svt[5][2], ytor[2][2];
        yo_source_vector_tor(&c, l, w, is, rs, g->mm, svt);
        yo_tor_solver(&c, l, w, rr, rs, ir, is, ytor);
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) {
                if (p->out == 1) ytor[a][b] = I_ * w * ytor[a][b];
                else if (p->out == 2) ytor[a][b] = -(w * w * ytor[a][b]);
            }
        for (int q = 0; q < 5; q++)
            ww[q] = (svt[q][0] * ytor[0][0] + svt[q][1] * ytor[0][1]) / (zeta * rr);
    }
    yo_cd svs[5][6], ysph[6][4];
    yo_source_vector_sph(&c, l, w, is, rs, g->mm, svs);
    if (p->grav == 2) {
        yo_sph_solver_g(&c, l, w, rr, rs, ir, is, m->fic, ysph);
    } else {
        yo_cd yng[4][4];
        yo_sph_solver_ngcow(&c, l, w, rr, rs, ir, is, m->fic, p->grav == 1, yng);
        for (int b = 0; b < 4; b++) {                  /* yspec.f90:367-374 */
            ysph[0][b] = yng[0][b];
            ysph[1][b] = yng[1][b];
            ysph[2][b] = 0.0;
            ysph[3][b] = yng[2][b];
            ysph[4][b] = yng[3][b];
            ysph[5][b] = 0.0;
        }
    }
    if (g_potential) {
        /* the potential (third solution component) in the output type,     */
        /* combined with the source vectors as uu (yspec.f90:396-398)        */
        for (int b = 0; b < 4; b++) {
            if (p->out == 1) ysph[2][b] = I_ * w * ysph[2][b];
            else if (p->out == 2) ysph[2][b] = -(w * w * ysph[2][b]);
        }
        for (int q = 0; q < 5; q++)
            uu[q] = (ysph[2][0] * svs[q][0] + ysph[2][1] * svs[q][1] +
                     ysph[2][2] * svs[q][3] + ysph[2][3] * svs[q][4]) / rr;
        return;
    }
    if (p->out == 1) {
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 4; b++) ysph[a][b] = I_ * w * ysph[a][b];
    } else if (p->out == 2) {
        if (p->cor == 0) {
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 4; b++) ysph[a][b] = -(w * w * ysph[a][b]);
        } else {                                        /* yspec.f90:388-391 */
            double gr = m->grav[ir];
            for (int b = 0; b < 4; b++) {
                yo_cd c1 = -((double)(l + 1) * ysph[2][b] + 2.0 * gr * ysph[0][b]) / rr;
                yo_cd c2 = zeta * (ysph[2][b] + gr * ysph[0][b]) / rr;
                ysph[0][b] = -(w * w * ysph[0][b]) + c1;
                ysph[1][b] = -(w * w * ysph[1][b]) + c2;
            }
        }
    }
    for (int q = 0; q < 5; q++) {                       /* yspec.f90:396-400 */
        uu[q] = (ysph[0][0] * svs[q][0] + ysph[0][1] * svs[q][1] +
                 ysph[0][2] * svs[q][3] + ysph[0][3] * svs[q][4]) / rr;
        vv[q] = (ysph[1][0] * svs[q][0] + ysph[1][1] * svs[q][1] +
                 ysph[1][2] * svs[q][3] + ysph[1][3] * svs[q][4]) / (zeta * rr);
    }
}

/* yspec.f90:144-150 */
void yo_geometry(const yo_params *p, double *delta, double *azep, double *azst)
{
    double lats = p->lat_s;
    if (lats == 90.0) lats = 89.98;
    for (int i = 0; i < p->nr; i++) {
        yo_delaz(p->lat_r[i], p->lon_r[i], lats, p->lon_s, &delta[i], &azep[i], &azst[i]);
        azep[i] = YO_TWOPI_D - azep[i];
        azst[i] = YO_PI_D - azst[i];
    }
}

/* yspec.f90:155-170; xa etc. are (lmax+1, 3, nr) column-major */
void yo_legendre_table(const double *delta, int nr, int lmax, double *xa, double *xpa,
                       double *xca)
{
    size_t L1 = (size_t)lmax + 1;
    memset(xa, 0, L1 * 3 * (size_t)nr * sizeof(double));
    memset(xpa, 0, L1 * 3 * (size_t)nr * sizeof(double));
    memset(xca, 0, L1 * 3 * (size_t)nr * sizeof(double));
    for (int i = 0; i < nr; i++) {
        for (int l = 0; l <= lmax; l++) {
            int mm = l == 0 ? 0 : (l == 1 ? 1 : 2);
            double x[3], xp[3], xc[3];
            yo_legendre(delta[i], l, mm, x, xp, xc);
            for (int q = 0; q <= mm; q++) {
                size_t idx = (size_t)l + L1 * ((size_t)q + 3 * (size_t)i);
                xa[idx] = x[q];
                xpa[idx] = xp[q];
                xca[idx] = xc[q];
            }
        }
    }
}

static yo_cd cpowi(yo_cd a, int m)
{
    /* integer power as libgfortran's pow_c8_i4 forms it */
    yo_cd pw = 1.0, x = a;
    unsigned u;
    if (m == 0) return pw;
    if (m < 0) { u = (unsigned)(-m); x = pw / x; } else u = (unsigned)m;
    for (;;) {
        if (u & 1) pw = pw * x;
        u >>= 1;
        if (u) x = x * x; else break;
    }
    return pw;
}

typedef struct {
    const yo_model *m;
    const yo_norms *n;
    const yo_params *p;
    const yo_grid *g;
    yo_cd *ur, *ut, *up;
    const double *xa, *xpa, *xca;
    const yo_cd *eia;
    int lo, hi, jmax, jstride, next;
    int jofs, ncol;                 /* job k takes j = 1 + jofs + (k-1) jstride; */
                                    /* ncol > 0: stored in column k-1 of ncol    */
    pthread_mutex_t lock;
} spectra_job;

typedef struct {
    spectra_job *job;
    yo_counts *cnt;
} spectra_arg;

/* one omega_j: every l in increasing order, then its l-sum contribution */
static void spectra_one(const spectra_job *jb, int j, int col, yo_counts *cnt)
{
    const yo_params *p = jb->p;
    int nr = p->nr, nw = jb->ncol > 0 ? jb->ncol : jb->g->nw;
    size_t L1 = (size_t)p->lmax + 1;
    const double *xa = jb->xa, *xpa = jb->xpa, *xca = jb->xca;
    yo_cd *ur = jb->ur, *ut = jb->ut, *up = jb->up;
    for (int l = jb->lo; l <= jb->hi; l++) {
        yo_cd coef[15];
        yo_solve_pair(jb->m, jb->n, p, jb->g, l, j, coef, cnt);
        yo_cd *uu = coef, *vv = coef + 5, *ww = coef + 10;
        for (int k = 0; k < nr; k++) {
            size_t o = (size_t)col + (size_t)nw * (size_t)k;
            if (l == 0) {
                ur[o] = ur[o] + uu[2] * xa[L1 * 3 * (size_t)k];
                continue;
            }
            for (int mq = -2; mq <= 2; mq++) {
                int am = mq < 0 ? -mq : mq;
                double msign = (mq < 0 && (mq & 1)) ? -1.0 : 1.0;
                size_t idx = (size_t)l + L1 * ((size_t)am + 3 * (size_t)k);
                double x = msign * xa[idx], xp = msign * xpa[idx];
                yo_cd ei = cpowi(jb->eia[k], mq);
                if (l > 1 && mq != 0) {                 /* yspec.f90:318-335 */
                    ut[o] = ut[o] + I_ * (double)mq * ww[mq + 2] * x * ei;
                    up[o] = up[o] - ww[mq + 2] * xp * ei;
                }
            }
            for (int mq = -2; mq <= 2; mq++) {          /* yspec.f90:402-419 */
                int am = mq < 0 ? -mq : mq;
                double msign = (mq < 0 && (mq & 1)) ? -1.0 : 1.0;
                size_t idx = (size_t)l + L1 * ((size_t)am + 3 * (size_t)k);
                double x = msign * xa[idx], xp = msign * xpa[idx], xc = msign * xca[idx];
                yo_cd ei = cpowi(jb->eia[k], mq);
                ur[o] = ur[o] + uu[mq + 2] * x * ei;
                ut[o] = ut[o] + vv[mq + 2] * xp * ei;
                up[o] = up[o] + I_ * (double)mq * vv[mq + 2] * xc * ei;
            }
        }
    }
}

static void *spectra_worker(void *a)
{
    spectra_arg *arg = (spectra_arg *)a;
    spectra_job *jb = arg->job;
    for (;;) {
        pthread_mutex_lock(&jb->lock);
        int k = ++jb->next;
        pthread_mutex_unlock(&jb->lock);
        int j = 1 + jb->jofs + (k - 1) * jb->jstride;
        if (j > jb->jmax) break;
        spectra_one(jb, j, jb->ncol > 0 ? k - 1 : j - 1, arg->cnt);
    }
    return NULL;
}

/* (omega,l) loop + l-sum, yspec.f90:250-426.  For each omega_j the l-sum   */
/* runs in increasing l, the reference's order for every (j,k).             */
static int spectra_run(const yo_model *m, const yo_norms *n, const yo_params *p,
                       const yo_grid *g, yo_cd *ur, yo_cd *ut, yo_cd *up, int nthreads,
                       int lo, int hi, int jofs, int jstride, int jmax, int ncol,
                       yo_counts *cnt)
{
    int nr = p->nr, lmax = p->lmax;
    int nw = ncol > 0 ? ncol : g->nw;
    double *delta = (double *)malloc((size_t)nr * sizeof(double));
    double *azep = (double *)malloc((size_t)nr * sizeof(double));
    double *azst = (double *)malloc((size_t)nr * sizeof(double));
    size_t L1 = (size_t)lmax + 1;
    double *xa = (double *)malloc(L1 * 3 * (size_t)nr * sizeof(double));
    double *xpa = (double *)malloc(L1 * 3 * (size_t)nr * sizeof(double));
    double *xca = (double *)malloc(L1 * 3 * (size_t)nr * sizeof(double));
    yo_cd *eia = (yo_cd *)malloc((size_t)nr * sizeof(yo_cd));
    yo_geometry(p, delta, azep, azst);
    yo_legendre_table(delta, nr, lmax, xa, xpa, xca);
    for (int k = 0; k < nr; k++) eia[k] = cexp(I_ * azst[k]);
    memset(ur, 0, (size_t)nw * nr * sizeof(yo_cd));
    memset(ut, 0, (size_t)nw * nr * sizeof(yo_cd));
    memset(up, 0, (size_t)nw * nr * sizeof(yo_cd));

    int nth = nthreads > 0 ? nthreads : (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nth < 1) nth = 1;
    if (jmax <= jofs) nth = 1;
    else if (nth > (jmax - 1 - jofs) / jstride + 1) nth = (jmax - 1 - jofs) / jstride + 1;
    yo_counts *tc = (yo_counts *)calloc((size_t)nth, sizeof(yo_counts));
    spectra_job job = {m, n, p, g, ur, ut, up, xa, xpa, xca, eia, lo, hi, jmax, jstride, 0,
                       jofs, ncol, PTHREAD_MUTEX_INITIALIZER};
    pthread_t *th = (pthread_t *)malloc((size_t)nth * sizeof(pthread_t));
    spectra_arg *args = (spectra_arg *)malloc((size_t)nth * sizeof(spectra_arg));
    for (int t = 0; t < nth; t++) {
        args[t].job = &job;
        args[t].cnt = &tc[t];
        pthread_create(&th[t], NULL, spectra_worker, &args[t]);
    }
    for (int t = 0; t < nth; t++) pthread_join(th[t], NULL);
    free(th);
    free(args);
    if (cnt) {
        for (int t = 0; t < nth; t++) {
            for (int q = 0; q < 16; q++) {
                cnt->nrhs[q] += tc[t].nrhs[q];
                cnt->nstep[q] += tc[t].nstep[q];
            }
            cnt->nsolve_tor += tc[t].nsolve_tor;
            cnt->nsolve_sph += tc[t].nsolve_sph;
            cnt->nsolve_rad += tc[t].nsolve_rad;
        }
    }
    free(tc); free(delta); free(azep); free(azst); free(xa); free(xpa); free(xca); free(eia);
    return 0;
}

int yo_spectra(const yo_model *m, const yo_norms *n, const yo_params *p,
               const yo_grid *g, yo_cd *ur, yo_cd *ut, yo_cd *up, int nthreads,
               int lsub_lo, int lsub_hi, int jsub, yo_counts *cnt)
{
    int lo = p->lmin, hi = p->lmax, nw = g->nw;
    if (lsub_hi >= 0) { lo = lsub_lo; hi = lsub_hi; }
    int jmax = nw, jstride = 1;
    if (jsub > 0 && jsub < nw) jmax = jsub;
    if (jsub < 0) jstride = -jsub;
    return spectra_run(m, n, p, g, ur, ut, up, nthreads, lo, hi, 0, jstride, jmax, 0, cnt);
}

/* The spectra of a frequency shard: column c (0-based) holds omega_j with  */
/* j = 1 + jofs + c jstride, c < count (the device's jofs/jstride fields).  */
int yo_spectra_shard(const yo_model *m, const yo_norms *n, const yo_params *p,
                     const yo_grid *g, int jofs, int jstride, int count, yo_cd *ur,
                     yo_cd *ut, yo_cd *up, int nthreads)
{
    if (jofs < 0 || jstride < 1 || count < 1 || jofs + (count - 1) * jstride >= g->nw)
        return YO_ERR_ARG;
    return spectra_run(m, n, p, g, ur, ut, up, nthreads, p->lmin, p->lmax, jofs, jstride,
                       jofs + (count - 1) * jstride + 1, count, NULL);
}

typedef struct {
    const yo_model *m;
    const yo_norms *n;
    const yo_params *p;
    const yo_grid *g;
    int npair;
    const int *ls, *js;
    yo_cd *coef;
    int next;
    pthread_mutex_t lock;
} coef_job;

static void *coef_worker(void *a)
{
    coef_job *jb = (coef_job *)a;
    for (;;) {
        pthread_mutex_lock(&jb->lock);
        int k = jb->next++;
        pthread_mutex_unlock(&jb->lock);
        if (k >= jb->npair) break;
        yo_solve_pair(jb->m, jb->n, jb->p, jb->g, jb->ls[k], jb->js[k], jb->coef + 15 * (size_t)k,
                      NULL);
    }
    return NULL;
}

/* yspec.f90:259-400 for a list of (l, omega_j) pairs, spread over threads */
int yo_coef_list(const yo_model *m, const yo_norms *n, const yo_params *p, const yo_grid *g,
                 int npair, const int *ls, const int *js, yo_cd *coef, int nthreads)
{
    for (int k = 0; k < npair; k++)
        if (ls[k] < 0 || js[k] < 1 || js[k] > g->nw) return YO_ERR_ARG;
    int nth = nthreads > 0 ? nthreads : (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nth < 1) nth = 1;
    if (nth > npair) nth = npair > 0 ? npair : 1;
    coef_job job = {m, n, p, g, npair, ls, js, coef, 0, PTHREAD_MUTEX_INITIALIZER};
    pthread_t *th = (pthread_t *)malloc((size_t)nth * sizeof(pthread_t));
    for (int t = 0; t < nth; t++) pthread_create(&th[t], NULL, coef_worker, &job);
    for (int t = 0; t < nth; t++) pthread_join(th[t], NULL);
    free(th);
    return 0;
}

/* The two-point solvers' outputs for one (omega, l): the solution at the   */
/* receiver radius for unit jumps at the source radius (module_solver.f90).  */
/* kind 0 tor_solver (2 x 2), 1 rad_solver_ng (2 x 2), 2 rad_solver_wg      */
/* (2 x 2), 3 sph_solver / sph_solver_fic (6 x 4), 4 the no-gravity and 5   */
/* the Cowling sph_solver variants (4 x 4).  out is row-major complex.      */
int yo_green(const yo_model *m, const yo_norms *n, int kind, int l, double wr, double wi,
             int ats, double rr, double rs, int ir, int is, yo_cd *out)
{
    yo_counts cnt;
    memset(&cnt, 0, sizeof cnt);
    yo_ctx c;
    memset(&c, 0, sizeof c);
    c.M = m;
    c.N = n;
    c.ats = (double)ats;
    c.cnt = &cnt;
    yo_cd w = wr + I_ * wi;
    if (ir < 1 || is < 1 || ir > m->nsl || is > m->nsl || l < 0) return YO_ERR_ARG;
    if (kind == 0) {
        yo_cd y[2][2];
        if (l < 2) return YO_ERR_ARG;
        yo_tor_solver(&c, l, w, rr, rs, ir, is, y);
        for (int a = 0; a < 2; a++) for (int b = 0; b < 2; b++) out[2 * a + b] = y[a][b];
    } else if (kind == 1 || kind == 2) {
        yo_cd y[2][2];
        if (kind == 1) yo_rad_solver_ng(&c, w, rr, rs, ir, is, y);
        else yo_rad_solver_wg(&c, w, rr, rs, ir, is, y, NULL);
        for (int a = 0; a < 2; a++) for (int b = 0; b < 2; b++) out[2 * a + b] = y[a][b];
    } else if (kind == 3) {
        yo_cd y[6][4];
        if (l < 1) return YO_ERR_ARG;
        yo_sph_solver_g(&c, l, w, rr, rs, ir, is, m->fic, y);
        for (int a = 0; a < 6; a++) for (int b = 0; b < 4; b++) out[4 * a + b] = y[a][b];
    } else if (kind == 4 || kind == 5) {
        yo_cd y[4][4];
        if (l < 1) return YO_ERR_ARG;
        yo_sph_solver_ngcow(&c, l, w, rr, rs, ir, is, m->fic, kind == 5, y);
        for (int a = 0; a < 4; a++) for (int b = 0; b < 4; b++) out[4 * a + b] = y[a][b];
    } else {
        return YO_ERR_ARG;
    }
    return 0;
}

/* module_fourier.f90:7-50 fourrow_dp on one row of length n */
static void fourrow(yo_cd *data, int n, int isign)
{
    int n2 = n / 2, j = n2;
    for (int i = 1; i <= n - 2; i++) {
        if (j > i) { yo_cd t = data[j]; data[j] = data[i]; data[i] = t; }
        int m = n2;
        for (;;) {
            if (m < 2 || j < m) break;
            j = j - m;
            m = m / 2;
        }
        j = j + m;
    }
    int mmax = 1;
    while (n > mmax) {
        int istep = 2 * mmax;
        double theta = YO_PI_D / (double)(isign * mmax);
        double s = sin(0.5 * theta);
        yo_cd wp = -2.0 * (s * s) + I_ * sin(theta);
        yo_cd w = 1.0;
        for (int m = 1; m <= mmax; m++) {
            yo_cd ws = w;
            for (int i = m; i <= n; i += istep) {
                int jj = i + mmax;
                yo_cd temp = ws * data[jj - 1];
                data[jj - 1] = data[i - 1] - temp;
                data[i - 1] = data[i - 1] + temp;
            }
            w = w * wp + w;
        }
        mmax = istep;
    }
}

/* module_fourier.f90:55-145 ifft + yspec.f90:433-486 post-processing */
int yo_traces(const yo_norms *n, const yo_params *p, const yo_grid *g, const yo_cd *ur,
              const yo_cd *ut, const yo_cd *up, const double *azep, double *out, int *nout_p)
{
    int nt = g->nt, nr = p->nr, nw = g->nw, i1 = g->i1, i2 = g->i2;
    double df = g->df, dt = g->dt;
    double w1 = g->f11, w2 = g->f12, w3 = g->f21, w4 = g->f22;
    int nofilt = (w1 == 0.0 && w2 == 0.0 && w3 == 0.0 && w4 == 0.0);
    double *filt = (double *)malloc(((size_t)nt / 2 + 2) * sizeof(double));
    double fprev = 0.0;
    for (int i = 1; i <= nt / 2 + 1; i++) {
        double w = (double)(i - 1) * df, f = fprev;
        if (w < w1) f = 0.0;
        else if (w >= w1 && w < w2) { f = YO_PI_D * (w - w1) / (w2 - w1); f = 0.5 * (1.0 - cos(f)); }
        else if (w >= w2 && w < w3) f = 1.0;
        else if (w >= w3 && w < w4) { f = YO_PI_D * (w4 - w) / (w4 - w3); f = 0.5 * (1.0 - cos(f)); }
        else if (w >= w4) f = 0.0;
        filt[i] = f;
        fprev = f;
    }
    int nout = nt;
    for (int i = 1; i <= nt; i++) {
        double t = (double)(i - 1) * dt;
        if (t > g->tout) { nout = i; break; }
    }
    double norm = p->out == 0 ? n->r_norm : (p->out == 1 ? n->vel_norm : n->acl_norm);
    yo_cd *row[3];
    for (int c = 0; c < 3; c++) row[c] = (yo_cd *)malloc((size_t)nt * sizeof(yo_cd));
    for (int k = 0; k < nr; k++) {
        const yo_cd *spec[3] = {ur + (size_t)nw * k, ut + (size_t)nw * k, up + (size_t)nw * k};
        for (int c = 0; c < 3; c++) {
            yo_cd *d = row[c];
            for (int i = 1; i <= nt; i++) d[i - 1] = 0.0;
            for (int i = i1; i <= i2; i++) d[i - 1] = spec[c][i - i1];
            if (!nofilt)
                for (int i = 1; i <= nt / 2 + 1; i++) d[i - 1] = filt[i] * d[i - 1];
            int jj = 0;
            for (int i = nt / 2 + 2; i <= nt; i++) {
                jj++;
                d[i - 1] = conj(d[nt / 2 - jj]);
            }
            fourrow(d, nt, 1);
            double sc = dt * (double)nt;
            for (int i = 0; i < nt; i++) d[i] = d[i] / sc;
            for (int i = 1; i <= nt; i++) {
                double t = (double)(i - 1) * dt;
                d[i - 1] = d[i - 1] * exp(g->ep * t);
            }
            for (int i = 0; i < nt; i++) d[i] = d[i] * norm;
        }
        double ca = cos(azep[k]), sa = sin(azep[k]);
        for (int i = 1; i <= nout; i++) {
            yo_cd t1 = row[1][i - 1], t2 = row[2][i - 1];
            yo_cd n_ = -(t1 * ca) + t2 * sa;
            yo_cd e_ = t1 * sa + t2 * ca;
            double t = (double)(i - 1) * dt * n->t_norm;
            size_t base = (size_t)(i - 1) + (size_t)nout * 4 * (size_t)k;
            out[base] = t;
            out[base + (size_t)nout] = creal(row[0][i - 1]);
            out[base + 2 * (size_t)nout] = creal(n_);
            out[base + 3 * (size_t)nout] = creal(e_);
        }
    }
    for (int c = 0; c < 3; c++) free(row[c]);
    free(filt);
    *nout_p = nout;
    return 0;
}

int yo_run(const char *param_file, double **out, int *nout, int *nr, int nthreads)
{
    yo_norms n;
    yo_params p;
    yo_model m;
    yo_grid g;
    yo_set_parameters(&n);
    int rc = yo_read_params(param_file, &p);
    if (rc) return rc;
    rc = yo_read_model(p.model_file, &n, &m);
    if (rc) { yo_free_params(&p); return rc; }
    rc = yo_event_setup(&m, &n, &p, &g);
    if (rc) { yo_free_model(&m); yo_free_params(&p); return rc; }
    size_t ns = (size_t)g.nw * p.nr;
    yo_cd *ur = (yo_cd *)malloc(ns * sizeof(yo_cd));
    yo_cd *ut = (yo_cd *)malloc(ns * sizeof(yo_cd));
    yo_cd *upp = (yo_cd *)malloc(ns * sizeof(yo_cd));
    yo_spectra(&m, &n, &p, &g, ur, ut, upp, nthreads, 0, -1, 0, NULL);
    double *delta = (double *)malloc((size_t)p.nr * sizeof(double));
    double *azep = (double *)malloc((size_t)p.nr * sizeof(double));
    double *azst = (double *)malloc((size_t)p.nr * sizeof(double));
    yo_geometry(&p, delta, azep, azst);
    int no = g.nt;
    for (int i = 1; i <= g.nt; i++)
        if ((double)(i - 1) * g.dt > g.tout) { no = i; break; }
    *out = (double *)malloc((size_t)no * 4 * p.nr * sizeof(double));
    yo_traces(&n, &p, &g, ur, ut, upp, azep, *out, nout);
    *nr = p.nr;
    free(ur); free(ut); free(upp); free(delta); free(azep); free(azst);
    yo_free_model(&m);
    yo_free_params(&p);
    return 0;
}

/* gfortran E15.6: [-]0.dddddd E+ee right-justified in 15 columns */
static void fmt_e15_6(double x, char *buf)
{
    char tmp[64], s[32];
    int neg = signbit(x) ? 1 : 0;
    double ax = fabs(x);
    int e10;
    char dig[8];
    if (ax == 0.0) {
        memcpy(dig, "000000", 7);
        e10 = 0;
    } else {
        snprintf(tmp, sizeof tmp, "%.5e", ax);
        dig[0] = tmp[0];
        memcpy(dig + 1, tmp + 2, 5);
        dig[6] = 0;
        e10 = atoi(strchr(tmp, 'e') + 1) + 1;
    }
    int ae = e10 < 0 ? -e10 : e10;
    if (ae <= 99)
        snprintf(s, sizeof s, "%s0.%sE%c%02d", neg ? "-" : "", dig, e10 < 0 ? '-' : '+', ae);
    else
        snprintf(s, sizeof s, "%s0.%s%c%03d", neg ? "-" : "", dig, e10 < 0 ? '-' : '+', ae);
    snprintf(buf, 16, "%15.15s", s);
}

/* yspec.f90:488-503 and module_util.f90:428-444 string_cat_int */
int yo_write_traces(const char *pref_out, const double *out, int nout, int nr)
{
    char path[600], line[128], f[4][16];
    for (int k = 1; k <= nr; k++) {
        char stmp[16];
        snprintf(stmp, sizeof stmp, "%10d", k);
        int j = (int)floorf(log10f((float)k));
        snprintf(path, sizeof path, "%s.%s", pref_out, stmp + (9 - j));
        FILE *fp = fopen(path, "w");
        if (!fp) return YO_ERR_IO;
        for (int i = 0; i < nout; i++) {
            for (int c = 0; c < 4; c++)
                fmt_e15_6(out[(size_t)i + (size_t)nout * ((size_t)c + 4 * (size_t)(k - 1))], f[c]);
            snprintf(line, sizeof line, "%s%s%s%s\n", f[0], f[1], f[2], f[3]);
            fputs(line, fp);
        }
        fclose(fp);
    }
    return 0;
}
