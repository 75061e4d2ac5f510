/*
 * yo_solver.c -- oracle restatement of module_int.f90, module_start.f90,
 * module_solver.f90 and the sbessj2/bfs_dum start-value helpers of
 * module_function.f90.  TEST INFRASTRUCTURE ONLY (see yo.h).
 *
 * The reference keeps the per-solve state (l, omega, current layer) in
 * module globals (module_int.f90:93-117); here it travels in a context
 * struct so solves can run concurrently.  Expression order follows the
 * Fortran (left to right, real-by-complex products stay real-by-complex).
 */
#include "yo.h"
#include "yo_const.h"
#include "yo_internal.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define I_ (_Complex_I)

/* ------------------------------------------------------------------------ */
/* module_int.f90:2072-2118 set_l, set_omega, set_ats                       */
/* ------------------------------------------------------------------------ */
void yo_set_l(yo_ctx *c, int l)
{
    c->ll = l;
    c->llp1 = l + 1;
    c->zeta2 = (double)(float)(c->ll * c->llp1);
    c->zeta = sqrt(c->zeta2);
    c->zeta2m2 = c->zeta2 - 2.0;
    c->szeta2m2 = c->zeta2m2 > 0.0 ? sqrt(c->zeta2m2) : 0.0;
    c->nu = (double)(float)(2 * c->ll + 1) / YO_FOURPI_D;
    c->nu = sqrt(c->nu);
}

void yo_set_omega(yo_ctx *c, yo_cd w)
{
    c->omega = w;
    c->omega2 = w * w;
    c->omegai = 1.0 / w;
    c->omegai2 = c->omegai * c->omegai;
    yo_cd z = (I_ * c->omega) / c->M->tref;
    c->lno = 2.0 * clog(z) / YO_PI_D;
    c->lno = c->ats * c->lno;
}

/* module_int.f90:2121-2138 steps */
static double steps(const yo_ctx *c, int i1)
{
    const yo_model *m = c->M;
    double tmp = i1 < m->nknot ? fmax(m->alpha[i1], m->alpha[i1 + 1]) : m->alpha[i1];
    double s = (double)YO_NW * creal(c->omega) / tmp;
    return 1.0 / s;
}

static int iminloc(const double *a, int lo, int hi)
{
    int im = lo;
    for (int i = lo + 1; i <= hi; i++)
        if (a[i] < a[im]) im = i;
    return im;
}

/* module_int.f90:188-209 tor_steps; :394-414 rad_steps; :1145-1166 sph_steps */
static void tor_steps(yo_ctx *c)
{
    int im = iminloc(c->M->beta, c->M->noc + 1, c->M->nsl);
    if (creal(c->omega) == 0.0) c->dr = 1.0 / YO_NW;
    else c->dr = 1.0 / ((double)YO_NW * creal(c->omega) / c->M->beta[im]);
}

static void alpha_steps(yo_ctx *c)
{
    int im = iminloc(c->M->alpha, 1, c->M->nknot);
    if (creal(c->omega) == 0.0) c->dr = 1.0 / YO_NW;
    else c->dr = 1.0 / ((double)YO_NW * creal(c->omega) / c->M->alpha[im]);
}

#define SPL(name, rr, k) yo_splint_dis(m->r, m->name, m->name##_cs, rr, k)

/* ------------------------------------------------------------------------ */
/* Toroidal system, module_int.f90:134-184                                  */
/* ------------------------------------------------------------------------ */
static void tor_derivs(yo_ctx *c, double rr, const yo_cd *y, yo_cd *dydx)
{
    const yo_model *m = c->M;
    int il = c->il;
    double rrho = SPL(rho, rr, il), rlcon = SPL(lcon, rr, il);
    double rncon = SPL(ncon, rr, il), rqmu = SPL(qmu, rr, il);
    yo_cd qll = 1.0 + rqmu * c->lno;
    yo_cd clcon = rlcon * qll, cncon = rncon * qll;
    double ri = 1.0 / rr;
    double t = 2.0 * ri;
    yo_cd k = 1.0 / clcon;
    yo_cd s = -(c->omega2 * rrho) + ri * ri * c->zeta2m2 * cncon;
    dydx[0] = t * y[0] + k * y[1];
    dydx[1] = s * y[0] - t * y[1];
    c->cnt->nrhs[2]++;
}

/* ------------------------------------------------------------------------ */
/* Radial system, module_int.f90:261-392.  rad_derivs_ng calls the gravity  */
/* matrix rad_amat (module_int.f90:388), which is kept here.                */
/* ------------------------------------------------------------------------ */
static void rad_amat(yo_ctx *c, double rr, yo_cd *t, yo_cd *k, yo_cd *s)
{
    const yo_model *m = c->M;
    int il = c->il;
    double rrho = SPL(rho, rr, il), racon = SPL(acon, rr, il);
    double rccon = SPL(ccon, rr, il), rfcon = SPL(fcon, rr, il);
    double rncon = SPL(ncon, rr, il), gg = SPL(grav, rr, il);
    double rqmu = SPL(qmu, rr, il), rxlam = SPL(xlam, rr, il);
    double rxa2 = SPL(xa2, rr, il);
    yo_cd qaa = 1.0 + rxa2 * c->lno, qff = 1.0 + rxlam * c->lno;
    yo_cd qll = 1.0 + rqmu * c->lno;
    yo_cd cacon = racon * qaa, cccon = rccon * qaa, cfcon = rfcon * qff;
    yo_cd cncon = rncon * qll;
    cccon = 1.0 / cccon;
    yo_cd gamma = cacon - cncon - cfcon * cfcon * cccon;
    double ri = 1.0 / rr;
    *t = (1.0 - 2.0 * cfcon * cccon) * ri;
    *k = cccon;
    *s = -(c->omega2 * rrho) + 4.0 * (gamma - rrho * gg * rr) * ri * ri;
}

static void rad_derivs(yo_ctx *c, double rr, const yo_cd *y, yo_cd *dydx)
{
    yo_cd t, k, s;
    rad_amat(c, rr, &t, &k, &s);
    dydx[0] = t * y[0] + k * y[1];
    dydx[1] = s * y[0] - t * y[1];
    c->cnt->nrhs[2]++;
}

/* ------------------------------------------------------------------------ */
/* Spheroidal coefficient matrices, module_int.f90:500-786                  */
/* ------------------------------------------------------------------------ */
typedef struct {
    yo_cd t11, t12, t21, t22, t31, t33, k11, k22, k33, s11, s12, s13, s22, s23;
} sph_coef;

static void sph_solid_amat(yo_ctx *c, double rr, int kind, sph_coef *a)
{
    /* kind: 2 = full gravity (:500-560), 0 = no gravity (:564-616),
     *       1 = Cowling (:619-672) */
    const yo_model *m = c->M;
    int il = c->il;
    double rrho = SPL(rho, rr, il), racon = SPL(acon, rr, il);
    double rccon = SPL(ccon, rr, il), rfcon = SPL(fcon, rr, il);
    double rncon = SPL(ncon, rr, il), rlcon = SPL(lcon, rr, il);
    double gg = kind != 0 ? SPL(grav, rr, il) : 0.0;
    double rqmu = SPL(qmu, rr, il), rxlam = SPL(xlam, rr, il);
    double rxa2 = SPL(xa2, rr, il);
    yo_cd qaa = 1.0 + rxa2 * c->lno, qff = 1.0 + rxlam * c->lno;
    yo_cd qll = 1.0 + rqmu * c->lno;
    yo_cd cacon = racon * qaa, cccon = rccon * qaa, cfcon = rfcon * qff;
    yo_cd cncon = rncon * qll, clcon = rlcon * qll;
    cccon = 1.0 / cccon;
    yo_cd gamma = cacon - cncon - cfcon * cfcon * cccon;
    double ri = 1.0 / rr;
    double pib = c->N->pibigg;
    a->t11 = (1.0 - 2.0 * cfcon * cccon) * ri;
    a->t12 = c->zeta * ri * cfcon * cccon;
    a->t21 = -(c->zeta * ri);
    a->t22 = 2.0 * ri;
    a->k11 = cccon;
    a->k22 = 1.0 / clcon;
    a->s22 = -(c->omega2 * rrho) + (c->zeta2 * (gamma + cncon) - 2.0 * cncon) * ri * ri;
    if (kind == 0) {
        a->s11 = -(c->omega2 * rrho) + 4.0 * gamma * ri * ri;
        a->s12 = -2.0 * c->zeta * gamma * ri * ri;
    } else {
        a->s11 = -(c->omega2 * rrho) + 4.0 * (gamma - rrho * gg * rr) * ri * ri;
        a->s12 = c->zeta * (rrho * gg * rr - 2.0 * gamma) * ri * ri;
    }
    if (kind == 2) {
        a->t31 = -(4 * pib * rrho);
        a->t33 = -((double)c->ll * ri);
        a->k33 = 4.0 * pib;
        a->s13 = -(rrho * (double)c->llp1 * ri);
        a->s23 = rrho * c->zeta * ri;
    }
}

static void sph_fluid_amat(yo_ctx *c, double rr, int kind, sph_coef *a)
{
    /* kind 2: module_int.f90:676-715; 0: :720-747; 1: :751-786 */
    const yo_model *m = c->M;
    int il = c->il;
    double rrho = SPL(rho, rr, il), rccon = SPL(ccon, rr, il);
    double gg = kind != 0 ? SPL(grav, rr, il) : 0.0;
    double rxa2 = SPL(xa2, rr, il);
    yo_cd qaa = 1.0 + rxa2 * c->lno;
    yo_cd cccon = rccon * qaa;
    cccon = 1.0 / cccon;
    double ri = 1.0 / rr;
    double pib = c->N->pibigg;
    yo_cd k = cccon - c->zeta2 * c->omegai2 * ri * ri / rrho;
    if (kind == 2) {
        a->t11 = (gg * c->zeta2 * c->omegai2 * ri - 1.0) * ri;
        a->t12 = c->zeta2 * c->omegai2 * ri * ri;
        a->t21 = -4.0 * pib * rrho;
        a->t22 = -((double)c->ll * ri);
        a->k11 = k;
        a->k22 = 4.0 * pib;
        a->s11 = -(c->omega2 * rrho) +
                 rrho * gg * (gg * c->zeta2 * ri * c->omegai2 - 4.0) * ri;
        a->s12 = rrho * (gg * c->zeta2 * ri * c->omegai2 - (double)c->llp1) * ri;
        a->s22 = rrho * c->zeta2 * ri * ri * c->omegai2;
    } else if (kind == 0) {
        a->t11 = -ri;
        a->k11 = k;
        a->s11 = -(c->omega2 * rrho);
    } else {
        a->t11 = (gg * c->zeta2 * c->omegai2 * ri - 1.0) * ri;
        a->k11 = k;
        a->s11 = -(c->omega2 * rrho) +
                 rrho * gg * (gg * c->zeta2 * ri * c->omegai2 - 4.0) * ri;
    }
}

/* module_int.f90:818-871 sph_minors_solid_derivs (14 components) */
static void minors_solid_g(yo_ctx *c, double rr, const yo_cd *m, yo_cd *d)
{
    sph_coef a;
    sph_solid_amat(c, rr, 2, &a);
    yo_cd t11 = a.t11, t12 = a.t12, t21 = a.t21, t22 = a.t22, t31 = a.t31;
    yo_cd t33 = a.t33, k11 = a.k11, k22 = a.k22, k33 = a.k33, s11 = a.s11;
    yo_cd s12 = a.s12, s13 = a.s13, s22 = a.s22, s23 = a.s23;
    yo_cd a123 = t11 + t22 + t33, a126 = t11 + t22 - t33;
    yo_cd a135 = t11 - t22 + t33, a234 = -t11 + t22 + t33;
    /* m(k) is m[k-1] */
    d[0] = k33 * m[3] - k22 * m[5] + k11 * m[9] + m[0] * a123;
    d[1] = -k22 * m[6] + m[0] * s13 - m[2] * t21 + m[1] * t22 - m[3] * t31;
    d[2] = -k11 * m[10] + m[0] * s23 + m[2] * t11 - m[1] * t12;
    d[3] = k22 * m[8] - k11 * m[11] + m[3] * a126;
    d[4] = -k33 * m[7] - m[0] * s12 + m[9] * t12 - m[5] * t21 + m[2] * t31 + m[4] * t33;
    d[5] = -k33 * m[8] - k11 * m[12] - m[0] * s22 - 2.0 * m[4] * t12 + m[5] * a135;
    d[6] = m[2] * s12 + m[5] * s13 - m[1] * s22 - m[4] * s23 + m[10] * t12 -
           m[6] * t22 + m[8] * t31;
    d[7] = m[3] * s12 - m[2] * s13 - m[1] * s23 + m[11] * t12 - m[8] * t21 - m[7] * t33;
    d[8] = k11 * m[13] + m[3] * s22 - 2.0 * m[2] * s23 - 2.0 * m[7] * t12 - m[8] * a234;
    d[9] = -k33 * m[11] + k22 * m[12] + m[0] * s11 + 2.0 * m[4] * t21 -
           2.0 * m[1] * t31 + m[9] * a234;
    d[10] = -m[2] * s11 + m[1] * s12 - m[4] * s13 - m[9] * s23 - m[10] * t11 +
            m[6] * t21 - m[7] * t31;
    d[11] = -k22 * m[13] - m[3] * s11 + 2.0 * m[1] * s13 + 2.0 * m[7] * t21 - m[11] * a135;
    d[12] = k33 * m[13] - m[5] * s11 + 2.0 * m[4] * s12 + m[9] * s22 +
            2.0 * m[6] * t31 - m[12] * a126;
    d[13] = m[8] * s11 - 2.0 * m[7] * s12 + 2.0 * m[6] * s13 - m[11] * s22 +
            2.0 * m[10] * s23 - m[13] * a123;
    c->cnt->nrhs[14]++;
}

/* module_int.f90:874-936 sph_minors_solid_derivs_ng / _cow (5 components) */
static void minors_solid_ngcow(yo_ctx *c, double rr, const yo_cd *m, yo_cd *d, int kind)
{
    sph_coef a;
    sph_solid_amat(c, rr, kind, &a);
    yo_cd a11 = a.t11 + a.t22, a22 = a.t11 - a.t22;
    d[0] = a11 * m[0] + a.k22 * m[2] - a.k11 * m[3];
    d[1] = a.s12 * m[0] - a.t21 * m[2] + a.t12 * m[3];
    d[2] = a.s22 * m[0] - 2.0 * a.t12 * m[1] + a22 * m[2] + a.k11 * m[4];
    d[3] = -a.s11 * m[0] + 2.0 * a.t21 * m[1] - a22 * m[3] - a.k22 * m[4];
    d[4] = -2.0 * a.s12 * m[1] + a.s11 * m[2] - a.s22 * m[3] - a11 * m[4];
    c->cnt->nrhs[5]++;
}
static void minors_solid_ng(yo_ctx *c, double rr, const yo_cd *m, yo_cd *d)
{ minors_solid_ngcow(c, rr, m, d, 0); }
static void minors_solid_cow(yo_ctx *c, double rr, const yo_cd *m, yo_cd *d)
{ minors_solid_ngcow(c, rr, m, d, 1); }

/* module_int.f90:941-967 sph_minors_fluid_derivs (5 components) */
static void minors_fluid_g(yo_ctx *c, double rr, const yo_cd *m, yo_cd *d)
{
    sph_coef a;
    sph_fluid_amat(c, rr, 2, &a);
    d[0] = a.k22 * m[2] - a.k11 * m[3] + m[0] * (a.t11 + a.t22);
    d[1] = m[0] * a.s12 + m[3] * a.t12 - m[2] * a.t21;
    d[2] = a.k11 * m[4] + m[0] * a.s22 - 2.0 * m[1] * a.t12 + m[2] * (a.t11 - a.t22);
    d[3] = -a.k22 * m[4] - m[0] * a.s11 + 2.0 * m[1] * a.t21 + m[3] * (-a.t11 + a.t22);
    d[4] = m[2] * a.s11 - 2.0 * m[1] * a.s12 - m[3] * a.s22 - m[4] * (a.t11 + a.t22);
    c->cnt->nrhs[5]++;
}

/* module_int.f90:971-1012 sph_minors_fluid_derivs_ng / _cow (2 components) */
static void minors_fluid_ngcow(yo_ctx *c, double rr, const yo_cd *m, yo_cd *d, int kind)
{
    sph_coef a;
    sph_fluid_amat(c, rr, kind, &a);
    d[0] = a.t11 * m[0] + a.k11 * m[1];
    d[1] = a.s11 * m[0] - a.t11 * m[1];
    c->cnt->nrhs[2]++;
}
static void minors_fluid_ng(yo_ctx *c, double rr, const yo_cd *m, yo_cd *d)
{ minors_fluid_ngcow(c, rr, m, d, 0); }
static void minors_fluid_cow(yo_ctx *c, double rr, const yo_cd *m, yo_cd *d)
{ minors_fluid_ngcow(c, rr, m, d, 1); }

/* module_int.f90:1016-1057 sph_bvec_solid_derivs (14 components) */
static void bvec_solid_g(yo_ctx *c, double rr, const yo_cd *b, yo_cd *d)
{
    sph_coef a;
    sph_solid_amat(c, rr, 2, &a);
    yo_cd t11 = a.t11, t12 = a.t12, t21 = a.t21, t22 = a.t22, t31 = a.t31;
    yo_cd t33 = a.t33, k11 = a.k11, k22 = a.k22, k33 = a.k33, s11 = a.s11;
    yo_cd s12 = a.s12, s13 = a.s13, s22 = a.s22, s23 = a.s23;
    d[0] = s11 * b[6] + s12 * (b[7] - b[2]) + s13 * b[8] - s22 * b[3] - s23 * b[4] -
           (t11 + t22) * b[0] + t31 * b[5];
    d[1] = s11 * b[9] + s12 * b[10] - s13 * (2.0 * b[2] + b[7]) - s23 * b[3] -
           t21 * b[5] - (t11 + t33) * b[1];
    d[2] = s12 * b[11] + s13 * b[12] + t12 * b[3] - t21 * b[6] - t31 * b[9];
    d[3] = -k22 * b[0] - s11 * b[11] + s13 * b[13] + t21 * (b[2] - b[7]) +
           (t22 - t11) * b[3] - t31 * b[10];
    d[4] = -k33 * b[1] - s11 * b[12] - s12 * b[13] - t21 * b[8] +
           t31 * (2.0 * b[2] + b[7]) + (t33 - t11) * b[4];
    d[5] = s12 * b[9] - s13 * b[6] + s22 * b[10] - s23 * (b[2] + 2.0 * b[7]) -
           t12 * b[1] - (t22 + t33) * b[5];
    d[6] = k11 * b[0] + s22 * b[11] + s23 * b[12] - t12 * (b[2] - b[7]) + (t11 - t22) * b[6];
    d[7] = -s12 * b[11] + s23 * b[13] - t12 * b[3] + t21 * b[6];
    d[8] = -k33 * b[5] - s12 * b[12] - s22 * b[13] - t12 * b[4] - t22 * b[8] +
           t31 * b[6] + t33 * b[8];
    d[9] = k11 * b[1] + s23 * b[11] + t12 * b[10] + (t11 - t33) * b[9];
    d[10] = k22 * b[5] - s13 * b[11] + t21 * b[9] + (t22 - t33) * b[10];
    d[11] = -k11 * b[3] + k22 * b[6] + (t11 + t22) * b[11];
    d[12] = -k11 * b[4] + k33 * b[9] + t12 * b[13] + (t11 + t33) * b[12];
    d[13] = -k22 * b[8] + k33 * b[10] + t21 * b[12] - t31 * b[11] + (t22 + t33) * b[13];
    c->cnt->nrhs[14]++;
}

/* module_int.f90:1060-1110 sph_bvec_solid_derivs_ng / _cow (4 components) */
static void bvec_solid_ngcow(yo_ctx *c, double rr, const yo_cd *b, yo_cd *d, int kind)
{
    sph_coef a;
    sph_solid_amat(c, rr, kind, &a);
    d[0] = -a.s11 * b[2] - a.s12 * b[3] - a.t11 * b[0] - a.t21 * b[1];
    d[1] = -a.s12 * b[2] - a.s22 * b[3] - a.t12 * b[0] - a.t22 * b[1];
    d[2] = -a.k11 * b[0] + a.t11 * b[2] + a.t12 * b[3];
    d[3] = -a.k22 * b[1] + a.t21 * b[2] + a.t22 * b[3];
    c->cnt->nrhs[4]++;
}
static void bvec_solid_ng(yo_ctx *c, double rr, const yo_cd *m, yo_cd *d)
{ bvec_solid_ngcow(c, rr, m, d, 0); }
static void bvec_solid_cow(yo_ctx *c, double rr, const yo_cd *m, yo_cd *d)
{ bvec_solid_ngcow(c, rr, m, d, 1); }

/* ------------------------------------------------------------------------ */
/* module_int.f90:1847-1968 yint and :2016-2064 rkck                        */
/* ------------------------------------------------------------------------ */
static void rkck(yo_ctx *c, const yo_cd *y, const yo_cd *dydx, double x, double h,
                 yo_cd *yout, int n, yo_derivs derivs)
{
    static const double a2 = 0.2, a3 = 0.3, a4 = 0.6, a5 = 1.0, a6 = 0.875;
    static const double b21 = 0.2, b31 = 3.0 / 40.0, b32 = 9.0 / 40.0;
    static const double b41 = 0.3, b42 = -0.9, b43 = 1.2;
    static const double b51 = -11.0 / 54.0, b52 = 2.5, b53 = -70.0 / 27.0,
                        b54 = 35.0 / 27.0;
    static const double b61 = 1631.0 / 55296.0, b62 = 175.0 / 512.0,
                        b63 = 575.0 / 13824.0, b64 = 44275.0 / 110592.0,
                        b65 = 253.0 / 4096.0;
    static const double c1 = 37.0 / 378.0, c3 = 250.0 / 621.0,
                        c4 = 125.0 / 594.0, c6 = 512.0 / 1771.0;
    yo_cd ak2[14], ak3[14], ak4[14], ak5[14], ak6[14], yt[14];
    for (int i = 0; i < n; i++) yt[i] = y[i] + b21 * h * dydx[i];
    derivs(c, x + a2 * h, yt, ak2);
    for (int i = 0; i < n; i++) yt[i] = y[i] + h * (b31 * dydx[i] + b32 * ak2[i]);
    derivs(c, x + a3 * h, yt, ak3);
    for (int i = 0; i < n; i++)
        yt[i] = y[i] + h * (b41 * dydx[i] + b42 * ak2[i] + b43 * ak3[i]);
    derivs(c, x + a4 * h, yt, ak4);
    for (int i = 0; i < n; i++)
        yt[i] = y[i] + h * (b51 * dydx[i] + b52 * ak2[i] + b53 * ak3[i] + b54 * ak4[i]);
    derivs(c, x + a5 * h, yt, ak5);
    for (int i = 0; i < n; i++)
        yt[i] = y[i] + h * (b61 * dydx[i] + b62 * ak2[i] + b63 * ak3[i] +
                            b64 * ak4[i] + b65 * ak5[i]);
    derivs(c, x + a6 * h, yt, ak6);
    for (int i = 0; i < n; i++)
        yout[i] = y[i] + h * (c1 * dydx[i] + c3 * ak3[i] + c4 * ak4[i] + c6 * ak6[i]);
}

/* Step refinement for the oracle's own convergence checks: each knot       */
/* interval takes (ns - 1) * refine steps instead of the reference's ns - 1. */
/* 1 (the default) is the reference's rule.  Process-wide; not for use while */
/* other threads run the oracle.                                             */
static int g_step_refine = 1;

void yo_set_step_refine(int refine) { g_step_refine = refine < 1 ? 1 : refine; }

void yo_yint(yo_ctx *c, int i1, int i2, double r1, double r2, yo_cd *y, int n,
             yo_derivs derivs, int *scale)
{
    const yo_model *m = c->M;
    yo_cd dydx[14];
    int up;
    if (r2 > r1) up = 1;
    else if (r2 < r1) up = 0;
    else return;
    int istep = up ? 1 : -1;
    for (int i = i1; up ? (i <= i2) : (i >= i2); i += istep) {
        double rr1, rr2;
        if (up) {
            rr1 = (i == i1) ? r1 : m->r[i];
            rr2 = (i == i2) ? r2 : m->r[i + 1];
        } else {
            rr1 = (i == i1) ? r1 : m->r[i + 1];
            rr2 = (i == i2) ? r2 : m->r[i];
        }
        if (rr1 == rr2) continue;
        c->il = i;
        double drr = steps(c, i);
        int ns = 2 + (int)floor(fabs(rr2 - rr1) / drr);
        if (g_step_refine > 1) ns = (ns - 1) * g_step_refine + 1;
        drr = (rr2 - rr1) / (double)(ns - 1);
        for (int j = 1; j <= ns - 1; j++) {
            double rr = rr1 + (double)(j - 1) * drr;
            derivs(c, rr, y, dydx);
            rkck(c, y, dydx, rr, drr, y, n, derivs);
            c->cnt->nstep[n]++;
            if (scale) {
                int all_small = 1, any_big = 0;
                for (int k = 0; k < n; k++)
                    if (!(cabs(y[k]) < YO_TINY)) { all_small = 0; break; }
                if (all_small) {
                    (*scale)++;
                    for (int k = 0; k < n; k++) y[k] = y[k] * YO_HUGE;
                }
                for (int k = 0; k < n; k++)
                    if (cabs(y[k]) > YO_HUGE) { any_big = 1; break; }
                if (any_big) {
                    (*scale)--;
                    for (int k = 0; k < n; k++) y[k] = y[k] * YO_TINY;
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* module_start.f90:80-178 start_level, :14-32 tor_, :35-75 sph_start_level */
/* ------------------------------------------------------------------------ */
static int start_level(const yo_model *m, int l, double w, int i1, int i2, int wt)
{
    int isign = (i2 >= i1) ? 1 : -1;
    double pp = (double)(float)(l * (l + 1)) / (w * w);
    const double *v = (wt == 1) ? m->beta : m->alpha;
    int j = i2;
    for (int i = i1; isign == 1 ? i <= i2 : i >= i2; i += isign) {
        double q1 = 1.0 / (v[i] * v[i]) - pp / (m->r[i] * m->r[i]);
        if (isign == 1) {
            if (q1 > 0.0) { j = (i - 1 > i1) ? i - 1 : i1; break; }
        } else {
            if (q1 < 0.0) { j = i; break; }
        }
    }
    int is = j;
    int lo = i1 < i2 ? i1 : i2;
    if (is == lo) return is;
    int j1 = is, j2 = lo;
    is = j2;
    double sum = 0.0;
    for (int i = j1; i >= j2 + 1; i--) {
        double q1 = 1.0 / (v[i] * v[i]) - pp / (m->r[i] * m->r[i]);
        double q2 = 1.0 / (v[i - 1] * v[i - 1]) - pp / (m->r[i - 1] * m->r[i - 1]);
        if (q1 > 0.0 || q2 > 0.0) {
            sum = 0.0;
        } else {
            q1 = sqrt(-q1);
            q2 = sqrt(-q2);
            sum = sum + 0.5 * w * (q1 + q2) * (m->r[i] - m->r[i - 1]);
        }
        if (sum > YO_TOL_START) { is = i - 1; break; }
    }
    return is;
}

int yo_tor_start_level(const yo_model *m, int l, double w, int it)
{
    return start_level(m, l, w, m->noc + 1, it, 1);
}

int yo_sph_start_level(const yo_model *m, const yo_norms *n, int l, double w, int it)
{
    const double aw = -2.00e-3, bw = 2.25e-3, dw = 1.28e-3;
    double wdim = w * n->fre_norm;
    double wsoc = aw + dw * (double)l;
    int is;
    if (wdim <= wsoc) {
        is = start_level(m, l, w, m->noc + 1, it, 1);
        if (is == m->nsl) is = is - 1;
        if (is > m->noc + 1) return is;
    }
    double wsic = aw + bw * (double)l;
    if (wdim <= wsic) {
        is = start_level(m, l, w, m->nic + 1, m->noc, 2);
        if (is == m->noc) is = is - 1;
        if (is > m->nic + 1) return is;
    }
    if (m->fic) is = start_level(m, l, w, 2, m->nic, 2);
    else is = start_level(m, l, w, 2, m->nic, 1);
    if (is == m->nic) is = is - 1;
    return is;
}

/* ------------------------------------------------------------------------ */
/* Start values.  sbessj2 (module_function.f90:447-490) is a stub returning */
/* x/(2l+3); bfs_dum (:497-516) uses sqrt(|x^2|) as the argument.            */
/* ------------------------------------------------------------------------ */
static yo_cd sbessj2(int l, yo_cd x) { return x / (double)(float)(2 * l + 3); }

static yo_cd bfs_dum(int l, yo_cd xsq)
{
    yo_cd fp;
    yo_bfs(l, xsq, 1.e-9, &fp);
    double x = sqrt(cabs(xsq));
    return ((double)l - fp) / x;
}

/* module_int.f90:213-250 tor_ystart */
static void tor_ystart(yo_ctx *c, int is, double rr, yo_cd *y)
{
    const yo_model *m = c->M;
    double rrho = SPL(rho, rr, is), rmu = SPL(mu, rr, is), rqmu = SPL(qmu, rr, is);
    yo_cd qll = 1.0 + rqmu * c->lno;
    yo_cd cmu = rmu * qll;
    yo_cd cbeta = csqrt(cmu / rrho);
    yo_cd kbeta = c->omega / cbeta;
    yo_cd arg = kbeta * rr;
    yo_cd ratio = sbessj2(c->llp1, arg);
    y[0] = rr;
    y[1] = cmu * ((double)(c->ll - 1) - arg * ratio);
    y[0] = c->zeta * y[0];
    y[1] = c->zeta * y[1];
}

/* module_int.f90:417-489 rad_ystart (grav=1) / rad_ystart_ng (grav=0) */
static void rad_ystart(yo_ctx *c, int is, double rr, yo_cd *y, int grav)
{
    const yo_model *m = c->M;
    double rrho = SPL(rho, rr, is), rmu = SPL(mu, rr, is), rqmu = SPL(qmu, rr, is);
    double rkappa = SPL(kappa, rr, is), rqkappa = SPL(qkappa, rr, is);
    yo_cd cmu = rmu * (1.0 + rqmu * c->lno);
    yo_cd ckappa = rkappa * (1.0 + rqkappa * c->lno);
    yo_cd calpha = ckappa + 4.0 * cmu / 3.0;
    yo_cd gamma;
    if (grav) gamma = c->omega2 + 16.0 * c->N->pibigg * rrho / 3.0;
    else gamma = c->omega2;
    gamma = rrho * gamma / calpha;
    yo_cd arg = gamma * rr;
    yo_cd ratio = sbessj2(1, arg);
    y[0] = rr * ratio;
    y[1] = rr * calpha * gamma - 4.0 * cmu * ratio;
}

/* module_int.f90:1192-1270 sph_solid_start; y is y[row-1][col-1] */
static void sph_solid_start(yo_ctx *c, int is, double rr, yo_cd y[6][3])
{
    const yo_model *m = c->M;
    double pib = c->N->pibigg;
    double rrho = SPL(rho, rr, is), rmu = SPL(mu, rr, is), rqmu = SPL(qmu, rr, is);
    double rkappa = SPL(kappa, rr, is), rqkappa = SPL(qkappa, rr, is);
    yo_cd cmu = rmu * (1.0 + rqmu * c->lno);
    yo_cd ckappa = rkappa * (1.0 + rqkappa * c->lno);
    yo_cd calpha = (ckappa + 1.3333333333 * cmu) / rrho;
    yo_cd cbeta = cmu / rrho;
    double sign = 1.0;
    yo_cd tmp1 = c->omega2 / cbeta;
    yo_cd tmp2 = c->omega2 + 5.3333333 * pib * rrho;
    tmp2 = tmp2 / calpha;
    yo_cd tmp3 = 2.666666666 * pib * c->zeta * rrho;
    tmp3 = tmp3 * tmp3 / (calpha * cbeta);
    double ll = (double)c->ll, llp1 = (double)c->llp1;
    for (int i = 0; i < 2; i++) {
        yo_cd d = tmp1 - tmp2;
        yo_cd gamma = d * d + tmp3;
        gamma = 0.5 * (tmp1 + tmp2) + 0.5 * sign * csqrt(gamma);
        yo_cd gamma2 = gamma;
        gamma = csqrt(gamma);
        yo_cd zt = 0.75 * cbeta * (gamma2 - tmp1) / (pib * rrho);
        yo_cd xi = zt - llp1;
        yo_cd args = gamma2 * rr * rr;
        yo_cd ratio = bfs_dum(c->ll, args);
        y[0][i] = ll * xi - zt * gamma * rr * ratio;
        y[1][i] = c->zeta * (xi + rr * gamma * ratio);
        y[2][i] = -(4.0 * pib * rrho * rr * zt);
        y[3][i] = -(rrho * calpha * zt * rr * gamma2) + 2.0 * cmu * ll * (ll - 1.0) * xi / rr +
                  2.0 * cmu * (2.0 * zt + c->zeta2) * gamma * ratio;
        y[4][i] = rr * gamma2 + 2.0 * (ll - 1.0) * xi / rr - 2.0 * (zt + 1.0) * gamma * ratio;
        y[4][i] = cmu * c->zeta * y[4][i];
        y[5][i] = -(rrho * (c->zeta2 + llp1 * zt));
        sign = -sign;
    }
    y[0][2] = ll;
    y[1][2] = c->zeta;
    y[2][2] = (c->omega2 - 4.0 * pib * rrho * ll / 3.0) * rr;
    y[3][2] = 2.0 * ll * (ll - 1.0) * cmu / rr;
    y[4][2] = 2.0 * c->zeta * (ll - 1.0) * cmu / rr;
    y[5][2] = ((double)(2 * c->ll + 1) * c->omega2 - 8.0 * pib * ll * (ll - 1.0) * rrho / 3.0);
    y[5][2] = 0.25 * y[5][2] / pib;
}

/* 32-bit wrap of the reference's default-integer products */
static int imul32(int a, int b) { return (int)((unsigned)a * (unsigned)b); }

/* module_int.f90:1275-1341 sph_solid_start_ng; y[row-1][col-1] */
static void sph_solid_start_ng(yo_ctx *c, int is, double rr, yo_cd y[4][2])
{
    const yo_model *m = c->M;
    double rrho = SPL(rho, rr, is), rmu = SPL(mu, rr, is), rqmu = SPL(qmu, rr, is);
    double rkappa = SPL(kappa, rr, is), rqkappa = SPL(qkappa, rr, is);
    yo_cd cmu = rmu * (1.0 + rqmu * c->lno);
    yo_cd ckappa = rkappa * (1.0 + rqkappa * c->lno);
    yo_cd calpha = (ckappa + 1.3333333333 * cmu) / rrho;
    yo_cd cbeta = cmu / rrho;
    int l = c->ll, lp1 = c->llp1;
    double ll = (double)l;
    yo_cd arg = c->omega * rr / csqrt(calpha);
    yo_cd jl1 = 1.0, jl2 = sbessj2(lp1, arg);
    y[0][0] = ll * jl1 - arg * jl2;
    y[1][0] = c->zeta * jl1;
    y[2][0] = -(rrho * calpha * arg * arg * jl1) +
              2.0 * cmu * ((double)imul32(l, l - 1) * jl1 + 2.0 * arg * jl2);
    y[2][0] = y[2][0] / rr;
    y[3][0] = 2.0 * c->zeta * cmu * ((double)(l - 1) * jl1 - arg * jl2);
    y[3][0] = y[3][0] / rr;
    arg = c->omega * rr / csqrt(cbeta);
    jl1 = 1.0;
    jl2 = sbessj2(lp1, arg);
    y[0][1] = -((double)imul32(l, lp1) * jl1);
    y[1][1] = -(c->zeta * (double)lp1 * jl1) + arg * jl2;
    y[2][1] = -2.0 * cmu * ((double)imul32(l, imul32(l, l) - 1) * jl1 -
                            (double)imul32(l, lp1) * arg * jl2);
    y[2][1] = y[2][1] / rr;
    y[3][1] = c->zeta * cmu * (arg * arg * jl1 - 2.0 * (double)(imul32(l, l) - 1) * jl1 -
                               2.0 * arg * jl2);
    y[3][1] = y[3][1] / rr;
}

/* module_int.f90:1346-1405 sph_fluid_start; y[row-1][col-1] */
static void sph_fluid_start(yo_ctx *c, int is, double rr, yo_cd y[4][2])
{
    const yo_model *m = c->M;
    double pib = c->N->pibigg;
    double rrho = SPL(rho, rr, is), rkappa = SPL(kappa, rr, is);
    double rqkappa = SPL(qkappa, rr, is);
    yo_cd ckappa = rkappa * (1.0 + rqkappa * c->lno);
    yo_cd calpha = ckappa / rrho;
    double gamg = 4.0 * pib * rrho / 3.0;
    yo_cd gamma = (c->omega2 + 4.0 * gamg - c->zeta2 * gamg * gamg * c->omegai2) / calpha;
    yo_cd gamma2 = gamma;
    gamma = csqrt(gamma);
    yo_cd zt = -c->omega2 / gamg;
    yo_cd xi = zt - (double)c->llp1;
    yo_cd args = gamma2 * rr * rr;
    yo_cd ratio = bfs_dum(c->ll, args);
    double ll = (double)c->ll;
    y[0][0] = ll * xi - zt * gamma * rr * ratio;
    y[1][0] = -(4.0 * pib * rrho * rr * zt);
    y[2][0] = -(rrho * calpha * zt * rr * gamma2);
    y[3][0] = -(rrho * (c->zeta2 + (double)c->llp1 * zt));
    y[0][1] = ll;
    y[1][1] = (c->omega2 - 4.0 * pib * rrho * ll / 3.0) * rr;
    y[2][1] = 0.0;
    y[3][1] = ((double)(2 * c->ll + 1) * c->omega2 - 8.0 * pib * ll * (ll - 1.0) * rrho / 3.0);
    y[3][1] = 0.25 * y[3][1] / pib;
}

/* module_int.f90:1407-1447 sph_fluid_start_ng (2 components) */
static void sph_fluid_start_ng(yo_ctx *c, int is, double rr, yo_cd *y)
{
    const yo_model *m = c->M;
    double rrho = SPL(rho, rr, is), rkappa = SPL(kappa, rr, is);
    double rqkappa = SPL(qkappa, rr, is);
    yo_cd ckappa = rkappa * (1.0 + rqkappa * c->lno);
    yo_cd calpha = ckappa / rrho;
    yo_cd arg = c->omega * rr / csqrt(calpha);
    yo_cd ratio = sbessj2(c->llp1, arg);
    y[0] = (double)c->ll - arg * ratio;
    y[1] = -(rrho * calpha * arg * arg);
    y[1] = y[1] / rr;
}

/* module_int.f90:1537-1560 det3, det2 */
static yo_cd det2(yo_cd a1, yo_cd a2, yo_cd b1, yo_cd b2) { return a1 * b2 - a2 * b1; }

static yo_cd det3(const yo_cd y[6][3], int i, int j, int k)
{
    /* rows i,j,k (1-based) of the three solution columns */
    yo_cd y1[3] = {y[i - 1][0], y[j - 1][0], y[k - 1][0]};
    yo_cd y2[3] = {y[i - 1][1], y[j - 1][1], y[k - 1][1]};
    yo_cd y3[3] = {y[i - 1][2], y[j - 1][2], y[k - 1][2]};
    return y1[0] * det2(y2[1], y2[2], y3[1], y3[2]) -
           y2[0] * det2(y1[1], y1[2], y3[1], y3[2]) +
           y3[0] * det2(y1[1], y1[2], y2[1], y2[2]);
}

/* module_int.f90:1451-1485 sph_minor_solid_start */
static void sph_minor_solid_start(yo_ctx *c, int is, double rr, yo_cd *m)
{
    yo_cd y[6][3];
    sph_solid_start(c, is, rr, y);
    static const int idx[14][3] = {{1, 2, 3}, {1, 2, 4}, {1, 2, 5}, {1, 2, 6},
                                   {1, 3, 4}, {1, 3, 5}, {1, 4, 5}, {1, 4, 6},
                                   {1, 5, 6}, {2, 3, 4}, {2, 4, 5}, {2, 4, 6},
                                   {3, 4, 5}, {4, 5, 6}};
    for (int q = 0; q < 14; q++) m[q] = det3(y, idx[q][0], idx[q][1], idx[q][2]);
}

static void minors2(const yo_cd y[4][2], yo_cd *m)
{
    /* module_int.f90:1499-1503 / :1527-1531 */
    m[0] = det2(y[0][0], y[1][0], y[0][1], y[1][1]);
    m[1] = det2(y[0][0], y[2][0], y[0][1], y[2][1]);
    m[2] = det2(y[0][0], y[3][0], y[0][1], y[3][1]);
    m[3] = det2(y[1][0], y[2][0], y[1][1], y[2][1]);
    m[4] = det2(y[2][0], y[3][0], y[2][1], y[3][1]);
}

static void sph_minor_solid_start_ng(yo_ctx *c, int is, double rr, yo_cd *m)
{
    yo_cd y[4][2];
    sph_solid_start_ng(c, is, rr, y);
    minors2(y, m);
}

static void sph_minor_fluid_start(yo_ctx *c, int is, double rr, yo_cd *m)
{
    yo_cd y[4][2];
    sph_fluid_start(c, is, rr, y);
    minors2(y, m);
}

/* module_int.f90:1563-1615 b_solid_start, b_solid_start_ngcow */
static void b_solid_start(const yo_cd *m, const yo_cd *s, yo_cd *b)
{
#define M(k) m[(k) - 1]
#define S(k) s[(k) - 1]
    b[0] = M(14) * S(3) - M(7) * S(4) - M(11) * S(5) - M(13) * S(6);
    b[1] = -M(14) * S(2) - M(8) * S(4) - M(12) * S(5) + M(11) * S(6);
    b[2] = M(7) * S(2) + M(8) * S(3) + M(2) * S(5) + M(5) * S(6);
    b[3] = M(11) * S(2) + M(12) * S(3) - M(2) * S(4) + M(10) * S(6);
    b[4] = M(13) * S(2) - M(11) * S(3) - M(5) * S(4) - M(10) * S(5);
    b[5] = M(14) * S(1) - M(9) * S(4) + M(8) * S(5) - M(7) * S(6);
    b[6] = -M(7) * S(1) + M(9) * S(3) + M(3) * S(5) + M(6) * S(6);
    b[7] = -M(11) * S(1) - M(8) * S(3) - M(3) * S(4) - M(5) * S(6);
    b[8] = -M(13) * S(1) + M(7) * S(3) - M(6) * S(4) + M(5) * S(5);
    b[9] = -M(8) * S(1) - M(9) * S(2) + M(4) * S(5) - M(3) * S(6);
    b[10] = -M(12) * S(1) + M(8) * S(2) - M(4) * S(4) + M(2) * S(6);
    b[11] = M(2) * S(1) + M(3) * S(2) + M(4) * S(3) - M(1) * S(6);
    b[12] = M(5) * S(1) + M(6) * S(2) - M(3) * S(3) + M(1) * S(5);
    b[13] = M(10) * S(1) - M(5) * S(2) + M(2) * S(3) - M(1) * S(4);
}

static void b_solid_start_ngcow(const yo_cd *m, const yo_cd *s, yo_cd *b)
{
    b[0] = -M(5) * S(2) - M(2) * S(3) - M(4) * S(4);
    b[1] = M(5) * S(1) - M(3) * S(3) + M(2) * S(4);
    b[2] = M(2) * S(1) + M(3) * S(2) - M(1) * S(4);
    b[3] = M(4) * S(1) - M(2) * S(2) + M(1) * S(3);
}

/* module_int.f90:1620-1700 solid<->fluid minor transforms */
static void s2f(const yo_cd *m1, yo_cd *m2)
{
    m2[0] = -m1[5]; m2[1] = -m1[6]; m2[2] = m1[8]; m2[3] = -m1[12]; m2[4] = m1[13];
}
static void s2f_ngcow(const yo_cd *m1, yo_cd *m2) { m2[0] = -m1[2]; m2[1] = -m1[4]; }
static void f2s(const yo_cd *m1, yo_cd *m2)
{
    for (int k = 0; k < 14; k++) m2[k] = 0.0;
    m2[0] = m1[0]; m2[1] = m1[1]; m2[3] = m1[2]; m2[9] = -m1[3]; m2[11] = -m1[4];
}
static void f2s_ngcow(const yo_cd *m1, yo_cd *m2)
{
    for (int k = 0; k < 5; k++) m2[k] = 0.0;
    m2[0] = m1[0];
    m2[3] = -m1[1];
}

/* module_int.f90:1705-1745 secular determinants */
static yo_cd delta_solid(const yo_cd *m1, const yo_cd *m2)
{
#define A(k) m1[(k) - 1]
#define B(k) m2[(k) - 1]
    return -A(14) * B(1) + 2.0 * A(7) * B(2) + 2.0 * A(11) * B(3) + A(13) * B(4) +
           2.0 * A(8) * B(5) + A(12) * B(6) - 2.0 * A(2) * B(7) - 2.0 * A(5) * B(8) -
           A(10) * B(9) + A(9) * B(10) - 2.0 * A(3) * B(11) - A(6) * B(12) -
           A(4) * B(13) + A(1) * B(14);
}
static yo_cd delta_solid_ngcow(const yo_cd *m1, const yo_cd *m2)
{
    return A(5) * B(1) + 2.0 * A(2) * B(2) + A(4) * B(3) + A(3) * B(4) + A(1) * B(5);
}
#undef A
#undef B

/* module_int.f90:1785-1837 sph_ysol, sph_ysol_ngcow */
static void sph_ysol(const yo_cd *m, const yo_cd *b, yo_cd *y)
{
#define BB(k) b[(k) - 1]
    y[0] = M(3) * BB(3) + M(1) * BB(6) + M(2) * BB(7) + 2.0 * M(3) * BB(8) + M(4) * BB(9) +
           M(5) * BB(10) + M(6) * BB(11) + M(7) * BB(12) + M(8) * BB(13) + M(9) * BB(14);
    y[1] = -M(1) * BB(2) - M(2) * (2.0 * BB(3) + BB(8)) - M(3) * BB(4) - M(4) * BB(5) -
           M(5) * BB(11) - M(8) * BB(14) + M(10) * BB(10) + M(11) * BB(12) + M(12) * BB(13);
    y[2] = M(1) * BB(1) - M(2) * BB(9) + M(3) * BB(5) + M(5) * (BB(8) - BB(3)) -
           M(6) * BB(4) + M(7) * BB(14) - M(10) * BB(7) - M(11) * BB(13) + M(13) * BB(12);
    y[3] = M(2) * BB(1) + M(5) * BB(2) - M(7) * BB(4) - M(8) * BB(5) + M(10) * BB(6) -
           M(11) * (BB(3) + 2.0 * BB(8)) - M(12) * BB(9) - M(13) * BB(11) + M(14) * BB(14);
    y[4] = M(3) * BB(1) - M(5) * BB(6) + M(6) * BB(2) + M(7) * (2.0 * BB(3) + BB(8)) +
           M(8) * BB(9) - M(9) * BB(5) + M(11) * BB(7) + M(13) * BB(10) - M(14) * BB(13);
    y[5] = M(2) * BB(6) - M(3) * BB(2) + M(4) * BB(1) + M(7) * BB(11) +
           M(8) * (BB(3) - BB(8)) + M(9) * BB(4) - M(11) * BB(10) + M(12) * BB(7) +
           M(14) * BB(12);
}
static void sph_ysol_ngcow(const yo_cd *m, const yo_cd *b, yo_cd *y)
{
    y[0] = M(1) * BB(2) + M(2) * BB(3) + M(3) * BB(4);
    y[1] = -M(1) * BB(1) + M(4) * BB(3) - M(2) * BB(4);
    y[2] = -M(2) * BB(1) - M(4) * BB(2) + M(5) * BB(4);
    y[3] = -M(3) * BB(1) + M(2) * BB(2) - M(5) * BB(3);
#undef BB
#undef M
#undef S
}

/* ------------------------------------------------------------------------ */
/* module_solver.f90:25-142 tor_solver; yout is yout[row][col], 2 x 2       */
/* ------------------------------------------------------------------------ */
void yo_tor_solver(yo_ctx *c, int l, yo_cd w, double rr, double rs, int ir, int is,
                   yo_cd yout[2][2])
{
    const yo_model *m = c->M;
    yo_set_l(c, l);
    yo_set_omega(c, w);
    tor_steps(c);
    int scale1 = 0, scale2 = 0, scale3 = 0, i1;
    double rt;
    yo_cd y1[2], y2[2], y3[2], delta, b;
    c->cnt->nsolve_tor++;
    /* ss = identity 2x2 (yspec.f90:230-232) */
    if (rr >= rs) {
        i1 = yo_tor_start_level(m, c->ll, creal(c->omega), is);
        if (i1 == is && i1 > m->noc + 1) i1 = i1 - 1;
        rt = m->r[i1];
        if (i1 == m->noc + 1) { y1[0] = 1.0; y1[1] = 0.0; }
        else tor_ystart(c, i1, rt, y1);
        yo_yint(c, i1, is, rt, rs, y1, 2, tor_derivs, &scale1);
        y3[0] = y1[0]; y3[1] = y1[1];
        if (rr != rs) yo_yint(c, is, ir, rs, rr, y3, 2, tor_derivs, &scale3);
        y2[0] = 1.0; y2[1] = 0.0;
        if (rr != m->r[m->nsl]) yo_yint(c, m->nsl - 1, ir, m->r[m->nsl], rr, y2, 2, tor_derivs, &scale2);
        delta = y2[1] * y3[0] - y2[0] * y3[1];
        delta = 1.0 / delta;
        for (int i = 0; i < 2; i++) {
            yo_cd s1 = (i == 0) ? 1.0 : 0.0, s2 = (i == 1) ? 1.0 : 0.0;
            b = y1[1] * s1 - y1[0] * s2;
            yout[0][i] = -(delta * y2[0] * b);
            yout[1][i] = -(delta * y2[1] * b);
        }
    } else {
        i1 = yo_tor_start_level(m, c->ll, creal(c->omega), ir);
        if (i1 == ir && i1 > m->noc + 1) i1 = i1 - 1;
        rt = m->r[i1];
        if (i1 == m->noc + 1) { y1[0] = 1.0; y1[1] = 0.0; }
        else tor_ystart(c, i1, rt, y1);
        yo_yint(c, i1, ir, rt, rr, y1, 2, tor_derivs, &scale1);
        y2[0] = 1.0; y2[1] = 0.0;
        if (rs != m->r[m->nsl]) yo_yint(c, m->nsl - 1, is, m->r[m->nsl], rs, y2, 2, tor_derivs, &scale2);
        y3[0] = y2[0]; y3[1] = y2[1];
        if (rr != rs) yo_yint(c, is, ir, rs, rr, y3, 2, tor_derivs, &scale3);
        delta = y3[1] * y1[0] - y3[0] * y1[1];
        delta = 1.0 / delta;
        for (int i = 0; i < 2; i++) {
            yo_cd s1 = (i == 0) ? 1.0 : 0.0, s2 = (i == 1) ? 1.0 : 0.0;
            b = y2[1] * s1 - y2[0] * s2;
            yout[0][i] = -(delta * y1[0] * b);
            yout[1][i] = -(delta * y1[1] * b);
        }
    }
    if (scale3 != 0) {
        double f = pow(YO_HUGE, (double)scale3);
        for (int i = 0; i < 2; i++) { yout[0][i] *= f; yout[1][i] *= f; }
    }
}

/* module_solver.f90:335-441 rad_solver_ng (uses rad_derivs_ng == rad_amat) */
void yo_rad_solver_ng(yo_ctx *c, yo_cd w, double rr, double rs, int ir, int is,
                      yo_cd yout[2][2])
{
    const yo_model *m = c->M;
    yo_set_l(c, 0);
    yo_set_omega(c, w);
    alpha_steps(c);
    int scale1 = 0, scale2 = 0, scale3 = 0;
    yo_cd y1[2], y2[2], y3[2], delta, b;
    double rt = fmin(0.1 * c->dr, 0.1 * m->r[2]);
    c->cnt->nsolve_rad++;
    if (rr >= rs) {
        rad_ystart(c, 1, rt, y1, 0);
        yo_yint(c, 1, is, rt, rs, y1, 2, rad_derivs, &scale1);
        y2[0] = 1.0; y2[1] = 0.0;
        if (rr != m->r[m->nknot]) yo_yint(c, m->nknot - 1, ir, m->r[m->nknot], rr, y2, 2, rad_derivs, &scale2);
        y3[0] = y2[0]; y3[1] = y2[1];
        if (rs != rr) yo_yint(c, ir, is, rr, rs, y3, 2, rad_derivs, &scale3);
        delta = y3[1] * y1[0] - y3[0] * y1[1];
        delta = cabs(delta) < 1.0e-100 ? 0.0 : 1.0 / delta;
        for (int i = 0; i < 2; i++) {
            yo_cd s1 = (i == 0) ? 1.0 : 0.0, s2 = (i == 1) ? 1.0 : 0.0;
            b = y1[1] * s1 - y1[0] * s2;
            yout[0][i] = -(delta * y2[0] * b);
            yout[1][i] = -(delta * y2[1] * b);
        }
        if (scale3 != 0) {
            double f = pow(YO_HUGE, (double)scale3);
            for (int i = 0; i < 2; i++) { yout[0][i] *= f; yout[1][i] *= f; }
        }
    } else {
        rad_ystart(c, 1, rt, y1, 0);
        yo_yint(c, 1, ir, rt, rr, y1, 2, rad_derivs, &scale1);
        y2[0] = 1.0; y2[1] = 0.0;
        if (rs != m->r[m->nsl]) yo_yint(c, m->nsl - 1, is, m->r[m->nsl], rs, y2, 2, rad_derivs, &scale2);
        y3[0] = y2[0]; y3[1] = y2[1];
        if (rr != rs) yo_yint(c, is, ir, rs, rr, y3, 2, rad_derivs, &scale3);
        delta = y3[1] * y1[0] - y3[0] * y1[1];
        delta = cabs(delta) < 1.0e-100 ? 0.0 : 1.0 / delta;
        for (int i = 0; i < 2; i++) {
            yo_cd s1 = (i == 0) ? 1.0 : 0.0, s2 = (i == 1) ? 1.0 : 0.0;
            b = y2[1] * s1 - y2[0] * s2;
            yout[0][i] = -(delta * y1[0] * b);
            yout[1][i] = -(delta * y1[1] * b);
        }
        /* module_solver.f90:433-437: only positive scale3 is undone */
        for (int k = 0; k < scale3; k++)
            for (int i = 0; i < 2; i++) { yout[0][i] *= YO_HUGE; yout[1][i] *= YO_HUGE; }
    }
}

/* module_model.f90:578-787 grid_count / make_grid (1-based outputs) */
static int grid_count(const yo_model *m, double drr, double rs, double rr)
{
    int ngrid = 0;
    for (int i = 1; i <= m->nknot - 1; i++) {
        double r1 = m->r[i], r2 = m->r[i + 1];
        if (r1 == r2) continue;
        int ls = (rs > r1 && rs <= r2), lr = (rr > r1 && rr <= r2);
        if (ls && lr) {
            if (rs < rr) {
                ngrid += (int)floor((rs - r1) / drr) + 2;
                ngrid += (int)floor((rr - rs) / drr) + 2 - 1;
                ngrid += (int)floor((r2 - rr) / drr) + 2 - 1;
            } else if (rr < rs) {
                ngrid += (int)floor((rr - r1) / drr) + 2;
                ngrid += (int)floor((rs - rr) / drr) + 2 - 1;
                ngrid += (int)floor((r2 - rs) / drr) + 2 - 1;
            } else {
                ngrid += (int)floor((rs - r1) / drr) + 2;
                ngrid += (int)floor((r2 - rs) / drr) + 2 - 1;
            }
        } else if (ls) {
            ngrid += (int)floor((rs - r1) / drr) + 2;
            ngrid += (int)floor((r2 - rs) / drr) + 2 - 1;
        } else if (lr) {
            ngrid += (int)floor((rr - r1) / drr) + 2;
            ngrid += (int)floor((r2 - rr) / drr) + 2 - 1;
        } else {
            ngrid += (int)floor((r2 - r1) / drr) + 2;
        }
    }
    return ngrid;
}

static void grid_seg(double a, double b, double drr, int i, int first, int *k,
                     int *igrid, double *rgrid)
{
    int nr = (int)floor((b - a) / drr) + 2;
    double drt = (b - a) / (double)(nr - 1);
    for (int j = first; j <= nr; j++) {
        (*k)++;
        rgrid[*k] = a + (double)(j - 1) * drt;
        igrid[*k] = i;
    }
}

static void make_grid(const yo_model *m, double drr, double rs, double rr, int *is,
                      int *ir, int *igrid, double *rgrid)
{
    int k = 0;
    for (int i = 1; i <= m->nknot - 1; i++) {
        double r1 = m->r[i], r2 = m->r[i + 1];
        if (r1 == r2) continue;
        int ls = (rs > r1 && rs <= r2), lr = (rr > r1 && rr <= r2);
        if (ls && lr) {
            if (rs < rr) {
                grid_seg(r1, rs, drr, i, 1, &k, igrid, rgrid); *is = k;
                grid_seg(rs, rr, drr, i, 2, &k, igrid, rgrid); *ir = k;
                grid_seg(rr, r2, drr, i, 2, &k, igrid, rgrid);
            } else if (rr < rs) {
                grid_seg(r1, rr, drr, i, 1, &k, igrid, rgrid); *ir = k;
                grid_seg(rr, rs, drr, i, 2, &k, igrid, rgrid); *is = k;
                grid_seg(rs, r2, drr, i, 2, &k, igrid, rgrid);
            } else {
                grid_seg(r1, rs, drr, i, 1, &k, igrid, rgrid); *is = k; *ir = k;
                grid_seg(rs, r2, drr, i, 2, &k, igrid, rgrid);
            }
        } else if (ls) {
            grid_seg(r1, rs, drr, i, 1, &k, igrid, rgrid); *is = k;
            grid_seg(rs, r2, drr, i, 2, &k, igrid, rgrid);
        } else if (lr) {
            grid_seg(r1, rr, drr, i, 1, &k, igrid, rgrid); *ir = k;
            grid_seg(rr, r2, drr, i, 2, &k, igrid, rgrid);
        } else {
            grid_seg(r1, r2, drr, i, 1, &k, igrid, rgrid);
        }
    }
}

/* module_solver.f90:446-561 rad_solver_wg.  The main program does not use */
/* the potential pout (yspec.f90:277-281); with pout1 non-NULL, pout(1, i)  */
/* of the two unit sources i is formed as at :534-554.                      */
void yo_rad_solver_wg(yo_ctx *c, yo_cd w, double rr, double rs, int ir, int is,
                      yo_cd yout[2][2], yo_cd *pout1)
{
    const yo_model *m = c->M;
    (void)ir; (void)is;
    yo_set_l(c, 0);
    yo_set_omega(c, w);
    alpha_steps(c);
    c->cnt->nsolve_rad++;
    int ngrid = grid_count(m, c->dr, rs, rr);
    int *igrid = (int *)calloc((size_t)ngrid + 2, sizeof(int));
    double *rgrid = (double *)calloc((size_t)ngrid + 2, sizeof(double));
    yo_cd *y1s = (yo_cd *)calloc(2 * ((size_t)ngrid + 2), sizeof(yo_cd));
    yo_cd *y2s = (yo_cd *)calloc(2 * ((size_t)ngrid + 2), sizeof(yo_cd));
    int iss = 0, irr = 0;
    make_grid(m, c->dr, rs, rr, &iss, &irr, igrid, rgrid);
    yo_cd y1[2], y2[2], delta, b;
    double rt = fmin(0.1 * c->dr, 0.1 * rgrid[2]);
    rad_ystart(c, 1, rt, y1, 1);
    yo_yint(c, 1, igrid[2], rt, rgrid[2], y1, 2, rad_derivs, NULL);
    y1s[2 * 2] = y1[0]; y1s[2 * 2 + 1] = y1[1];
    for (int ig = 2; ig <= iss - 1; ig++) {
        yo_yint(c, igrid[ig], igrid[ig + 1], rgrid[ig], rgrid[ig + 1], y1, 2, rad_derivs, NULL);
        y1s[2 * (ig + 1)] = y1[0]; y1s[2 * (ig + 1) + 1] = y1[1];
    }
    y2[0] = 1.0; y2[1] = 0.0;
    y2s[2 * ngrid] = y2[0]; y2s[2 * ngrid + 1] = y2[1];
    for (int ig = ngrid; ig >= iss + 1; ig--) {
        yo_yint(c, igrid[ig], igrid[ig - 1], rgrid[ig], rgrid[ig - 1], y2, 2, rad_derivs, NULL);
        y2s[2 * (ig - 1)] = y2[0]; y2s[2 * (ig - 1) + 1] = y2[1];
    }
    delta = y2[1] * y1[0] - y2[0] * y1[1];
    delta = 1.0 / delta;
    for (int i = 0; i < 2; i++) {
        yo_cd s1 = (i == 0) ? 1.0 : 0.0, s2 = (i == 1) ? 1.0 : 0.0;
        if (irr <= iss) {
            b = y2[1] * s1 - y2[0] * s2;
            yout[0][i] = -(delta * y1s[2 * irr] * b);
            yout[1][i] = -(delta * y1s[2 * irr + 1] * b);
        } else {
            b = y1[1] * s1 - y1[0] * s2;
            yout[0][i] = -(delta * y2s[2 * irr] * b);
            yout[1][i] = -(delta * y2s[2 * irr + 1] * b);
        }
        if (pout1) {
            /* ys(1, ig): below the source from y1s, above from y2s (:517-527); */
            /* phi = rr * trapezoid sum of -4 pibigg ys(1) / r, zero at ig = 1  */
            yo_cd bb = y2[1] * s1 - y2[0] * s2, ba = y1[1] * s1 - y1[0] * s2;
            yo_cd sum = 0.0, ctmp1, ctmp2;
            for (int ig = 1; ig <= irr - 1; ig++) {
                yo_cd ys1 = ig <= iss ? -(delta * y1s[2 * ig] * bb) : -(delta * y2s[2 * ig] * ba);
                yo_cd ys2 = ig + 1 <= iss ? -(delta * y1s[2 * (ig + 1)] * bb)
                                          : -(delta * y2s[2 * (ig + 1)] * ba);
                ctmp1 = ig == 1 ? 0.0 : -4.0 * c->N->pibigg * ys1 / rgrid[ig];
                ctmp2 = -4.0 * c->N->pibigg * ys2 / rgrid[ig + 1];
                sum = sum + 0.5 * (ctmp1 + ctmp2) * (rgrid[ig + 1] - rgrid[ig]);
            }
            pout1[i] = rr * sum;
        }
    }
    free(igrid); free(rgrid); free(y1s); free(y2s);
}

/* ------------------------------------------------------------------------ */
/* Spheroidal BVP drivers, module_solver.f90:640-1740.                      */
/* ------------------------------------------------------------------------ */

/* Full gravity: sph_solver (:640-823, fic = 0) and sph_solver_fic          */
/* (:1203-1382, fic = 1).  yout[row][col], 6 x 4.  Unit jumps in components  */
/* 1, 2, 4, 5 (yspec.f90:234-238).                                          */
void yo_sph_solver_g(yo_ctx *c, int l, yo_cd w, double rr, double rs, int ir, int is,
                     int fic, yo_cd yout[6][4])
{
    const yo_model *m = c->M;
    yo_set_l(c, l);
    yo_set_omega(c, w);
    alpha_steps(c);
    c->cnt->nsolve_sph++;
    int scale1 = 0, scale2 = 0, scale3 = 0, scale4, i1;
    double rt;
    yo_cd ms1[14], ms2[14], ms3[14], mf1[5], mf2[5], b[14], delta, ys[6];
    static const int jump[4] = {0, 1, 3, 4};
    int up = (rr >= rs);
    int it = up ? is : ir;
    double rtop = up ? rs : rr;
    i1 = yo_sph_start_level(m, c->N, c->ll, creal(c->omega), it);
    rt = m->r[i1];
    if (i1 == 1 && (up || fic)) rt = fmin(0.1 * c->dr, 0.1 * m->r[2]);
    if (i1 >= it) { i1 = it - 1; rt = m->r[i1]; }
    /* A fluid inner core starts from the fluid minor on both branches.   */
    /* The receiver-below-source branch of sph_solver_fic                  */
    /* (module_solver.f90:1323-1332) starts a solid minor there instead:   */
    /* with mu = 0 the shear wavenumber is infinite, bfs's continued       */
    /* fraction never converges and the reference does not return.  The   */
    /* receiver-above branch's fluid start (:1252-1256) is taken for both. */
    int ic_fluid_start = fic;
    if (i1 <= m->nic) {
        if (ic_fluid_start) {
            sph_minor_fluid_start(c, i1, rt, mf1);
            yo_yint(c, i1, m->noc, rt, m->r[m->noc], mf1, 5, minors_fluid_g, &scale1);
        } else {
            sph_minor_solid_start(c, i1, rt, ms1);
            yo_yint(c, i1, m->nic, rt, m->r[m->nic], ms1, 14, minors_solid_g, &scale1);
            s2f(ms1, mf1);
            yo_yint(c, m->nic + 1, m->noc, m->r[m->nic], m->r[m->noc], mf1, 5, minors_fluid_g, &scale1);
        }
        f2s(mf1, ms1);
        yo_yint(c, m->noc + 1, it, m->r[m->noc + 1], rtop, ms1, 14, minors_solid_g, &scale1);
    } else if (i1 > m->nic && i1 <= m->noc) {
        sph_minor_fluid_start(c, i1, rt, mf1);
        yo_yint(c, i1, m->noc, rt, m->r[m->noc], mf1, 5, minors_fluid_g, &scale1);
        f2s(mf1, ms1);
        yo_yint(c, m->noc + 1, it, m->r[m->noc + 1], rtop, ms1, 14, minors_solid_g, &scale1);
    } else if (i1 > m->noc && i1 <= m->nsl) {
        sph_minor_solid_start(c, i1, rt, ms1);
        yo_yint(c, i1, it, rt, rtop, ms1, 14, minors_solid_g, &scale1);
    }
    memcpy(ms3, ms1, sizeof ms1);
    if (up) {
        if (rr > rs) yo_yint(c, is, ir, rs, rr, ms3, 14, minors_solid_g, &scale3);
    } else {
        if (rs > rr) yo_yint(c, ir, is, rr, rs, ms3, 14, minors_solid_g, &scale3);
    }
    int ibot = up ? ir : is;
    double rbot = up ? rr : rs;
    if (m->ocean) {
        for (int k = 0; k < 5; k++) mf2[k] = 0.0;
        mf2[0] = 1.0;
        yo_yint(c, m->nknot - 1, m->nsl + 1, m->r[m->nknot], m->r[m->nsl + 1], mf2, 5,
                minors_fluid_g, &scale2);
        f2s(mf2, ms2);
        yo_yint(c, m->nsl, ibot, m->r[m->nsl], rbot, ms2, 14, minors_solid_g, &scale2);
    } else {
        for (int k = 0; k < 14; k++) ms2[k] = 0.0;
        ms2[0] = 1.0;
        yo_yint(c, up ? m->nknot - 1 : m->nknot, ibot, m->r[m->nknot], rbot, ms2, 14,
                minors_solid_g, &scale2);
    }
    delta = delta_solid(ms3, ms2);
    for (int i = 0; i < 4; i++) {
        yo_cd s[6] = {0, 0, 0, 0, 0, 0};
        s[jump[i]] = 1.0;
        scale4 = 0;
        if (up) {
            b_solid_start(ms1, s, b);
            yo_yint(c, is, ir, rs, rr, b, 14, bvec_solid_g, &scale4);
            sph_ysol(ms2, b, ys);
            for (int k = 0; k < 6; k++) ys[k] = -ys[k] / delta;
        } else {
            b_solid_start(ms2, s, b);
            for (int k = 0; k < 14; k++) b[k] = -b[k] / delta;
            yo_yint(c, is, ir, rs, rr, b, 14, bvec_solid_g, &scale4);
            sph_ysol(ms1, b, ys);
        }
        double f = pow(YO_HUGE, (double)(scale3 - scale4));
        for (int k = 0; k < 6; k++) yout[k][i] = ys[k] * f;
    }
}

/* No gravity / Cowling: sph_solver_ng (:827-1010), sph_solver_cow          */
/* (:1014-1195), sph_solver_ng_fic (:1386-1562), sph_solver_cow_fic          */
/* (:1568-1740).  yout[row][col], 4 x 4, ss = identity (yspec.f90:240-243).  */
void yo_sph_solver_ngcow(yo_ctx *c, int l, yo_cd w, double rr, double rs, int ir,
                         int is, int fic, int cow, yo_cd yout[4][4])
{
    const yo_model *m = c->M;
    yo_derivs dsol = cow ? minors_solid_cow : minors_solid_ng;
    yo_derivs dflu = cow ? minors_fluid_cow : minors_fluid_ng;
    yo_derivs dbv = cow ? bvec_solid_cow : bvec_solid_ng;
    yo_set_l(c, l);
    yo_set_omega(c, w);
    alpha_steps(c);
    c->cnt->nsolve_sph++;
    int scale1 = 0, scale2 = 0, scale3 = 0, scale4, i1;
    double rt;
    yo_cd ms1[5], ms2[5], ms3[5], mf1[2], mf2[2], b[4], delta, ys[4];
    int up = (rr >= rs);
    int it = up ? is : ir;
    double rtop = up ? rs : rr;
    i1 = yo_sph_start_level(m, c->N, c->ll, creal(c->omega), it);
    rt = m->r[i1];
    if (i1 == 1 && (up || fic)) rt = fmin(0.1 * c->dr, 0.1 * m->r[2]);
    if (i1 >= it) { i1 = it - 1; rt = m->r[i1]; }
    if (i1 <= m->nic) {
        if (fic) {
            sph_fluid_start_ng(c, i1, rt, mf1);
            yo_yint(c, i1, m->noc, rt, m->r[m->noc], mf1, 2, dflu, &scale1);
        } else {
            sph_minor_solid_start_ng(c, i1, rt, ms1);
            yo_yint(c, i1, m->nic, rt, m->r[m->nic], ms1, 5, dsol, &scale1);
            s2f_ngcow(ms1, mf1);
            yo_yint(c, m->nic + 1, m->noc, m->r[m->nic], m->r[m->noc], mf1, 2, dflu, &scale1);
        }
        f2s_ngcow(mf1, ms1);
        yo_yint(c, m->noc + 1, it, m->r[m->noc + 1], rtop, ms1, 5, dsol, &scale1);
    } else if (i1 > m->nic && i1 <= m->noc) {
        sph_fluid_start_ng(c, i1, rt, mf1);
        yo_yint(c, i1, m->noc, rt, m->r[m->noc], mf1, 2, dflu, &scale1);
        f2s_ngcow(mf1, ms1);
        yo_yint(c, m->noc + 1, it, m->r[m->noc + 1], rtop, ms1, 5, dsol, &scale1);
    } else if (i1 > m->noc && i1 <= m->nsl) {
        sph_minor_solid_start_ng(c, i1, rt, ms1);
        yo_yint(c, i1, it, rt, rtop, ms1, 5, dsol, &scale1);
    }
    memcpy(ms3, ms1, sizeof ms1);
    if (up) {
        if (rr > rs) yo_yint(c, is, ir, rs, rr, ms3, 5, dsol, &scale3);
    } else {
        if (rs > rr) yo_yint(c, ir, is, rr, rs, ms3, 5, dsol, &scale3);
    }
    int ibot = up ? ir : is;
    double rbot = up ? rr : rs;
    if (m->ocean) {
        mf2[0] = 1.0; mf2[1] = 0.0;
        yo_yint(c, m->nknot - 1, m->nsl + 1, m->r[m->nknot], m->r[m->nsl + 1], mf2, 2, dflu, &scale2);
        f2s_ngcow(mf2, ms2);
        yo_yint(c, m->nsl, ibot, m->r[m->nsl], rbot, ms2, 5, dsol, &scale2);
    } else {
        for (int k = 0; k < 5; k++) ms2[k] = 0.0;
        ms2[0] = 1.0;
        yo_yint(c, m->nknot, ibot, m->r[m->nknot], rbot, ms2, 5, dsol, &scale2);
    }
    delta = delta_solid_ngcow(ms3, ms2);
    for (int i = 0; i < 4; i++) {
        yo_cd s[4] = {0, 0, 0, 0};
        s[i] = 1.0;
        scale4 = 0;
        if (up) {
            b_solid_start_ngcow(ms1, s, b);
            yo_yint(c, is, ir, rs, rr, b, 4, dbv, &scale4);
            sph_ysol_ngcow(ms2, b, ys);
            for (int k = 0; k < 4; k++) ys[k] = ys[k] / delta;
        } else {
            b_solid_start_ngcow(ms2, s, b);
            for (int k = 0; k < 4; k++) b[k] = -b[k] / delta;
            yo_yint(c, is, ir, rs, rr, b, 4, dbv, &scale4);
            sph_ysol_ngcow(ms1, b, ys);
        }
        double f = pow(YO_HUGE, (double)(scale3 - scale4));
        for (int k = 0; k < 4; k++) yout[k][i] = ys[k] * f;
    }
}

/* ------------------------------------------------------------------------ */
/* Source vectors, module_solver.f90:145-215, :566-627, :1747-1847          */
/* ------------------------------------------------------------------------ */
void yo_source_vector_tor(yo_ctx *c, int l, yo_cd w, int is, double rs, const double *mm,
                          yo_cd svt[5][2])
{
    const yo_model *m = c->M;
    yo_set_l(c, l);
    yo_set_omega(c, w);
    double rlcon = SPL(lcon, rs, is), rqmu = SPL(qmu, rs, is);
    yo_cd qll = 1.0 + rqmu * c->lno;
    yo_cd clcon = rlcon * qll;
    for (int i = 0; i < 5; i++) svt[i][0] = svt[i][1] = 0.0;
    if (l >= 1) {
        svt[1][0] = 0.5 * rs * (-mm[2] + I_ * mm[1]) / clcon;
        svt[3][0] = 0.5 * rs * (mm[2] + I_ * mm[1]) / clcon;
    }
    if (l >= 2) {
        svt[0][1] = 0.25 * c->szeta2m2 * (-(I_ * mm[3]) + I_ * mm[5] + 2.0 * mm[4]);
        svt[4][1] = 0.25 * c->szeta2m2 * (I_ * mm[3] - I_ * mm[5] + 2.0 * mm[4]);
    }
    yo_cd den = I_ * w * rs * rs;
    for (int i = 0; i < 5; i++) {
        svt[i][0] = c->nu * svt[i][0] / den;
        svt[i][1] = c->nu * svt[i][1] / den;
    }
}

void yo_source_vector_rad(yo_ctx *c, yo_cd w, int is, double rs, const double *mm,
                          yo_cd s0[2])
{
    const yo_model *m = c->M;
    yo_set_l(c, 0);
    yo_set_omega(c, w);
    double rccon = SPL(ccon, rs, is), rfcon = SPL(fcon, rs, is);
    double rxa2 = SPL(xa2, rs, is), rxlam = SPL(xlam, rs, is);
    yo_cd qaa = 1.0 + rxa2 * c->lno, qff = 1.0 + rxlam * c->lno;
    yo_cd cccon = rccon * qaa;
    cccon = 1.0 / cccon;
    yo_cd cfcon = rfcon * qff;
    s0[0] = rs * mm[0] * cccon;
    s0[1] = -mm[3] - mm[5] + 2.0 * mm[0] * cfcon * cccon;
    yo_cd den = I_ * w * rs * rs;
    s0[0] = c->nu * s0[0] / den;
    s0[1] = c->nu * s0[1] / den;
}

/* qaa, qff, qll are declared real(dp) in the reference
 * (module_solver.f90:1771-1772), so only the real part of 1 + q*lno is kept. */
void yo_source_vector_sph(yo_ctx *c, int l, yo_cd w, int is, double rs, const double *mm,
                          yo_cd svs[5][6])
{
    const yo_model *m = c->M;
    yo_set_l(c, l);
    yo_set_omega(c, w);
    double rlcon = SPL(lcon, rs, is), rccon = SPL(ccon, rs, is);
    double rfcon = SPL(fcon, rs, is), rqmu = SPL(qmu, rs, is);
    double rxlam = SPL(xlam, rs, is), rxa2 = SPL(xa2, rs, is);
    double qaa = creal(1.0 + rxa2 * c->lno);
    double qff = creal(1.0 + rxlam * c->lno);
    double qll = creal(1.0 + rqmu * c->lno);
    yo_cd cccon = rccon * qaa;
    cccon = 1.0 / cccon;
    yo_cd cfcon = rfcon * qff;
    yo_cd clcon = rlcon * qll;
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 6; j++) svs[i][j] = 0.0;
    double z = c->zeta;
    if (l != 1) svs[0][4] = 0.25 * c->szeta2m2 * (-mm[3] + mm[5] - 2.0 * I_ * mm[4]);
    svs[1][1] = 0.5 * rs * (mm[1] + I_ * mm[2]) / clcon;
    svs[2][0] = rs * mm[0] * cccon;
    svs[2][3] = -mm[3] - mm[5] + 2.0 * mm[0] * cfcon * cccon;
    svs[2][4] = 0.5 * z * (mm[3] + mm[5]) - z * mm[0] * cfcon * cccon;
    svs[3][1] = 0.5 * rs * (-mm[1] + I_ * mm[2]) / clcon;
    if (l != 1) svs[4][4] = 0.25 * c->szeta2m2 * (-mm[3] + mm[5] + 2.0 * I_ * mm[4]);
    yo_cd den = I_ * w * rs * rs;
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 6; j++) svs[i][j] = c->nu * svs[i][j] / den;
}
