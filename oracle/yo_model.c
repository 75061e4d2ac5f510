/*
 * yo_model.c -- oracle restatement of the reference's model, spline,
 * geometry and frequency-grid routines.  TEST INFRASTRUCTURE ONLY (see yo.h).
 *
 * Citations are to da380/YSpec src/ (Fortran sources).
 */
#include "yo.h"
#include "yo_const.h"

#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* module_model.f90:474-492  set_parameters                                 */
/* ------------------------------------------------------------------------ */
void yo_set_parameters(yo_norms *n)
{
    n->r_norm = 6.371e+6;                 /* module_model.f90:18 */
    n->rho_norm = 5.515e+3;               /* module_model.f90:19 */
    n->vel_norm = n->r_norm * sqrt(YO_PI_D * YO_BIGG * n->rho_norm);
    n->acl_norm = YO_PI_D * YO_BIGG * n->rho_norm * n->r_norm;
    n->fre_norm = n->vel_norm / n->r_norm;
    n->t_norm = 1.0 / n->fre_norm;
    n->con_norm = n->vel_norm * n->vel_norm * n->rho_norm;
    n->grav_norm = YO_PI_D * YO_BIGG;
    {
        double r2 = n->r_norm * n->r_norm;
        double r5 = r2 * r2 * n->r_norm;
        n->moment_norm = r5 * (n->rho_norm * n->rho_norm) * n->grav_norm;
    }
    n->pot_norm = n->acl_norm * n->r_norm;
    n->pibigg = YO_PI_D * YO_BIGG / n->grav_norm;
}

/* ------------------------------------------------------------------------ */
/* Fortran list-directed record reader (enough of it for yspec's inputs).   */
/* A read statement consumes records until it has its values; the rest of   */
/* the last record is discarded (module_util.f90:301-355 read_*).           */
/* ------------------------------------------------------------------------ */
typedef struct {
    FILE *f;
    char line[4096];
} rec_reader;

static int rr_next(rec_reader *rr)
{
    if (!fgets(rr->line, sizeof rr->line, rr->f)) return 0;
    return 1;
}

static int rr_skip(rec_reader *rr, int n)
{
    for (int i = 0; i < n; i++)
        if (!rr_next(rr)) return 0;
    return 1;
}

/* Collect k value tokens, starting with a fresh record. */
static int rr_tokens(rec_reader *rr, int k, char tok[][256])
{
    int got = 0;
    while (got < k) {
        if (!rr_next(rr)) return got;
        char *s = rr->line;
        while (*s && got < k) {
            while (*s && (isspace((unsigned char)*s) || *s == ',')) s++;
            if (!*s) break;
            if (*s == '/') return got;      /* slash ends a list-directed read */
            char *t = tok[got];
            int len = 0;
            if (*s == '\'' || *s == '"') {
                char q = *s++;
                while (*s && *s != q && len < 255) t[len++] = *s++;
                if (*s == q) s++;
            } else {
                while (*s && !isspace((unsigned char)*s) && *s != ',' &&
                       *s != '/' && len < 255)
                    t[len++] = *s++;
            }
            t[len] = 0;
            got++;
        }
    }
    return got;
}

static double fortran_real(const char *s)
{
    char buf[256];
    size_t n = strlen(s);
    if (n > 255) n = 255;
    for (size_t i = 0; i < n; i++)
        buf[i] = (s[i] == 'd' || s[i] == 'D') ? 'e' : s[i];
    buf[n] = 0;
    return strtod(buf, NULL);
}

static int read_string(rec_reader *rr, char *out, int skip)
{
    char tok[1][256];
    if (!rr_skip(rr, skip)) return 0;
    if (rr_tokens(rr, 1, tok) != 1) return 0;
    strncpy(out, tok[0], 255);
    out[255] = 0;
    return 1;
}

static int read_int(rec_reader *rr, int *v, int skip)
{
    char tok[1][256];
    if (!rr_skip(rr, skip)) return 0;
    if (rr_tokens(rr, 1, tok) != 1) return 0;
    *v = (int)strtol(tok[0], NULL, 10);
    return 1;
}

static int read_float(rec_reader *rr, double *v, int skip)
{
    char tok[1][256];
    if (!rr_skip(rr, skip)) return 0;
    if (rr_tokens(rr, 1, tok) != 1) return 0;
    *v = fortran_real(tok[0]);
    return 1;
}

/* yspec.f90:79-139 parameter file layout. */
int yo_read_params(const char *path, yo_params *p)
{
    memset(p, 0, sizeof *p);
    rec_reader rr;
    rr.f = fopen(path, "r");
    if (!rr.f) return YO_ERR_PARAM_FILE;
    int ok = 1;
    ok &= read_string(&rr, p->pref_out, 4);
    ok &= read_string(&rr, p->model_file, 2);
    ok &= read_int(&rr, &p->ats, 2);
    ok &= read_int(&rr, &p->grav, 2);
    ok &= read_int(&rr, &p->out, 2);
    ok &= read_int(&rr, &p->cor, 2);
    ok &= read_int(&rr, &p->lmin, 2);
    ok &= read_int(&rr, &p->lmax, 2);
    ok &= read_float(&rr, &p->f1, 2);
    ok &= read_float(&rr, &p->f2, 2);
    ok &= read_float(&rr, &p->tout, 2);
    ok &= read_float(&rr, &p->dt, 2);
    ok &= read_float(&rr, &p->f11, 2);
    ok &= read_float(&rr, &p->f12, 2);
    ok &= read_float(&rr, &p->f21, 2);
    ok &= read_float(&rr, &p->f22, 2);
    ok &= read_float(&rr, &p->depth_s, 2);
    ok &= read_float(&rr, &p->lat_s, 2);
    ok &= read_float(&rr, &p->lon_s, 2);
    for (int i = 0; i < 6 && ok; i++) ok &= read_float(&rr, &p->mm[i], 2);
    ok &= read_float(&rr, &p->depth_r, 2);
    ok &= read_int(&rr, &p->nr, 2);
    if (ok && p->nr > 0) {
        ok &= rr_skip(&rr, 2);
        p->lat_r = (double *)calloc((size_t)p->nr, sizeof(double));
        p->lon_r = (double *)calloc((size_t)p->nr, sizeof(double));
        for (int i = 0; i < p->nr && ok; i++) {
            char tok[2][256];
            if (rr_tokens(&rr, 2, tok) != 2) { ok = 0; break; }
            p->lat_r[i] = fortran_real(tok[0]);
            p->lon_r[i] = fortran_real(tok[1]);
        }
    }
    fclose(rr.f);
    return ok ? 0 : YO_ERR_PARAM_READ;
}

void yo_free_params(yo_params *p)
{
    free(p->lat_r);
    free(p->lon_r);
    p->lat_r = p->lon_r = NULL;
}

/* ------------------------------------------------------------------------ */
/* module_spline.f90:40-73 spline_r and :426-449 tridag_ser_r.               */
/* x, y, y2 are 0-based views of n points.                                  */
/* ------------------------------------------------------------------------ */
static void tridag(const double *a, const double *b, const double *c,
                   const double *r, double *u, int n)
{
    /* a has n-1 entries (a(2:n) of the caller), c has n-1 (c(1:n-1)). */
    double *gam = (double *)malloc((size_t)(n + 1) * sizeof(double));
    double bet = b[0];
    u[0] = r[0] / bet;
    for (int j = 1; j < n; j++) {
        gam[j] = c[j - 1] / bet;
        bet = b[j] - a[j - 1] * gam[j];
        u[j] = (r[j] - a[j - 1] * u[j - 1]) / bet;
    }
    for (int j = n - 2; j >= 0; j--) u[j] = u[j] - gam[j + 1] * u[j + 1];
    free(gam);
}

void yo_spline(const double *x, const double *y, int n, double yp1,
               double ypn, double *y2)
{
    double *a = (double *)calloc((size_t)n + 1, sizeof(double));
    double *b = (double *)calloc((size_t)n + 1, sizeof(double));
    double *c = (double *)calloc((size_t)n + 1, sizeof(double));
    double *r = (double *)calloc((size_t)n + 1, sizeof(double));
    double *rtmp = (double *)calloc((size_t)n + 1, sizeof(double));
    /* 1-based indices mapped to [i-1] */
    for (int i = 1; i <= n - 1; i++) c[i - 1] = x[i] - x[i - 1];
    for (int i = 1; i <= n - 1; i++)
        r[i - 1] = 6.0 * ((y[i] - y[i - 1]) / c[i - 1]);
    /* r(2:n-1) = r(2:n-1) - r(1:n-2): whole-array semantics */
    for (int i = 0; i < n; i++) rtmp[i] = r[i];
    for (int i = 2; i <= n - 1; i++) r[i - 1] = rtmp[i - 1] - rtmp[i - 2];
    for (int i = 2; i <= n - 1; i++) a[i - 1] = c[i - 2];
    for (int i = 2; i <= n - 1; i++) b[i - 1] = 2.0 * (c[i - 1] + a[i - 1]);
    b[0] = 1.0;
    b[n - 1] = 1.0;
    if (yp1 > 0.99e30) {
        r[0] = 0.0;
        c[0] = 0.0;
    } else {
        r[0] = (3.0 / (x[1] - x[0])) * ((y[1] - y[0]) / (x[1] - x[0]) - yp1);
        c[0] = 0.5;
    }
    if (ypn > 0.99e30) {
        r[n - 1] = 0.0;
        a[n - 1] = 0.0;
    } else {
        r[n - 1] = (-3.0 / (x[n - 1] - x[n - 2])) *
                   ((y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]) - ypn);
        a[n - 1] = 0.5;
    }
    tridag(a + 1, b, c, r, y2, n);
    free(a); free(b); free(c); free(r); free(rtmp);
}

/* module_spline.f90:262-283 splint_dis_r; arrays 1-based, klo 1-based. */
double yo_splint_dis(const double *xa, const double *ya, const double *y2a,
                     double x, int klo)
{
    int khi = klo + 1;
    double h = xa[khi] - xa[klo];
    if (h == 0.0) return ya[klo];
    double a = (xa[khi] - x) / h;
    double b = (x - xa[klo]) / h;
    return a * ya[klo] + b * ya[khi] +
           ((a * a * a - a) * y2a[klo] + (b * b * b - b) * y2a[khi]) *
               (h * h) / 6.0;
}

/* ------------------------------------------------------------------------ */
/* module_model.f90:175-383 read_model                                      */
/* ------------------------------------------------------------------------ */
static double *alloc1(int n) { return (double *)calloc((size_t)n + 2, sizeof(double)); }

static void layer_spline(const yo_model *m, const double *y, double *y2)
{
    for (int i = 1; i <= m->nlayer; i++) {
        int lo = m->layer_lo[i], hi = m->layer_hi[i];
        yo_spline(m->r + lo, y + lo, hi - lo + 1, YO_BIG, YO_BIG, y2 + lo);
    }
}

/* module_model.f90:507-535 gauslv (5-point Gauss-Legendre from minos) */
static void gauslv(const yo_model *m, const double *intg, const double *qint,
                   double r1, double r2, int iq, double *fint)
{
    static const double w[2] = {.478628670499366, .236926885056189};
    static const double x[2] = {.538469310105683, .906179845938664};
    double y1 = 0.5 * (r2 + r1);
    double y2 = 0.5 * (r2 - r1);
    double vals = yo_splint_dis(m->r, intg, qint, y1, iq);
    double sum = .568888888888889 * vals;
    for (int i = 0; i < 2; i++) {
        double t1 = x[i] * y2;
        vals = yo_splint_dis(m->r, intg, qint, y1 + t1, iq);
        double vals1 = yo_splint_dis(m->r, intg, qint, y1 - t1, iq);
        sum = sum + w[i] * (vals + vals1);
    }
    *fint = *fint + y2 * sum;
}

int yo_read_model(const char *path, const yo_norms *nm, yo_model *m)
{
    memset(m, 0, sizeof *m);
    rec_reader rr;
    rr.f = fopen(path, "r");
    if (!rr.f) return YO_ERR_MODEL_FILE;
    char tok[9][256];
    if (rr_tokens(&rr, 1, tok) != 1) goto bad;                 /* title */
    if (rr_tokens(&rr, 2, tok) != 2) goto bad;
    int ians = (int)strtol(tok[0], NULL, 10);
    double tref = fortran_real(tok[1]);
    m->tref = (YO_TWOPI_D / tref) / nm->fre_norm;              /* :196-197 */
    m->ifanis = (ians == 1);
    if (rr_tokens(&rr, 3, tok) != 3) goto bad;
    m->nknot = (int)strtol(tok[0], NULL, 10);
    m->nic = (int)strtol(tok[1], NULL, 10);
    m->noc = (int)strtol(tok[2], NULL, 10);
    int n = m->nknot;
    if (n < 2) goto bad;
    double **arrs[] = {&m->r, &m->rho, &m->rho_cs, &m->acon, &m->acon_cs,
                       &m->ccon, &m->ccon_cs, &m->fcon, &m->fcon_cs,
                       &m->lcon, &m->lcon_cs, &m->ncon, &m->ncon_cs,
                       &m->kappa, &m->kappa_cs, &m->mu, &m->mu_cs,
                       &m->lambda, &m->qkappa, &m->qkappa_cs, &m->qmu,
                       &m->qmu_cs, &m->grav, &m->grav_cs, &m->beta,
                       &m->alpha, &m->rat, &m->rat_cs, &m->xlam,
                       &m->xlam_cs, &m->xa2, &m->xa2_cs};
    for (size_t k = 0; k < sizeof arrs / sizeof arrs[0]; k++) *arrs[k] = alloc1(n);

    for (int i = 1; i <= n; i++) {                             /* :209-222 */
        int want = m->ifanis ? 9 : 6;
        if (rr_tokens(&rr, want, tok) != want) goto bad;
        m->r[i] = fortran_real(tok[0]);
        m->rho[i] = fortran_real(tok[1]);
        m->ccon[i] = fortran_real(tok[2]);
        m->lcon[i] = fortran_real(tok[3]);
        m->qkappa[i] = fortran_real(tok[4]);
        m->qmu[i] = fortran_real(tok[5]);
        if (m->ifanis) {
            m->acon[i] = fortran_real(tok[6]);
            m->ncon[i] = fortran_real(tok[7]);
            m->fcon[i] = fortran_real(tok[8]);
        } else {
            m->acon[i] = m->ccon[i];
            m->ncon[i] = m->lcon[i];
            m->fcon[i] = 1.0;
        }
    }
    fclose(rr.f);
    rr.f = NULL;

    /* ocean / fluid inner core detection, :227-248 */
    m->ocean = (m->lcon[n] == 0.0);
    if (m->ocean) {
        m->nsl = 0;
        for (int i = n - 1; i >= 1; i--)
            if (m->lcon[i] > 0.0) { m->nsl = i; break; }
    } else {
        m->nsl = n;
    }
    m->fic = (m->lcon[1] == 0.0);

    /* normalise and convert velocities to moduli, :253-263 */
    for (int i = 1; i <= n; i++) {
        m->r[i] = m->r[i] / nm->r_norm;
        m->rho[i] = m->rho[i] / nm->rho_norm;
        m->acon[i] = m->acon[i] / nm->vel_norm;
        m->ccon[i] = m->ccon[i] / nm->vel_norm;
        m->lcon[i] = m->lcon[i] / nm->vel_norm;
        m->ncon[i] = m->ncon[i] / nm->vel_norm;
        m->acon[i] = m->rho[i] * (m->acon[i] * m->acon[i]);
        m->ccon[i] = m->rho[i] * (m->ccon[i] * m->ccon[i]);
        m->lcon[i] = m->rho[i] * (m->lcon[i] * m->lcon[i]);
        m->ncon[i] = m->rho[i] * (m->ncon[i] * m->ncon[i]);
        m->fcon[i] = (m->acon[i] - 2.0 * m->lcon[i]) * m->fcon[i];
        /* :269-277 */
        m->kappa[i] = m->ccon[i] + 4.0 * m->acon[i] - 4.0 * m->ncon[i] +
                      4.0 * m->fcon[i];
        m->kappa[i] = m->kappa[i] / 9.0;
        m->mu[i] = m->ccon[i] + m->acon[i] + 6.0 * m->lcon[i] +
                   5.0 * m->ncon[i] - 2.0 * m->fcon[i];
        m->mu[i] = m->mu[i] / 15.0;
        m->lambda[i] = m->kappa[i] - 2.0 * m->mu[i] / 3.0;
        m->beta[i] = sqrt(m->mu[i] / m->rho[i]);
        m->alpha[i] = sqrt((m->kappa[i] + 1.3333333333 * m->mu[i]) / m->rho[i]);
        /* :282-290 */
        if (m->qkappa[i] > 0.0) m->qkappa[i] = 1.0 / m->qkappa[i];
        if (m->qmu[i] > 0.0) m->qmu[i] = 1.0 / m->qmu[i];
        m->rat[i] = 4.0 * m->mu[i] / (3.0 * (m->lambda[i] + 2.0 * m->mu[i]));
        m->xlam[i] = (1.0 - m->rat[i]) * m->qkappa[i] - 0.5 * m->rat[i] * m->qmu[i];
        m->xlam[i] = m->xlam[i] / (1.0 - 1.5 * m->rat[i]);
        m->xa2[i] = (1.0 - m->rat[i]) * m->qkappa[i] + m->rat[i] * m->qmu[i];
    }

    /* layers split at repeated radii, :294-308 */
    m->nlayer = 1;
    for (int i = 2; i <= n; i++)
        if (m->r[i] == m->r[i - 1]) m->nlayer++;
    m->layer_lo = (int *)calloc((size_t)m->nlayer + 2, sizeof(int));
    m->layer_hi = (int *)calloc((size_t)m->nlayer + 2, sizeof(int));
    m->layer_lo[1] = 1;
    m->layer_hi[m->nlayer] = n;
    {
        int j = 0;
        for (int i = 2; i <= n; i++) {
            if (m->r[i] == m->r[i - 1]) {
                j++;
                m->layer_hi[j] = i - 1;
                m->layer_lo[j + 1] = i;
            }
        }
    }

    /* 13 splines per layer, :312-352 */
    layer_spline(m, m->rho, m->rho_cs);
    layer_spline(m, m->acon, m->acon_cs);
    layer_spline(m, m->ccon, m->ccon_cs);
    layer_spline(m, m->fcon, m->fcon_cs);
    layer_spline(m, m->lcon, m->lcon_cs);
    layer_spline(m, m->ncon, m->ncon_cs);
    layer_spline(m, m->kappa, m->kappa_cs);
    layer_spline(m, m->mu, m->mu_cs);
    layer_spline(m, m->qkappa, m->qkappa_cs);
    layer_spline(m, m->qmu, m->qmu_cs);
    layer_spline(m, m->rat, m->rat_cs);
    layer_spline(m, m->xlam, m->xlam_cs);
    layer_spline(m, m->xa2, m->xa2_cs);

    /* gravity by Gauss-Legendre on a spline of r^2 rho, :356-371 */
    {
        double *intg = alloc1(n), *qint = alloc1(n);
        for (int i = 1; i <= n; i++) intg[i] = (m->r[i] * m->r[i]) * m->rho[i];
        layer_spline(m, intg, qint);
        double fint = 0.0;
        m->grav[1] = 0.0;
        for (int i = 1; i <= n - 1; i++) {
            gauslv(m, intg, qint, m->r[i], m->r[i + 1], i, &fint);
            m->grav[i + 1] = fint;
        }
        for (int i = 1; i <= n; i++)
            if (m->r[i] > 0.0) m->grav[i] = (4.0 * m->grav[i]) / (m->r[i] * m->r[i]);
        free(intg);
        free(qint);
    }
    layer_spline(m, m->grav, m->grav_cs);                      /* :374-378 */
    return 0;
bad:
    if (rr.f) fclose(rr.f);
    return YO_ERR_MODEL_READ;
}

void yo_free_model(yo_model *m)
{
    double **arrs[] = {&m->r, &m->rho, &m->rho_cs, &m->acon, &m->acon_cs,
                       &m->ccon, &m->ccon_cs, &m->fcon, &m->fcon_cs,
                       &m->lcon, &m->lcon_cs, &m->ncon, &m->ncon_cs,
                       &m->kappa, &m->kappa_cs, &m->mu, &m->mu_cs,
                       &m->lambda, &m->qkappa, &m->qkappa_cs, &m->qmu,
                       &m->qmu_cs, &m->grav, &m->grav_cs, &m->beta,
                       &m->alpha, &m->rat, &m->rat_cs, &m->xlam,
                       &m->xlam_cs, &m->xa2, &m->xa2_cs};
    for (size_t k = 0; k < sizeof arrs / sizeof arrs[0]; k++) {
        free(*arrs[k]);
        *arrs[k] = NULL;
    }
    free(m->layer_lo);
    free(m->layer_hi);
    m->layer_lo = m->layer_hi = NULL;
}

/* module_model.f90:537-576 find_radius_index with up = -1 */
int yo_find_radius_index(const yo_model *m, double rr)
{
    if (rr < 0.0 || rr > 1.0) return 0;
    for (int i = 1; i <= m->nknot - 1; i++) {
        if (rr == m->r[i] && rr == m->r[i + 1]) return i;
        if (rr > m->r[i] && rr <= m->r[i + 1]) return i;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* module_function.f90:317-390 delaz                                        */
/* ------------------------------------------------------------------------ */
static double fsign(double a, double b) { return b >= 0.0 ? fabs(a) : -fabs(a); }

void yo_delaz(double eplati, double eplong, double stlati, double stlong,
              double *delta, double *azep, double *azst)
{
    const double geoco = 0.993277;
    const double hpi = 0.5 * YO_PI_D;
    const double rad = 0.0174533;
    double eplat = eplati, stlat = stlati;
    if (eplat == -90.0) eplat = -89.98;
    if (stlat == -90.0) stlat = -89.98;
    if (eplat == stlat && eplong == stlong) {
        *delta = 0.0;
        *azep = 0.0;
        *azst = 0.0;
        return;
    }
    double el = atan(geoco * tan(eplat * rad));
    el = hpi - el;
    double stl = atan(geoco * tan(stlat * rad));
    stl = hpi - stl;
    double elon = eplong * rad, slon = stlong * rad;
    double as = cos(stl), bs = sin(stl), cs = cos(slon), ds = sin(slon);
    double a = cos(el), b = sin(el), c = cos(elon), d = sin(elon);
    double cdel = a * as + b * bs * (c * cs + d * ds);
    if (fabs(cdel) > 1.0) cdel = fsign(1.0, cdel);
    double delt = acos(cdel);
    *delta = delt;
    double sdel = sin(delt);
    double caze = (as - a * cdel) / (sdel * b);
    if (fabs(caze) > 1.0) caze = fsign(1.0, caze);
    double aze = acos(caze);
    double cazs = 0.0;
    if (bs > 0.0) cazs = (a - as * cdel) / (bs * sdel);
    if (bs == 0.0) cazs = fsign(1.0, cazs);
    if (fabs(cazs) > 1.0) cazs = fsign(1.0, cazs);
    double azs = acos(cazs);
    double dif = ds * c - cs * d;
    if (dif < 0.0) aze = YO_TWOPI_D - aze;
    *azep = aze;
    if (dif > 0.0) azs = YO_TWOPI_D - azs;
    *azst = azs;
}

/* ------------------------------------------------------------------------ */
/* module_function.f90:6-132 legendre.  x, xp, xcosec have m+1 entries      */
/* (0-based here: x[0] = P_l0).  real(...) conversions are single precision */
/* in the reference; sqrt(real(...)) is an FP32 square root.                */
/* ------------------------------------------------------------------------ */
void yo_legendre(double theta, int l, int m, double *x, double *xp,
                 double *xcosec)
{
    int lp1 = l + 1, mp1 = m + 1;
    double th = theta, ct = cos(th), st = sin(th);
    double fct = sqrt((double)(float)(2 * l + 1) / YO_FOURPI_D);
    double sfl3 = (double)sqrtf((float)(l * (l + 1)));
    double compar = (double)(float)(2 * l + 1) / YO_FOURPI_D;
    double dsfl3 = sfl3;
    double small = 1.0e-16 * compar;
    double sum;
    for (int i = 0; i < mp1; i++) x[i] = xp[i] = xcosec[i] = 0.0;

    if (l <= 1 || fabs(theta) <= 1.0e-5) {
        x[0] = fct;
        if (l == 0) return;
        x[0] = ct * fct;
        x[1] = -st * fct / dsfl3;
        xp[0] = -st * fct;
        xp[1] = -0.5 * ct * fct * dsfl3;
        if (fabs(theta) < 1.0e-5)
            xcosec[1] = xp[1];
        else
            xcosec[1] = x[1] / st;
        return;
    }
    double x1 = 1.0, x2 = ct, x3;
    for (int i = 2; i <= l; i++) {
        x3 = ((double)(float)(2 * i - 1) * ct * x2 - (double)(float)(i - 1) * x1) /
             (double)(float)i;
        x1 = x2;
        x2 = x3;
    }
    double cot = ct / st;
    double cosec = 1.0 / st;
    x3 = x2 * fct;
    x2 = (double)(float)l * (x1 - ct * x2) * fct / st;
    x[0] = x3;
    x[1] = x2;
    sum = x3 * x3;
    xp[0] = -x2;
    xp[1] = (double)(float)(l * (l + 1)) * x3 - cot * x2;
    x[1] = -x[1] / sfl3;
    xcosec[1] = x[1] * cosec;
    xp[1] = -xp[1] / sfl3;
    sum = sum + 2.0 * x[1] * x[1];
    if (sum - compar > small) return;
    x1 = x3;
    x2 = -x2 / (double)sqrtf((float)(l * (l + 1)));
    for (int i = 3; i <= mp1; i++) {
        int k = i - 1;
        /* real(l+i-1)*(l-i+2): single-precision product, FP32 sqrt */
        double f1 = (double)sqrtf((float)(l + i - 1) * (float)(l - i + 2));
        double f2 = (double)sqrtf((float)(l + i - 2) * (float)(l - i + 3));
        double xm = (double)k;
        x3 = -(2.0 * cot * (xm - 1.0) * x2 + f2 * x1) / f1;
        sum = sum + 2.0 * x3 * x3;
        if (sum - compar > small && i != lp1) return;
        x[i - 1] = x3;
        xcosec[i - 1] = x[i - 1] * cosec;
        x1 = x2;
        xp[i - 1] = -(f1 * x2 + xm * cot * x3);
        x2 = x3;
    }
}

/* ------------------------------------------------------------------------ */
/* module_fourier.f90:362-397 fcal.  Returns YO_ERR_NYQUIST where the       */
/* reference stops silently.                                                */
/* ------------------------------------------------------------------------ */
int yo_fcal(double *f1, double *f2, double dt, double tout, int mex, int qex,
            double *df, double *ep, int *nt, int *i1, int *i2)
{
    double fn = 0.5 / dt;                      /* 0.5_sp is exact */
    if (fn < *f2) return YO_ERR_NYQUIST;
    *ep = (double)mex / tout;
    *df = *ep / (YO_TWOPI_D * (double)qex);
    *nt = (int)(1.0 / (*df * dt));             /* 1.0_sp exact; truncation */
    float lf = logf((float)*nt) / logf(2.0f) + 1.0f;
    int ne = (int)lf;
    *nt = 1 << ne;
    *df = 1.0 / ((double)*nt * dt);
    *i1 = (int)floor(*f1 / *df);
    if (*i1 < 2) *i1 = 2;
    *f1 = (double)(*i1 - 1) * *df;
    *i2 = (int)floor(*f2 / *df) + 2;
    *f2 = (double)(*i2 - 1) * *df;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* module_function.f90:520-581 bfs (Lentz continued fraction / series)      */
/* ------------------------------------------------------------------------ */
void yo_bfs(int l, yo_cd xsq, double eps, yo_cd *fp)
{
    if (creal(xsq) > 0.0) {
        yo_cd x = csqrt(xsq);
        int lp1 = l + 1;
        yo_cd rx = 2.0 / x;
        yo_cd nu = (double)lp1 - 0.5;
        yo_cd rj = nu * rx;
        rx = -rx;
        yo_cd denom = (nu + 1.0) * rx;
        yo_cd numer = denom + 1.0 / rj;
        rj = rj * numer / denom;
        int nm1 = 1;
        for (;;) {
            nm1 = nm1 + 1;
            rx = -rx;
            yo_cd a3 = (nu + (double)nm1) * rx;
            denom = a3 + 1.0 / denom;
            numer = a3 + 1.0 / numer;
            yo_cd ratio = numer / denom;
            rj = rj * ratio;
            if (fabs(cabs(ratio) - 1.0) <= eps) break;
        }
        *fp = rj * x - (double)lp1;
    } else {
        yo_cd f = 1.0, fpl = (double)(float)l, a = 1.0;
        yo_cd b = (double)(float)(l + l) + 1.0, c = 2.0, d = (double)(float)l + 2.0;
        for (;;) {
            a = -a * xsq / (c * (b + c));
            f = f + a;
            fpl = fpl + a * d;
            if (cabs(a * d) < eps) break;
            c = c + 2.0;
            d = d + 2.0;
        }
        *fp = fpl / f;
    }
}
