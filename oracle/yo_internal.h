/* yo_internal.h -- private declarations of the oracle.  TEST INFRASTRUCTURE. */
#ifndef YO_INTERNAL_H
#define YO_INTERNAL_H

#include "yo.h"

/* Per-solve state that module_int.f90:93-117 keeps in module globals. */
typedef struct {
    const yo_model *M;
    const yo_norms *N;
    int ll, llp1;
    double zeta, zeta2, zeta2m2, szeta2m2, nu, dr, ats;
    yo_cd omega, omega2, omegai, omegai2, lno;
    int il;
    yo_counts *cnt;
} yo_ctx;

typedef void (*yo_derivs)(yo_ctx *c, double r, const yo_cd *y, yo_cd *dydx);

void yo_set_l(yo_ctx *c, int l);
void yo_set_omega(yo_ctx *c, yo_cd w);
void yo_yint(yo_ctx *c, int i1, int i2, double r1, double r2, yo_cd *y, int n,
             yo_derivs derivs, int *scale);
int yo_tor_start_level(const yo_model *m, int l, double w, int it);
int yo_sph_start_level(const yo_model *m, const yo_norms *n, int l, double w, int it);

void yo_tor_solver(yo_ctx *c, int l, yo_cd w, double rr, double rs, int ir, int is,
                   yo_cd yout[2][2]);
void yo_rad_solver_ng(yo_ctx *c, yo_cd w, double rr, double rs, int ir, int is,
                      yo_cd yout[2][2]);
void yo_rad_solver_wg(yo_ctx *c, yo_cd w, double rr, double rs, int ir, int is,
                      yo_cd yout[2][2], yo_cd *pout1);
void yo_sph_solver_g(yo_ctx *c, int l, yo_cd w, double rr, double rs, int ir, int is,
                     int fic, yo_cd yout[6][4]);
void yo_sph_solver_ngcow(yo_ctx *c, int l, yo_cd w, double rr, double rs, int ir,
                         int is, int fic, int cow, yo_cd yout[4][4]);
void yo_source_vector_tor(yo_ctx *c, int l, yo_cd w, int is, double rs,
                          const double *mm, yo_cd svt[5][2]);
void yo_source_vector_rad(yo_ctx *c, yo_cd w, int is, double rs, const double *mm,
                          yo_cd s0[2]);
void yo_source_vector_sph(yo_ctx *c, int l, yo_cd w, int is, double rs,
                          const double *mm, yo_cd svs[5][6]);

#endif
