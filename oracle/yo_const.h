/*
 * yo_const.h -- constants of the oracle restatement.  TEST INFRASTRUCTURE.
 *
 * nrtype.f90:18-27 declares pi_d, pio2_d and twopi_d as real(dp) but
 * initialises them from _sp literals, so they hold the single-precision
 * rounding of pi.  fourpi_d and bigg are truncated decimal literals.
 */
#ifndef YO_CONST_H
#define YO_CONST_H

#define YO_PI_D ((double)3.14159265358979323846f)
#define YO_TWOPI_D ((double)6.28318530717958647692f)
#define YO_FOURPI_D 12.56637061
#define YO_BIGG 6.6723e-11
#define YO_BIG 1.0e+40                 /* module_model.f90:20 */
#define YO_TINY 1.0e-20                /* module_int.f90:80 */
#define YO_HUGE (1.0 / 1.0e-20)        /* module_int.f90:81 */
#define YO_NW 4                        /* module_int.f90:74 */
#define YO_TOL_START 11.0              /* module_start.f90:6 */

/* Nonzero status codes replacing the reference's `stop` statements. */
#define YO_ERR_PARAM_FILE 1     /* yspec.f90:81,85 */
#define YO_ERR_MODEL_FILE 2     /* yspec.f90:94 */
#define YO_ERR_PARAM_READ 3
#define YO_ERR_MODEL_READ 4
#define YO_ERR_NYQUIST 5        /* module_fourier.f90:377 (silent stop) */
#define YO_ERR_FEW_FREQ 6       /* yspec.f90:201,205 */
#define YO_ERR_SRC_MODEL 7      /* yspec.f90:211 */
#define YO_ERR_SRC_OCEAN 8      /* yspec.f90:212 */
#define YO_ERR_REC_MODEL 9      /* yspec.f90:214 */
#define YO_ERR_REC_OCEAN 10     /* yspec.f90:215 */
#define YO_ERR_IO 11
#define YO_ERR_ARG 20           /* oracle-only: an argument out of range */

#endif
