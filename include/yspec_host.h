/*
 * yspec_host.h -- host side of the `yspec input.in` program above the
 * ysg_* C-ABI.
 *
 * No Fortran compiler exists on the build or GPU images, so the reference's
 * Fortran host (yspec.f90 with module_model, module_spline, module_util and
 * the delaz / fcal helpers) is mirrored here in C++ with the same file
 * formats, argument meaning and stop conditions:
 *   ysh_read_params   yspec.f90:79-139, module_util.f90:301-355
 *   ysh_read_model    module_model.f90:175-383 (+ module_spline.f90:40-73,
 *                     :426-449; gauslv :507-535)
 *   ysh_event_setup   yspec.f90:144-215 (delaz, fcal, find_radius_index)
 *   ysh_write_traces  yspec.f90:488-503, module_util.f90:428-444
 *   ysh_run           the whole program, yspec.f90:74-511
 * Status codes are the YSH_* values below; ysh_status_string() returns the
 * reference's stop message for each.
 */
#ifndef YSPEC_HOST_H
#define YSPEC_HOST_H

#include "yspec_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
    YSH_OK = 0,
    YSH_ERR_PARAM_FILE = 101,   /* "can't find parameter file" (yspec.f90:81) */
    YSH_ERR_PARAM_READ = 102,   /* list-directed read failure */
    YSH_ERR_MODEL_FILE = 103,   /* "problem opening model file" (:94) */
    YSH_ERR_MODEL_READ = 104,
    YSH_ERR_NYQUIST = 105,      /* fcal stops when 1/(2 dt) < fmax (module_fourier.f90:377) */
    YSH_ERR_FEW_FREQ = 106,     /* "too few frequency steps" (:201, :205) */
    YSH_ERR_SRC_MODEL = 107,    /* "source not in model!" (:211) */
    YSH_ERR_SRC_OCEAN = 108,    /* "source in the ocean!" (:212) */
    YSH_ERR_REC_MODEL = 109,    /* "receiver not in model!" (:214) */
    YSH_ERR_REC_OCEAN = 110,    /* "receiver in the ocean!" (:215) */
    YSH_ERR_IO = 111            /* output file could not be written */
};

/* Parameter file contents in the reference's units (yspec.f90:88-137). */
typedef struct {
    char pref_out[256];
    char model_file[256];
    int ats, grav, out, cor, lmin, lmax;
    double f1, f2, tout, dt, f11, f12, f21, f22;
    double depth_s, lat_s, lon_s, mm[6];
    double depth_r;
    int nr;
    double *lat_r, *lon_r;          /* nr each, owned; free with ysh_free_params */
} ysh_params;

typedef struct ysh_model ysh_model;  /* owns the normalised model arrays */

/* Normalisation constants (module_model.f90:474-492). */
typedef struct {
    double r_norm, rho_norm, vel_norm, acl_norm, fre_norm, t_norm;
    double con_norm, grav_norm, moment_norm, pot_norm, pibigg;
} ysh_norms;

/* Event arrays owned by the caller: delta, azst, azep have nr entries. */
typedef struct {
    ysg_event ev;
    ysg_time tm;
    int nt, i1, i2;
    double *delta, *azst, *azep;
} ysh_event;

void ysh_norms_get(ysh_norms *n);
int ysh_read_params(const char *path, ysh_params *p);
void ysh_free_params(ysh_params *p);
int ysh_read_model(const char *path, ysh_model **m);
/* Fill the C-ABI view of the model (pointers stay valid while m lives). */
void ysh_model_view(const ysh_model *m, ysg_model *view);
/* Raw access for tests: number of knots and a named 1-based array. */
int ysh_model_nknot(const ysh_model *m);
const double *ysh_model_array(const ysh_model *m, const char *name);
void ysh_free_model(ysh_model *m);
/* Normalise the inputs, fcal, radius indices, geometry: yspec.f90:144-215.
 * Allocates e->delta/azst/azep (free with ysh_free_event). */
int ysh_event_setup(const ysh_model *m, const ysh_params *p, ysh_event *e);
void ysh_free_event(ysh_event *e);
/* The per-receiver files of yspec.f90:488-503 (pref_out.1 .. pref_out.nr,
 * nout lines of four E15.6 fields), byte-identical to the reference; the
 * receivers' files are formatted and written on several threads. */
int ysh_write_traces(const char *pref_out, const double *out, int nout, int nr);

/* One E15.6 field exactly as the writer forms it (15 characters and a NUL):
 * the text gfortran's E15.6 edit descriptor gives for x. */
void ysh_format_e15_6(double x, char field[16]);
/* The whole program: parameter file -> traces on `device`.  When out is
 * non-NULL it receives a malloc'd (nout, 4, nr) array (free with
 * ysh_free). When write_files is nonzero the per-receiver files are written
 * as the reference writes them. */
int ysh_run(const char *param_file, int device, int write_files, double **out, int *nout,
            int *nr);
/* The potential traces of the event (ysg_event_potential): out, when
 * non-NULL, receives a malloc'd (nout, 2, nr) array (time, potential in SI
 * units of the output type); with write_files, pref_out.pot.1 ..
 * pref_out.pot.nr, nout lines of two E15.6 fields each.  No reference
 * counterpart: the reference does not write potential traces. */
int ysh_run_potential(const char *param_file, int device, int write_files, double **out, int *nout,
                      int *nr);
int ysh_write_potential(const char *pref_out, const double *out, int nout, int nr);
/* Several parameter files in one go: the events that name the same model
 * deck run as one ysg_batch_run (one batched solve launch, one CUDA graph),
 * and each event's files are written under its own output prefix exactly as
 * a single run writes them.  On an error *failed (if non-NULL) is the index
 * of the parameter file concerned. */
int ysh_run_batch(int nfiles, const char *const *param_files, int device, int write_files,
                  int *failed);
void ysh_free(void *ptr);
const char *ysh_status_string(int status);

#ifdef __cplusplus
}
#endif
#endif
