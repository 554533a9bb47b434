/*
 * streams_b200_host.h -- host-side case set-up and run driver of the B200 backend.
 *
 * In the Fortran drop-in the reference's own equation object (singleideal.F90) parses
 * singleideal.ini, builds the grid and the initial field, and then drives the backend through
 * streams_b200.h.  These entry points provide the same set-up and the run() loop in C++ so the
 * backend can be used stand-alone (tests, benchmarks, and callers without the Fortran code).
 * Replaces: equation_singleideal_object%initialize (code/src/singleideal/singleideal.F90:284-864)
 * and equation_singleideal_cpu_object%run (code/src/singleideal/singleideal_cpu.F90:1519-1693).
 */
#ifndef STREAMS_B200_HOST_H
#define STREAMS_B200_HOST_H

#include "streams_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct streams_b200_case streams_b200_case;

/*
 * Build a case.  dir holds singleideal.ini (read unless ini_text is non-empty) and any grid or
 * restart files (x.dat, y.dat, z.dat, yn.dat, rst.bin, field_info0.dat).  An optional
 * [synthetic] section selects a seeded synthetic channel field:
 *   kind = channel_poiseuille, amp, seed, y_stretch, reynolds_bulk.
 */
int streams_b200_case_load(const char* dir, const char* ini_text, streams_b200_case** out);
int streams_b200_case_free(streams_b200_case* c);
const char* streams_b200_case_error(void);

/* Parameters and grid for streams_b200_create; grid pointers stay valid while the case lives. */
int streams_b200_case_params(const streams_b200_case* c, int precision, streams_b200_params* out);
int streams_b200_case_grid(const streams_b200_case* c, streams_b200_grid* out);
/* Initial field w(1-ng:nx+ng,1-ng:ny+ng,1-ng:nz+ng,5) of the case. */
const double* streams_b200_case_field(const streams_b200_case* c);
/* out[0..11] = u0, rho0, l0, mu0, num_iter, print_control, iter_dt_recompute, icyc0, time0, cfl,
 *              volchan, t_bulk_target */
int streams_b200_case_info(const streams_b200_case* c, double out[12]);
/* Write x.dat, y.dat, z.dat, yn.dat, rst.bin and field_info0.dat of the case into dir. */
int streams_b200_case_write_restart(const streams_b200_case* c, const char* dir);
/*
 * Restart files of a running solve: w (the ghosted field of streams_b200_copy_to_field) at step
 * icyc and time, written as x/y/z/yn.dat, rst.bin, field_info0.dat (the keys read_field_info of
 * code/src/singleideal/singleideal.F90:2546-2590 reads) and singleideal.ini = the case's input
 * with restart_type = 1, so that the case resumes from dir here or in the reference.
 */
int streams_b200_case_write_state(const streams_b200_case* c, const double* w, int icyc, double time,
                                  const char* dir);

/*
 * The run() loop of the solver on the device: initial ghost fill and sensor, then nsteps time
 * steps (num_iter when nsteps < 0); every print_control steps compute_residual and a progress
 * row.  Rows (14 columns of progress.out) are written to progress_path when it is non-NULL and
 * the last row is returned in last_row[14] when non-NULL.  The final field is written to
 * w_out when non-NULL.  Returns STREAMS_B200_ENAN when the residual becomes NaN.
 */
int streams_b200_run_case(const streams_b200_case* c, int nsteps, int precision, const char* progress_path,
                          double* last_row, double* w_out);

#ifdef __cplusplus
}
#endif

#endif /* STREAMS_B200_HOST_H */
