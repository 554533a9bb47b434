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
 * The same with running statistics: stat.bin (and stat3d.bin when w_stat_3d is non-NULL) with
 * w_stat(70, nx, ny), w_stat_3d(14, nx, ny, nz) (statistic index fastest), field_info0.dat with
 * itav and time_from_last_stat, and singleideal.ini with restart_type = 2, so that the
 * averaging continues on resume (read_stats, singleideal.F90:1646-1700).
 */
int streams_b200_case_write_state_stats(const streams_b200_case* c, const double* w, int icyc, double time,
                                        const double* w_stat, const double* w_stat_3d, int itav,
                                        double time_from_last_stat, const char* dir);
/*
 * Statistics settings and restart state of the case: out[0..4] = dtstat (< 0 when [output] has
 * no dtstat), enable_stat_time, enable_stat_3d, itav, time_from_last_stat.
 */
int streams_b200_case_stats_info(const streams_b200_case* c, double out[5]);
/*
 * Averages read on a restart with restart_type = 2: which = 0 w_stat (70*nx*ny doubles),
 * 2 w_stat_3d (14*nx*ny*nz); zeros when the case starts the averages afresh.
 */
int streams_b200_case_stats(const streams_b200_case* c, int which, double* out, long long n);

/*
 * The run() loop of the solver on the device: initial ghost fill and sensor, then nsteps time
 * steps (num_iter when nsteps < 0); every print_control steps compute_residual and a progress
 * row.  Rows (14 columns of progress.out) are written to progress_path when it is non-NULL and
 * the last row is returned in last_row[14] when non-NULL.  The final field is written to
 * w_out when non-NULL.  Returns STREAMS_B200_ENAN when the residual becomes NaN.  When the
 * input sets [output] dtstat, the statistics are sampled as manage_output does
 * (singleideal_gpu.F90:2012-2034: time_from_last_stat += dt after every step, a sample when it
 * reaches dtstat), starting from the case's restart averages.
 */
int streams_b200_run_case(const streams_b200_case* c, int nsteps, int precision, const char* progress_path,
                          double* last_row, double* w_out);
/*
 * run_case that also returns the statistics at the end: w_stat_out (70*nx*ny), w_stat_3d_out
 * (14*nx*ny*nz) and stat_clock[2] = itav, time_from_last_stat (each may be NULL).  With
 * output_dir non-NULL the files that the end of run() writes are written there
 * (singleideal_gpu.F90:1660-1683: rst.bin, stat.bin, stat3d.bin, field_info0.dat).
 */
int streams_b200_run_case_stats(const streams_b200_case* c, int nsteps, int precision, const char* progress_path,
                                double* last_row, double* w_out, double* w_stat_out, double* w_stat_3d_out,
                                double* stat_clock, const char* output_dir);

#ifdef __cplusplus
}
#endif

#endif /* STREAMS_B200_HOST_H */
