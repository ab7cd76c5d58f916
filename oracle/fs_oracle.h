/*
 * fs_oracle.h -- CPU FP64 restatement of FilSim's hot path, used ONLY to check
 * results, by the tests, by __graft_entry__.smoke() and by bench.py's CPU
 * baseline. It is not part of the product and the product never calls it.
 *
 * Parity status: the reference (MPI + FFTW 2.1.5 + Armadillo) cannot be built
 * here, and the reference ships no golden vectors or known-answer files, so the
 * restatement is "parity unpinned" against reference outputs. It is pinned
 * instead against analytic known answers (sinusoidal Stokes forcing, Stokes
 * drag, single-bead periodic self-mobility) and its FFT against numpy.fft.
 */
#ifndef FS_ORACLE_H
#define FS_ORACLE_H
#include "../include/filsim_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } or_cpx;

/* FFT checks */
void or_fft_r2c_3d(const double *in, or_cpx *out, int nx, int ny, int nz);
void or_fft_c2r_3d(or_cpx *in, double *out, int nx, int ny, int nz);

/* FCM */
int or_fcm_mobility(const fs_params *p, int np, const double *Y, const double *F, const double *T,
                    double *V, double *W, double *fgrid, double *ugrid);
int or_flow_solve(const fs_params *p, const double *f, double *u);
void or_fcm_friction(const fs_params *p, int np, const double *F, const double *T, double *V, double *W);

/* cells + collision barrier */
void or_cells_dims(const fs_params *p, int *mxyz);
void or_cells_bulkmap(const int *mxyz, int *map);
void or_cells_link(const fs_params *p, int np, const double *Xs, int *head, int *list);
int or_collision_barrier(const fs_params *p, int np, const int *fil_id, const int *seg_id,
                         const double *Y, const int *head, const int *list, const int *map, int nt,
                         double *F, double *min_dist2, int *pairs, int max_pairs);

/* filament suspension + implicit step */
typedef struct or_system or_system;
or_system *or_system_create(const fs_params *p, const fs_host_state *s);
void or_system_destroy(or_system *sys);
void or_system_get(or_system *sys, fs_host_state *s);
void or_system_set(or_system *sys, const fs_host_state *s);
double *or_system_array(or_system *sys, const char *which);
void or_initial_guess(or_system *sys);
/* swimming drive: swim = per filament (alpha, beta, phase, wavenumber, angular
 * frequency) or NULL (off); spring links: nlinks bead pairs (global indices) */
void or_set_swimming(or_system *sys, const double *swim, double curvature, int sperm_decay);
void or_set_spring_links(or_system *sys, int nlinks, const int *beads, double k, double l0);
void or_filament_forces(or_system *sys, int nt);
/* barrier pair filter (FS_BARRIER_*) used by the implicit step */
void or_set_barrier_mode(or_system *sys, int mode);
/* one step of the gait-reset driver: iters[3], vwf: [3][Nw0][9] (V, W, F of filament 0) or NULL */
int or_step_gait_reset(or_system *sys, int nt, int *iters, double *vwf);
void or_build_jacobian(or_system *sys, int nt);
void or_get_jinv(or_system *sys, int f, double *out);
int or_error_check(or_system *sys, const double *V, const double *W, double *err, int nt);
void or_jsolve(or_system *sys, const double *b, double *x, int iter);
void or_set_cols(or_system *sys, const double *c, const double *d, int iter);
void or_update(or_system *sys, const double *upd);
void or_step(or_system *sys, int nt);
int or_step_implicit(or_system *sys, int nt, int *iters);
int or_run_steps(or_system *sys, int nt_start, int nsteps, int *iters);
/* CPU-baseline timing sample: stage wall times of one iteration, each stage run
 * on every stride-th work unit and scaled back (parts: 9 doubles) */
int or_sample_costs(or_system *sys, int stride, double *parts);
/* the same for the stages selected by mask (bit i: parts[i]); stride 1 = full
 * size; warm = 1 runs the stages once untimed first */
int or_stage_costs(or_system *sys, int stride, unsigned mask, int warm, double *parts);
/* last step's barrier minimum squared distance */
double or_last_min_dist2(or_system *sys);
long long or_mobility_solves(or_system *sys);

/* the seeded suspension generator, restated (or_suspension.c): X (nfil*nw x 3),
 * Q (nfil*nw x 4); 0 = placed, 8 = a filament could not be placed, 1 = bad args */
int or_suspension_random(const fs_params *p, int nfil, int nw, unsigned long long seed, double min_sep,
                         int max_tries, double *X, double *Q);

#ifdef __cplusplus
}
#endif
#endif
