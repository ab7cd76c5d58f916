/*
 * filsim_gpu.h -- C-ABI of libfilsim_gpu, the sm_100a (B200) implementation of
 * FilSim's hot path: the Force Coupling Method (FCM) mobility solve, the
 * cell-linked-list collision barrier, and the implicit BDF2 + Broyden step that
 * drives them.
 *
 * Conventions (shared by every entry point):
 *   - All arrays are plain contiguous C arrays. Per-bead vectors are Np x 3
 *     row-major doubles (x0 y0 z0 x1 y1 z1 ...), exactly the storage behind the
 *     reference's `double**` bead arrays (c_array_functions.cpp:12-21), so a
 *     caller passes `&fcm.Y[0][0]`.
 *   - Pointers are DEVICE pointers unless the parameter name ends in `_h`
 *     (host memory).
 *   - Every entry point returns an fs_status (0 = FS_OK). No C++ exception
 *     crosses the ABI. fs_status_string() gives a message.
 *   - One fs_ctx per CUDA stream; a context is not thread-safe. Work is queued
 *     on the context's stream; entry points that return host values
 *     synchronise that stream.
 *   - There is no CPU fallback: on a machine without a usable sm_100 GPU,
 *     fs_create returns FS_ERR_NO_DEVICE.
 *
 * Reference interfaces replaced (file:line inside the FilSim sources):
 *   struct Fcm               FCMfunctions.hpp:7-59
 *   struct LinkedList        CollisionBarrierFilament.hpp:19-57
 *   class filamentJsolver    FilamentJacobianSolver.hpp:14-87
 *   Filament per-step calls  Filament.hpp:227-505, 803-1120
 *   ErrorCheckFCM            MobilityConstraints.cpp:447-770
 *   time loop                main.cpp:284-754
 */
#ifndef FILSIM_GPU_H
#define FILSIM_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FS_ABI_VERSION 2

typedef int fs_status;
enum {
  FS_OK = 0,
  FS_ERR_INVALID_ARG = 1,     /* bad size, null pointer, unsupported parameter */
  FS_ERR_NO_DEVICE = 2,       /* no CUDA device, or not sm_100 */
  FS_ERR_CUDA = 3,            /* a CUDA runtime call failed */
  FS_ERR_CUFFT = 4,           /* a cuFFT call failed */
  FS_ERR_OOM = 5,             /* device allocation failed */
  FS_ERR_NOT_CONVERGED = 6,   /* Broyden reached broyden_maxiter (state is still advanced, as the reference does) */
  FS_ERR_NONFINITE = 7,       /* NaN/Inf met in a residual */
  FS_ERR_CAPACITY = 8,        /* an internal fixed-size list overflowed (reported, never written out of bounds) */
  FS_ERR_STATE = 9,           /* call order violated (e.g. barrier before link) */
  FS_ERR_IO = 10              /* a file could not be opened, written or parsed */
};

/* Precision of the FCM spread / FFT / interpolation chain. */
enum { FS_PREC_FP64 = 0, FS_PREC_FP32 = 1 };

/*
 * Runtime parameters. They replace the compile-time macros of config.hpp and the
 * derived constants of multi_filament_header.hpp:32-81. fs_params_default()
 * fills the values the reference derives (sigma = a/sqrt(pi),
 * sigma_dip = a/(36 pi)^(1/6), dx = sigma_dip/1.5, cell width 2.5a, ...).
 */
typedef struct fs_params {
  int npts_x, npts_y, npts_z;   /* NPTS_X/Y/Z: periodic FCM grid */
  int ngd;                      /* Gaussian support points per axis (reference `ngd`), 2..20, at most the grid size */
  double a;                     /* bead radius (FCM kernels, drag) */
  double ah;                    /* radius of bead 0 of each filament (Jacobian, `ah`) */
  double mu;                    /* viscosity MU */
  double dx;                    /* grid spacing; box length = npts * dx */
  double sigma;                 /* monopole Gaussian width */
  double sigma_dip;             /* dipole Gaussian width */
  double dl;                    /* bead spacing DL */
  double dt;                    /* time step */
  double gravity[3];            /* external force added to every bead (WeightPerLength*DL) */
  double strain_twist[3];       /* intrinsic strain-twist (STRAINTWISTZ, X, Y) */
  double tol;                   /* Broyden tolerance: any(|Err| > tol) keeps iterating */
  int broyden_maxiter;          /* Broyden iteration cap (reference: 300) */
  int impl_euler_steps;         /* ImplEulerSteps: nt <= this uses implicit Euler */
  int initial_friction_steps;   /* initialFrictionSteps: nt <= this uses Stokes drag only */
  int precision;                /* FS_PREC_FP64 or FS_PREC_FP32 for the FCM chain */
  double barrier_fs_over_2a;    /* Barrier_FS_over_2a */
  double barrier_distance_cap;  /* Barrier_distance_cap */
  double cell_width;            /* Rref: ideal collision cell width (2.5a) */
  int lambda_extrap_step;       /* nt at which lambda extrapolation turns linear (reference: 12) */
  int reserved0;
} fs_params;

/* Per-call diagnostics of the last fs_run_steps / fs_step_implicit call. */
typedef struct fs_diag {
  int last_nt;                  /* last completed time step */
  int last_iters;               /* Broyden iterations of the last step */
  long long total_iters;        /* Broyden iterations summed over the call */
  long long mobility_solves;    /* FCM (or friction) solves issued */
  int not_converged_steps;      /* steps that stopped at broyden_maxiter */
  int nonfinite;                /* 1 if a NaN/Inf residual was seen */
  int explosion;                /* 1 if any |Err| > 1e6 was seen (reference warning) */
  int reserved;
  double min_dist2;             /* last collision-barrier minimum squared distance */
  double last_max_abs_err;      /* max |Err| at the end of the last step */
  long long learned_filaments;  /* filament-steps started from the learned iterate */
  long long fallback_filaments; /* filament-steps put back to the plain start (worse first residual) */
  long long escalated_iters;    /* Broyden iterations FP32 steps ran in FP64 (fs_set_precision_escalation) */
} fs_diag;

/*
 * Host-side view of the filament suspension, used to upload and download the
 * device-resident state. Layouts (all host pointers):
 *   fil_start[nfil+1]   bead prefix: filament f owns beads [fil_start[f], fil_start[f+1])
 *   X, Xs, Xt, U, Us, Ut, F, TAU   np*3   (Bead.hpp:33-44; Xs/Us/qs = iterate, X/U/q = current, Xt/Ut/qt = previous)
 *   q, qs, qt                      np*4   (scalar first)
 *   lam, lam1, lam2                (np-nfil)*3, link l of filament f at fil_start[f]-f+l
 *   kap, c                         nfil   (bending, twist moduli: myKAP, myC)
 * Any pointer may be NULL on download to skip that field.
 */
typedef struct fs_host_state {
  int nfil;
  int np;
  const int *fil_start;
  double *X, *Xs, *Xt;
  double *U, *Us, *Ut;
  double *q, *qs, *qt;
  double *F, *TAU;
  double *lam, *lam1, *lam2;
  double *kap, *c;
} fs_host_state;

typedef struct fs_ctx fs_ctx;

/* ---- library / context ---------------------------------------------------- */

int fs_abi_version(void);
const char *fs_status_string(fs_status s);
void fs_params_default(fs_params *p, int npts_x, int npts_y, int npts_z);

/* Allocates grids, cuFFT plans and bead buffers for up to max_beads beads and
 * max_filaments filaments (the suspension itself is uploaded later).
 * Replaces Fcm::initialise (FCMfunctions.cpp:10-168) and
 * LinkedList::initialise (CollisionBarrierFilament.cpp:274-304).
 * stream: a cudaStream_t, or NULL for a context-owned blocking stream (ordered
 * against the legacy default stream). */
fs_status fs_create(const fs_params *p, int max_beads, int max_filaments, void *stream, fs_ctx **out);
/* Replaces Fcm::free_memory (FCMfunctions.cpp:468-519). */
fs_status fs_destroy(fs_ctx *ctx);
fs_status fs_get_params(const fs_ctx *ctx, fs_params *p_h);
fs_status fs_set_precision(fs_ctx *ctx, int precision);
fs_status fs_synchronize(fs_ctx *ctx);
/* Bytes of device memory the context holds. */
fs_status fs_device_bytes(const fs_ctx *ctx, size_t *bytes_h);

/* ---- FCM mobility (struct Fcm) -------------------------------------------- */

/* V, W (np x 3) from positions Y, forces F and torques T (np x 3), periodic
 * Stokes flow. Replaces Fcm::mobility_solve (FCMfunctions.cpp:175-464):
 * GA_setup :536-547, gaussian_setup :549-593, spread :596-646, forward FFT
 * :360-372, flow_solve :648-736, inverse FFT :403-406, particle_velocities
 * :740-770, particle_rotations :774-808. Y may lie anywhere in (-L, L) per axis
 * (the reference's fmod output). Precision follows fs_set_precision. */
fs_status fs_fcm_mobility(fs_ctx *ctx, const double *Y, const double *F, const double *T,
                          double *V, double *W, int np);
/* Same call on HOST buffers: copies in, solves, copies out, synchronises. */
fs_status fs_fcm_mobility_host(fs_ctx *ctx, const double *Y_h, const double *F_h, const double *T_h,
                               double *V_h, double *W_h, int np);
/* Stokes drag only: V = F/(6 pi mu a), W = T/(8 pi mu a^3).
 * Replaces Fcm::friction_mobility_solve (FCMfunctions.cpp:865-880). */
fs_status fs_fcm_friction(fs_ctx *ctx, const double *F, const double *T, double *V, double *W, int np);
/* The force-distribution step alone (GA_setup + gaussian_setup +
 * mono_and_dipole_force_distribution, FCMfunctions.cpp:536-646) in the
 * context's precision (FP32: the FP32 chain's spread, widened): writes the
 * spread force grid f (device, 3 x Nx x Ny x Nz doubles, component-major,
 * z fastest). */
fs_status fs_fcm_spread(fs_ctx *ctx, const double *Y, const double *F, const double *T, int np, double *f);
/* Copies the velocity grid u of the last FP64 mobility solve (3 x Nx x Ny x Nz
 * doubles) to host; count is the number of doubles grid_h holds. */
fs_status fs_fcm_get_grid(fs_ctx *ctx, double *grid_h, size_t count);
/* Runs flow_solve alone on a given force grid (3 x Nx x Ny x Nz, device):
 * forward FFT, projection, inverse FFT, result written to u (same layout).
 * Used for the reference's sinusoidal-forcing check (FCMfunctions.cpp:252-275). */
fs_status fs_fcm_flow_solve(fs_ctx *ctx, const double *f, double *u);

/* ---- collision barrier (struct LinkedList) -------------------------------- */

/* Cell grid sizes M_X, M_Y, M_Z (CollisionBarrierFilament.cpp:277-281). */
fs_status fs_cells_dims(const fs_ctx *ctx, int *mxyz_h);
/* Bins beads into cells from unwrapped positions Xs (np x 3) with a counting
 * sort; the result is the reference's head/list linked list. Synchronises the
 * context's stream; FS_ERR_CAPACITY if a cell holds 4096 beads or more (the
 * barrier's visiting-order key keeps list positions in 12 bits).
 * Replaces LinkedList::link (CollisionBarrierFilament.cpp:370-433). */
fs_status fs_cells_link(fs_ctx *ctx, const double *Xs, int np);
/* Copies the linked list out: head (ncell), list (np), map (13*ncell); any may be NULL. */
fs_status fs_cells_get_lists(fs_ctx *ctx, int *head_h, int *list_h, int *map_h);
/* Adds the barrier forces for positions Y into F_inout (both np x 3, device)
 * using the cells of the last fs_cells_link. min_dist2_h (may be NULL)
 * receives the minimum squared separation examined.
 * fil_id, seg_id: per-bead filament/segment number (device ints) or NULL to
 * use the uploaded suspension. Synchronises the context's stream;
 * FS_ERR_CAPACITY (discard F_inout) if the last link overflowed a cell or a
 * bead takes part in more than 64 barrier interactions.
 * Replaces LinkedList::apply_collision_barrier (CollisionBarrierFilament.cpp:24-271). */
fs_status fs_collision_barrier(fs_ctx *ctx, const double *Y, double *F_inout, int np, int nt,
                               const int *fil_id, const int *seg_id, double *min_dist2_h);
/* Lists the interacting pairs (i, j) in the reference's visiting order
 * (pairs_h: 2*max_pairs ints); *npairs_h receives the total count. */
fs_status fs_collision_pairs(fs_ctx *ctx, const double *Y, int np, int nt,
                             const int *fil_id, const int *seg_id,
                             int *pairs_h, int max_pairs, int *npairs_h);

/* ---- one box over several ranks: x slabs ------------------------------------ */

/* The pieces of an FCM mobility solve split over ranks by x slabs, as the
 * reference splits it with FFTW-MPI (FCMfunctions.cpp:16-23, 360-406, 460-461);
 * filsim_b200/slab.py drives them and makes the exchanges between ranks.
 * A rank owning planes [x0, x0 + nxs) of an nx_box-plane box creates its context
 * for a WINDOW of nxs + H planes (H >= ngd - 1) and calls fs_set_slab(ctx, x0,
 * nx_box): fs_fcm_spread and fs_fcm_interpolate then take the beads whose
 * stencil starts in the rank's planes (others are clamped into the window, not
 * spread correctly: the caller passes only its own beads). nx_box = 0 ends
 * slab mode. */
fs_status fs_set_slab(fs_ctx *ctx, int x0, int nx_box);
/* particle_velocities + particle_rotations (FCMfunctions.cpp:740-808) from a
 * given velocity grid u (device, 3 x the context's grid, component-major, z
 * fastest) in the context's precision. */
fs_status fs_fcm_interpolate(fs_ctx *ctx, const double *u, const double *Y, int np, double *V, double *W);
/* Slab transforms (FP64; complex values as (re, im) double pairs):
 * forward: f [3][nxs][Ny][Nz] real -> spec [3][nxs][Nz/2+1][Ny], z real-to-complex
 * then y; solve_x: spec_t [3][nkz][Ny][Nx] (the rank's kz range [kz0, kz0 + nkz),
 * every x) -> forward x, the projection of flow_solve (FCMfunctions.cpp:648-736),
 * inverse x, in place; inverse: spec (consumed) -> u [3][nxs][Ny][Nz], inverse
 * y, the imaginary parts of kz = 0 and kz = Nz/2 dropped (the reference's
 * halfcomplex inverse), real inverse z. Unnormalised but for the projection's
 * 1/(Nx Ny Nz), as the reference. Require fs_set_slab. */
fs_status fs_slab_forward_yz(fs_ctx *ctx, const double *f, int nxs, double *spec);
fs_status fs_slab_solve_x(fs_ctx *ctx, double *spec_t, int kz0, int nkz);
fs_status fs_slab_inverse_yz(fs_ctx *ctx, double *spec, int nxs, double *u);

/* ---- collision barrier without device allocation --------------------------- */

/* No counterpart in the reference. For callers that cannot allocate device
 * memory -- a host program that hands this library a fixed budget through its
 * own memory pool, or a step loop that must not pay cudaMalloc's device-wide
 * synchronisation -- this one call bins beads into cells from unwrapped
 * positions Xs and adds the barrier forces for positions Y into F_inout, as
 * fs_cells_link followed by fs_collision_barrier do, without a context. It
 * allocates nothing: its working memory is one static 4 MiB device array that
 * every GPU loading this library holds until the process exits, which limits
 * a call to FS_NOALLOC_MAX_BEADS beads and FS_NOALLOC_MAX_CELLS cells (larger
 * calls, and a cell width that is not finite and positive, return
 * FS_ERR_INVALID_ARG). The first call on a device looks up the
 * array's device address on that device, so make it before any stream capture.
 * All calls share the array: calls that overlap on the GPU (different streams or
 * host threads) race. stream: a cudaStream_t or NULL; the call synchronises it.
 * All array arguments are device pointers; min_dist2_h (may be NULL) is host.
 * FS_ERR_CAPACITY: a cell holds 4096 beads or more (F_inout is left unchanged),
 * or a bead takes part in more than 64 barrier interactions (F_inout then
 * holds the sums of the interactions that fitted and must be discarded). */
#define FS_NOALLOC_MAX_BEADS 65536
#define FS_NOALLOC_MAX_CELLS 262144
fs_status fs_collision_barrier_noalloc(const fs_params *p, const double *Xs, const double *Y, double *F_inout,
                                       int np, int nt, const int *fil_id, const int *seg_id, void *stream,
                                       double *min_dist2_h);

/* ---- filament suspension and the implicit step ----------------------------- */

/* Uploads / downloads the suspension (fs_host_state layouts). */
fs_status fs_state_upload(fs_ctx *ctx, const fs_host_state *s_h);
fs_status fs_state_download(fs_ctx *ctx, fs_host_state *s_h);
/* Device pointers of the resident bead arrays, for callers that drive the
 * step themselves: which = "Xs", "X", "Xt", "Us", "U", "Ut", "qs", "q", "qt",
 * "F", "TAU", "Y", "V", "W", "lam", "err", "update". */
fs_status fs_state_device_ptr(fs_ctx *ctx, const char *which, double **ptr_h);

/* Filament::initialGuess (Filament.hpp:227-237, Bead.hpp:202-217). */
fs_status fs_initial_guess(fs_ctx *ctx);
/* Filament::unRobotArmify, setZeroForcesTorques, applyElasticTorques,
 * applyConstraintForcesTorques, applyExternalForcesTorques
 * (Filament.hpp:271-402, 489-505), then Fcm::assign_filament_data
 * (FCMfunctions.cpp:882-918): Y = fmod(Xs, L), F, T into the FCM arrays. */
fs_status fs_filament_forces(fs_ctx *ctx, int nt);
/* Swimming drive (applyElasticTorques, Filament.hpp:297-326; set up per
 * filament as filament_initialisation_functions.cpp:806-833 does): swim_h is
 * nfil x 5 host doubles (Alpha, Beta, Phase, Wavenumber, AngFrequency) of the
 * uploaded suspension, or NULL to switch the drive off. On link i at time
 * t = nt dt the strain twist's components 1 and 2 are Beta facPref cos(Wavenumber s
 * - AngFrequency t + Phase) and Alpha facPref sin(...), s = dL (i + 1/2),
 * T0 = curvature / (Nw dL) and facPref = T0 (L - s) / L, or with sperm_decay
 * T0 for s <= L/2 and 2 T0 (L - s) / L beyond (L = (Nw - 1) dL); the Jacobian
 * uses the last link's values as the reference's buildJacobian does. As in the
 * reference, components 1 and 2 of fs_params.strain_twist are replaced on
 * every link (zero without a drive); component 0 stays constant. Steps with a
 * drive run host-driven (a captured step graph would bake nt in), so an
 * ensemble batch, whose steps are captured, refuses a box with a drive
 * (FS_ERR_STATE). An upload with another filament layout drops the drive. */
fs_status fs_set_swimming(fs_ctx *ctx, const double *swim_h, double curvature, int sperm_decay);
/* Spring links between beads (spring_links::apply_spring_link_forces,
 * spring_link_functions.cpp:24-45, applied after the filaments' own forces as
 * main.cpp:354-357): beads_h holds 2 global bead indices per link, in link
 * order; each link adds k (|d| - l0) along the minimum-image displacement d of
 * its beads (VecPeriodicX, :139-145), - on the first bead and + on the second
 * (F -= k (|d| - l0) d / |d| on the first). nlinks 0 removes the links. The
 * indices must be distinct beads of the uploaded suspension; an upload with
 * another filament layout drops the links. */
fs_status fs_set_spring_links(fs_ctx *ctx, int nlinks, const int *beads_h, double k, double l0);

/* Pair filters of the collision barrier in the implicit step: the reference's
 * LinkedList::apply_collision_barrier (CollisionBarrierFilament.cpp:24-271),
 * apply_collision_barrier_not_swimmer (:441-697: no pairs between filament 0,
 * the swimmer, and the other filaments), apply_collision_barrier_not_test_particles
 * (:698-945: no pairs with either of the last two beads), or no barrier. */
enum {
  FS_BARRIER_ALL = 0,
  FS_BARRIER_NOT_SWIMMER = 1,
  FS_BARRIER_NOT_TEST_PARTICLES = 2,
  FS_BARRIER_OFF = 3
};
fs_status fs_set_barrier_mode(fs_ctx *ctx, int mode);
/* One time step of the gait-reset driver (main_gaitreset.cpp:302-830): three
 * solves of the implicit step from the same committed state, (0) without the
 * barrier, (1) without swimmer-network barrier pairs, (2) with the context's
 * barrier mode, and only the last one commits (Filament::step); lambda carries
 * from one solve to the next as in the reference. iters_h[3]: Broyden
 * iterations of each solve. vwf_h (optional): per solve, filament 0's beads'
 * V, W and F after the solve ([3][Nw0][9]), the rows the reference writes with
 * save_swimmer_velocity_data_to_file. Host-driven (no step graph). */
fs_status fs_step_gait_reset(fs_ctx *ctx, int nt, int *iters_h, double *vwf_h);
/* filamentJsolver::buildJacobian (FilamentJacobianSolver.hpp:36-47 and
 * Filament.hpp:803-1120): per filament the approximate Jacobian is built and
 * LU-factorised; Broyden history is cleared. */
fs_status fs_jacobian_build(fs_ctx *ctx, int nt);
/* Copies the explicit inverse J0^-1 of filament f (6Nw x 6Nw row-major, with
 * the reference's 1/dt row scaling, Filament.hpp:862-865) to host. */
fs_status fs_jacobian_get_inverse(fs_ctx *ctx, int f, double *jinv_h, int n);
/* ErrorCheckFCM (MobilityConstraints.cpp:447-770): err (6Np) from V, W (np x 3);
 * *check_h = 1 if any |err| > tol. */
fs_status fs_error_check(fs_ctx *ctx, const double *V, const double *W, double *err, int nt, int *check_h);
/* filamentJsolver::solve (FilamentJacobianSolver.hpp:49-73): x = J0^-1 b plus
 * the bad-Broyden corrections of the first `iter` history columns. */
fs_status fs_broyden_apply(fs_ctx *ctx, const double *b, double *x, int iter);
/* addCmatCol / addDmatCol (FilamentJacobianSolver.hpp:76-84). */
fs_status fs_broyden_set_cols(fs_ctx *ctx, const double *c, const double *d, int iter);
/* Filament::update (Filament.hpp:425-452): state -= update (6Np). */
fs_status fs_state_update(fs_ctx *ctx, const double *update);
/* Filament::step (Filament.hpp:455-478). */
fs_status fs_step(fs_ctx *ctx, int nt);
/* One full implicit time step nt (main.cpp:284-754 loop body). */
fs_status fs_step_implicit(fs_ctx *ctx, int nt, int *iters_h);
/* nsteps implicit steps from nt_start; iters_h (may be NULL) receives the
 * Broyden iteration count of each step. */
fs_status fs_run_steps(fs_ctx *ctx, int nt_start, int nsteps, int *iters_h);
fs_status fs_get_diag(fs_ctx *ctx, fs_diag *d_h);
/* 1: steps in the steady regime (nt above impl_euler_steps, initial_friction_steps
 * and lambda_extrap_step) run as one CUDA graph each, with the Broyden loop on
 * the device (a conditional WHILE node) and one host synchronisation per
 * fs_run_steps call instead of one per iteration; results are bitwise those of
 * the host-driven step. With the learned warm start on, only the steps its cost
 * gate gives the plain start run as graphs (one synchronisation per step);
 * learned-start and recording steps run host-driven. No reference counterpart. */
fs_status fs_set_graph_mode(fs_ctx *ctx, int on);

/* ---- autotuner (no reference counterpart) -----------------------------------
 * choice = {beads staged per spread pass (32 | 64), beads per interpolation CTA
 * (4 | 8 | 16), FP32 power-of-two grids: 0 warp FFT | 1 cuFFT, FP32 spread: x
 * width of a warp's column block in the 16^3 tile (2 | 4 | 8; the block is
 * w x 16 x 16/w points)}: four ints. fs_autotune times every combination on the
 * uploaded suspension (reps mobility solves each, after one warm-up) and keeps
 * the fastest; best_ms_h: its time per solve. */
fs_status fs_autotune(fs_ctx *ctx, int reps, int *choice_h, float *best_ms_h);
fs_status fs_set_tuning(fs_ctx *ctx, const int *choice_h);

/* ---- ensembles of independent boxes (no reference counterpart; the reference
 * runs such sweeps one program at a time, batch_compile.py) ------------------- */
typedef struct fs_batch fs_batch;
/* n contexts with distinct streams, each holding its own box (grid, params,
 * suspension); the batch does not own them. */
fs_status fs_batch_create(fs_ctx *const *ctxs, int n, fs_batch **out);
fs_status fs_batch_destroy(fs_batch *b);
/* nsteps steady-regime steps (nt_start past every box's start-up steps) of every
 * box. Each ensemble step is one CUDA graph launch holding every box's captured
 * step on its own stream (fork/join), Broyden loops on the device; one host
 * synchronisation for the whole call. iters_h, box_ms_h: [nsteps x n] iteration
 * counts and per-box step device times (may be NULL); total_ms_h: the call's
 * device time. The graph is captured at the first call. */
fs_status fs_batch_run(fs_batch *b, int nt_start, int nsteps, int *iters_h, float *box_ms_h, float *total_ms_h);

/* ---- stage profiling ---------------------------------------------------------- */

/* Device time per stage, taken with CUDA events on the context's stream. The
 * stages follow the columns of the reference's profiler (profilers.hpp:22-60,
 * printed per step by profilers.cpp:46-65). */
enum {
  FS_STAGE_SPREAD = 0,      /* binning + force distribution (FCMGauss + FCMForcD) */
  FS_STAGE_FFT_FWD = 1,     /* forward real transform x3 (FCMFFTFw); FP32 power-of-two grids: z and y passes */
  FS_STAGE_PROJECT = 2,     /* Stokes projection (FCMFlowS); FP32 power-of-two grids: with the x transforms */
  FS_STAGE_FFT_INV = 3,     /* inverse real transform x3 (FCMFFTBk); FP32 power-of-two grids: y and z passes */
  FS_STAGE_INTERP = 4,      /* U and Omega interpolation (FCMParVR) */
  FS_STAGE_LINK = 5,        /* cell binning (ColBarri, link) */
  FS_STAGE_BARRIER = 6,     /* pair forces (ColBarri) */
  FS_STAGE_FORCES = 7,      /* unRobotArmify + filament forces + assign (Assign F) */
  FS_STAGE_JACOBIAN = 8,    /* J build + Schur-complement inverse (Bld Jinv) */
  FS_STAGE_ERROR_CHECK = 9, /* ErrorChk */
  FS_STAGE_BROYDEN = 10,    /* J0^-1 applications + history (Slv Jinv) */
  FS_STAGE_UPDATE = 11,     /* state update + step */
  FS_STAGE_FRICTION = 12,   /* Stokes-drag mobility */
  FS_STAGE_LEARN = 13,      /* warm-start features + MLP inference, and MLP training steps */
  /* single kernels inside the stages above (their time also counts there) */
  FS_STAGE_K_SPREAD = 14,   /* the force-distribution kernel alone (no binning or records) */
  FS_STAGE_K_FFT_Z_FWD = 15, /* FP32 transform: the forward pass over z lines */
  FS_STAGE_K_FFT_Y_FWD = 16, /* FP32 transform: the forward pass over y lines */
  FS_STAGE_K_FFT_Y_INV = 17, /* FP32 transform: the inverse pass over y lines */
  FS_STAGE_K_FFT_Z_INV = 18, /* FP32 transform: the inverse pass over z lines */
  FS_STAGE_K_INTERP = 19,   /* the interpolation kernel alone */
  FS_STAGE_COUNT = 32
};
typedef struct fs_profile {
  double ms[FS_STAGE_COUNT];     /* summed device milliseconds */
  long long calls[FS_STAGE_COUNT];
} fs_profile;
/* Turns stage timing on (1) or off (0); either resets the sums. */
fs_status fs_profile_enable(fs_ctx *ctx, int on);
/* Synchronises and returns the sums since the last enable. */
fs_status fs_profile_get(fs_ctx *ctx, fs_profile *out_h);
/* Number of kernels this library has launched in the process (cuFFT's own
 * kernels are not counted). */
unsigned long long fs_kernel_launches(void);

/* ---- learned Broyden warm start (no reference counterpart) --------------------
 *
 * A per-filament MLP (features -> 3 x [Linear(hidden) + SiLU] -> Linear) that
 * predicts, for filaments of nw beads, the update from the extrapolated guess
 * of Filament::initialGuess (Filament.hpp:227-237) to the converged state of
 * the step, in the Broyden unknowns' layout [X0 (3) | U (3 nw) | lambda
 * (3 nw - 3)], and a correction to the diagonal of the initial inverse
 * Jacobian (6 nw). Trained and evaluated by this library's BF16 tensor-core
 * GEMMs (FP32 accumulation, FP32 master weights, Adam).
 *
 * Features per filament (n_features = 19 nw + 9 (nw - 1) + 1), for bead i:
 * X_i - centroid (3), q_i (4), (X_i - Xt_i)/dt (3), U_i/dt (3), Ut_i/dt (3),
 * (X_i - 2 Xt_i + Xtt_i)/dt^2 (3; Xtt: positions two steps back, kept by the
 * library from the steps it ran, zero after an upload that changes X or Xt);
 * for link j: lambda_j, lambda1_j, lambda2_j (9); then log K_B. Targets per filament
 * (n_targets = 12 nw): converged - guess (6 nw), then diag(sum_i C_i D_i^T) of
 * the Broyden history at convergence (6 nw). Inputs and targets are normalised
 * with the statistics given to fs_mlp_set_normalization. */

/* Creates (or replaces) the context's model for filaments of nw beads; hidden is
 * a multiple of 128; batch_capacity rows per GEMM pass (rounded up to 128);
 * weights uniform in +-1/sqrt(fan_in) from seed. */
fs_status fs_mlp_create(fs_ctx *ctx, int nw, int hidden, int batch_capacity, unsigned long long seed);
/* dims_h[8] = {nw, n_features, k_in (padded), hidden, n_targets, k_out (padded),
 * batch capacity, parameter count}. */
fs_status fs_mlp_dims(const fs_ctx *ctx, int *dims_h);
fs_status fs_mlp_set_normalization(fs_ctx *ctx, const float *in_mean_h, const float *in_std_h,
                                   const float *out_mean_h, const float *out_std_h);
/* Flat FP32 parameters [W1 b1 W2 b2 W3 b3 W4 b4], W_l row-major [out x in] with the
 * padded widths. Setting them resets the Adam moments. */
fs_status fs_mlp_get_params(fs_ctx *ctx, float *params_h, size_t count);
fs_status fs_mlp_set_params(fs_ctx *ctx, const float *params_h, size_t count);
/* Denormalised predictions [n x n_targets] of raw features [n x n_features] (device). */
fs_status fs_mlp_forward(fs_ctx *ctx, const float *features_d, int n, float *out_d);
/* Gradients of the mean-square loss of one batch (n <= capacity rows), in the
 * flat parameter layout, without an update. */
fs_status fs_mlp_gradients(fs_ctx *ctx, const float *features_d, const float *targets_d, int n, float *grads_h,
                           size_t count, double *loss_h);
/* One Adam step (beta 0.9, 0.999, eps 1e-8) on a batch; loss_h may be NULL (no sync). */
fs_status fs_mlp_train_step(fs_ctx *ctx, const float *features_d, const float *targets_d, int n, float lr,
                            double *loss_h);
/* Features [nfil x n_features] of the uploaded state (filaments of another
 * length get zeros). */
fs_status fs_learn_features(fs_ctx *ctx, float *features_d);
/* While on, every implicit step keeps its targets for fs_learn_targets. */
fs_status fs_learn_record(fs_ctx *ctx, int on);
/* Targets [nfil x n_targets] of the last recorded step. */
fs_status fs_learn_targets(fs_ctx *ctx, float *targets_d);
/* The next warm-started step uses pred_d [nfil x n_targets] (denormalised, as
 * fs_mlp_forward returns) instead of the network's output: for checking the
 * start and fallback logic with known predictions. */
fs_status fs_learn_override(fs_ctx *ctx, const float *pred_d);
/* 0: the reference's start; 1: learned iterate; 2: learned iterate and
 * inverse-Jacobian diagonal. A filament whose first residual (max |Err| over its
 * rows) from the learned start exceeds that of the plain start is put back to
 * the plain start. */
fs_status fs_set_warm_start(fs_ctx *ctx, int mode);
/* Start of each implicit step's Broyden iteration (no reference counterpart).
 * order 1 (the default): Filament::initialGuess, the first bead of each filament
 * from 2X - Xt (Filament.hpp:227-237, Bead.hpp:202-216). order 2: the first bead
 * from 3X - 3Xt + Xtt, Xtt its position two steps back, which the context keeps
 * from then on; order 1 until that history spans two steps the context ran
 * itself (the first two steps, and the first two after an upload that changes X
 * or Xt: an uploaded Xt need not come from a step); every other unknown starts
 * as in order 1. The reference's start extrapolates the orientations (through
 * Us = 2U - Ut, U a per-step increment) to second order but the first bead's
 * position, which carries the whole filament, to first order only; order 2
 * makes it second order too. The Broyden loop and its convergence test are
 * unchanged: a step converges to the same tolerance from either start. A
 * learned start (fs_set_warm_start) corrects whichever start is set. */
fs_status fs_set_start_order(fs_ctx *ctx, int order);
/* Tension start of each step, set by Filament::step for the next one (no
 * reference counterpart). order 2 (the default): the reference's constant
 * extrapolation before lambda_extrap_step, linear at it, quadratic
 * (3 lam - 3 lam1 + lam2) after it. order 1: linear (2 lam - lam1) from
 * lambda_extrap_step on: the converged tensions carry the Broyden tolerance's
 * noise, which the quadratic extrapolation amplifies up to 7x and the linear one
 * up to 3x. The Broyden loop and its convergence test are unchanged. */
fs_status fs_set_tension_extrapolation(fs_ctx *ctx, int order);
/* Velocity predictor (no reference counterpart): with weight w > 0 each implicit
 * step, before its first residual (which needs a mobility solve), takes one
 * Broyden update x <- x - w H E(x; V*, W*) from the residual evaluated with the
 * velocities extrapolated from the last two converged states, V* = 2 V1 - V2 and
 * W* = 2 W1 - W2: no solve. H is the iteration's inverse Jacobian at that point
 * (J0^-1 and any Broyden columns the memory carried). The iteration proper starts
 * at the updated iterate; the update adds no history column and counts as no
 * iteration, and the convergence test is unchanged. Without two converged states
 * since creation, a layout change or an upload that changes X or Xt the update is
 * zero. w in [0, 2]; 0 (the default) turns it off. */
fs_status fs_set_velocity_predictor(fs_ctx *ctx, double weight);
/* Broyden memory across steps (no reference counterpart). The reference starts
 * each step's iteration from J0^-1, the approximate inverse Jacobian of the
 * filaments without their hydrodynamic coupling, adds one rank-one "bad Broyden"
 * term per iteration (main.cpp:640-663) and drops them at the end of the step.
 * With the memory on:
 *  - after a converged step of fewer than `threshold` iterations whose history
 *    holds at most keep_columns columns, the next step keeps that J0 (no rebuild)
 *    and all the columns;
 *  - after a converged step of `threshold` or more iterations, its last
 *    carry_columns columns start the next step beside a new J0;
 *  - otherwise the next step starts as the reference's does;
 *  - a step running on carried state that reaches restart_after iterations
 *    (0: never) rebuilds J0 at its current iterate and empties the history.
 * An upload that changes X, Xt or the layout drops the carried state. The
 * convergence test is unchanged. The history grows to broyden_maxiter +
 * max(keep_columns, carry_columns) columns of 12 Np doubles. keep_columns =
 * carry_columns = 0 (the default) turns it off; each at most FS_BROYDEN_MEMORY_MAX. */
#define FS_BROYDEN_MEMORY_MAX 64
fs_status fs_set_broyden_memory(fs_ctx *ctx, int keep_columns, int carry_columns, int threshold, int restart_after);
/* Precision escalation of the mixed-precision chain (no reference counterpart):
 * with after_iters > 0 and the context in FS_PREC_FP32, a step still not
 * converged after after_iters Broyden iterations runs its remaining iterations
 * with the FP64 chain (host-driven and captured steps alike), then the next
 * step starts in FP32 again. The FP32 chain's error (~1e-6 of the velocities)
 * can leave a step that starts close to the tolerance wandering near it; the
 * FP64 iterations end that. 0 (the default) turns it off. */
fs_status fs_set_precision_escalation(fs_ctx *ctx, int after_iters);
/* Cost gate of the learned start (no reference counterpart): with period > 0,
 * each step runs the start whose running mean of mobility solves per step is
 * lower (the learned one only when it is lower by at least the margin of
 * fs_warm_start_gate_margin over at least two of its steps: a tie goes to the
 * reference's start), and probes the
 * other one so that its mean stays
 * current: after period steps, an interval that doubles (up to 16 x period)
 * while the probes leave the choice unchanged and returns to period when one
 * changes it; the learned start pays off only when it saves more
 * Broyden iterations than its own extra solves. period 0 (the default) runs the
 * learned start every step. Resets the statistics. */
fs_status fs_warm_start_gate(fs_ctx *ctx, int period);
/* The gate's margin: mobility solves per step the learned start must save to be
 * chosen, standing for its own cost (inference, a host-driven step); default
 * 0.25, about that cost at 512^3. Kept across fs_warm_start_gate calls. */
fs_status fs_warm_start_gate_margin(fs_ctx *ctx, double margin);
/* Carried bound of the learned start's fallback (no reference counterpart):
 * with refresh > 0, only every refresh-th learned step solves both starts (and
 * puts back, in that step, each filament whose learned first residual is
 * worse); it keeps each filament's plain-start first residual. The learned
 * steps in between cost one mobility solve: they solve the learned start
 * alone, and a filament whose first residual exceeds its carried plain one
 * takes the plain start from the next step until the next comparison. The
 * Broyden loop and its convergence test are unchanged. refresh 0 (the
 * default) compares with the plain start on every learned step. */
fs_status fs_warm_start_bound(fs_ctx *ctx, int refresh);
/* steps_h[2], solves_h[2]: steps run and running mean solves per step, [0] plain
 * start, [1] learned start, since the last fs_warm_start_gate. */
fs_status fs_warm_start_gate_stats(fs_ctx *ctx, long long *steps_h, double *solves_h);
/* D[M x N] (FP32) = A[M x K] B[N x K]^T with BF16 operands on the tensor cores;
 * M, N multiples of 128, K of 64. */
fs_status fs_gemm_bf16(fs_ctx *ctx, const void *A_d, const void *B_d, float *D_d, int M, int N, int K);

/* ---- synthetic inputs (host only, no GPU needed) ------------------------------ */

/* Seeded straight-filament suspension: nfil filaments of nw beads with the
 * placement of Filament::initialFilamentSetupIsoRandCentred (Filament.cpp:47-66)
 * and the periodic overlap rejection of Filament::checkOverlapWithPeriodic
 * (Filament.cpp:126-153) at separation min_sep. X_h: nfil*nw*3 unwrapped bead
 * positions; q_h: nfil*nw*4 quaternions (all beads of a filament share one).
 * Returns FS_ERR_CAPACITY if a filament cannot be placed in max_tries. */
fs_status fs_suspension_random(const fs_params *p, int nfil, int nw, unsigned long long seed, double min_sep,
                               int max_tries, double *X_h, double *q_h);

/* ---- reference-compatible run files (host only, no GPU needed) ---------------
 * Text files in the reference's formats, so runs resume each other's
 * checkpoints and feed the reference's plotting scripts. Numbers in .bak and
 * .dat files are written as C++ streams with precision(16) and ios::fixed
 * print them (printf "%.16f"), each followed by one space; .par values use the
 * stream default (printf "%g"). Quaternions are scalar first. Filaments are in
 * fs_host_state order (fil_start). */

/* Columns of the .par file (save_parameter_values_to_file,
 * file_functions.cpp:6-80), in the reference's names. Only Nsw and the bead
 * numbers are read back (continue_from_checkpoint); the rest documents the run. */
typedef struct fs_run_info {
  char simulation_name[128], simulation_tag[128];
  double a, ah, dl, sp4, kap, c, mu, curvature, k0;
  double time_steps, steps_per_period, tol;
  int broyden_maxiter;
  double box[3];            /* LfcmBox_x, LfcmBox_y, LfcmBox_z */
  int plot_steps;
  double strain_twist[3];   /* STRAINTWISTX, STRAINTWISTY, STRAINTWISTZ */
  double kap_network_filaments, bnumber, steps_per_settling_time, dt;
  int initial_friction_steps, enable_spring_links;
  double cn_num_swimming_filaments, cn_num_nodes, cn_connection_radius, cn_min_node_spacing,
      cn_spacing_away_from_node, network_spring_constant, network_spring_natural_length;
} fs_run_info;

/* .par (file_functions.cpp:6-80): the column names, the values, BeadNumbers
 * from s->fil_start and the bending factors s->kap[f] / info->kap (s->kap[f]
 * itself when info->kap is 0). */
fs_status fs_par_write(const char *path, const fs_run_info *info, const fs_host_state *s);
/* The layout continue_from_checkpoint reads from a .par (file_functions.cpp:236-272):
 * the third item of the second line is the filament count, the fifth line holds
 * the bead numbers. fil_start_h receives nfil + 1 offsets (capacity max_fil + 1);
 * *np_out the bead count. FS_ERR_CAPACITY if the file holds more than max_fil. */
fs_status fs_par_read_layout(const char *path, int *nfil_out, int *np_out, int *fil_start_h, int max_fil);
/* .bak (save_backup_data_to_file, file_functions.cpp:210-221, and
 * Filament::writeBackupData, Filament.hpp:650-679): nt, then per filament and
 * bead X, Xt, qs (q when s->qs is NULL), qt, U, Ut, then per link lam, lam1,
 * lam2; overwrites. */
fs_status fs_backup_write(const char *path, const fs_host_state *s, int nt);
/* Reads a .bak written for the layout s->fil_start / s->nfil / s->np
 * (continue_from_checkpoint, file_functions.cpp:274-303, and
 * Filament::continue_from_checkpoint, Filament.hpp:683-748): fills X, Xt, q,
 * qt, U, Ut, lam, lam1, lam2 and sets Xs = X, qs = q, Us = U; *nt_next = the
 * file's nt + 1, the step the reference resumes at. */
fs_status fs_backup_read(const char *path, fs_host_state *s, int *nt_next);
/* .dat (save_data_column_names_to_file, file_functions.cpp:84-97, and
 * save_data_to_file, :150-161; Filament::writeDataNames / writeData,
 * Filament.hpp:509-560): the header overwrites the file ("it", then X Y Z qr qi
 * qj qk per bead); a row appends nt and per bead Xs, qs. */
fs_status fs_data_write_header(const char *path, const fs_host_state *s);
fs_status fs_data_append(const char *path, const fs_host_state *s, int nt);

#ifdef __cplusplus
}
#endif
#endif /* FILSIM_GPU_H */
