// fs_internal.cuh -- context layout and helpers shared by the sm_100a kernels
// of libfilsim_gpu.
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include "../../include/filsim_gpu.h"

#define FS_PI 3.14159265358979323846264338327950288

// Spread tile edge (grid points); spread bins have the same width.
#define FS_TILE 16
// largest Gaussian support per axis (the reference's default, config_template.hpp:76)
#define FS_NGD_MAX 20
// dynamic shared memory a CTA may ask for on sm_100 (227 KB)
#define FS_SMEM_MAX (227 * 1024)
// spread bins per axis whose beads can reach a tile: a stencil of ngd points
// starting in bin t - k reaches tile t when 16 k <= ngd + 14
__host__ __device__ inline int fs_cand_bins(int ngd) { return (ngd + 14) / FS_TILE + 1; }
// Beads staged in shared memory per spread pass (a multiple of 32).
#define FS_SPREAD_CHUNK 64
// Collision events kept per bead (pairs inside the barrier range).
#define FS_MAX_EVENTS 64
// Flag words (device int array ctx->flags).
enum { FLAG_CHECK = 0, FLAG_NONFINITE = 1, FLAG_EXPLODE = 2, FLAG_CAPACITY = 3, FLAG_PIVOT = 4, FLAG_COUNT = 8 };

struct fs_sort {
  // counting sort of `n` items by integer key in [0, nkeys)
  int nkeys;
  int *key;      // per item
  int *count;    // nkeys
  int *start;    // nkeys + 1
  int *cursor;   // nkeys
  int *sorted;   // items in (key, id) order
  int *block_sums;
};

#define FS_PROF_SLOTS 512
struct fs_prof {
  bool on, created;
  cudaEvent_t ev[2 * FS_PROF_SLOTS];
  int stage[FS_PROF_SLOTS];
  int n;  // pending slots
  double ms[FS_STAGE_COUNT];
  long long calls[FS_STAGE_COUNT];
};

struct fs_ctx {
  fs_params p;
  fs_prof prof;
  int device;
  cudaStream_t stream;
  bool own_stream;
  int max_beads, max_fil;
  int precision;

  // FCM grid
  int nx, ny, nz, nzh;
  size_t N, NH;
  double L[3];
  void *grid_real;   // 3 x N reals (force grid f, then velocity grid u)
  void *grid_cplx;   // 3 x NH complex
  cufftHandle plan_fwd[2], plan_inv[2];  // [precision]
  bool plan_ok[2];
  int nbin[3], nbins;  // spread bins (FS_TILE wide in stencil-start space)
  fs_sort bins;
  int *bead_sw;        // per bead, wrapped Gaussian stencil start per axis
  float4 *spread_wb;   // FP32 chain: per sorted bead, stencil starts, F, T/2 and weights
  int last_grid_prec;  // precision of the grids from the last solve (-1: none)
  int tune_spread_chunk;  // beads staged per spread pass: 32 or 64 (fs_autotune)
  int tune_spread_cols;   // FP32 spread: x width of a warp's column block (2, 4 or 8)
  int tune_interp_wpb;    // beads (warps) per interpolation CTA: 4, 8 or 16
  int tune_fft32;         // FP32 power-of-two grids: 0 warp FFT (fs_fft.cu), 1 cuFFT
  void *fft_tw;        // FP32 transform twiddle tables (null: grid not handled by fs_fft.cu, cuFFT is used)

  // collision cells
  int M[3], ncell;
  fs_sort cells;
  int *head, *list, *map;
  int *cell_rank;      // descending-id rank of each bead inside its cell
  int *pair_count, *pair_off, *pair_scan_tmp;
  int cells_np;        // beads in the last link (-1: none)
  bool min_dist2_valid;  // a barrier has written min_dist2_bits
  int num_sms;           // streaming multiprocessors of the context's device
  int slab_x0, slab_nx;  // slab window: first plane and x extent of the whole box (0: not a window)
  struct fs_slab_plans *slab;  // cuFFT plans and scratch of the slab transforms (fs_slab.cu)
  double *min_dist2;   // device scalar
  unsigned long long *min_dist2_bits;

  // filament suspension (device)
  int nfil, np, nlink;
  bool have_state;
  int *fil_start_h;      // host copy of the uploaded layout (nfil + 1)
  int *fil_start, *fil_id, *seg_id;
  double *X, *Xs, *Xt, *U, *Us, *Ut, *q, *qs, *qt, *F, *TAU, *lam, *lam1, *lam2, *kap, *cc, *radius;
  double *Y, *V, *W;
  double *err, *newerr, *upd, *tmp, *dE;
  double *Cmat, *Dmat;   // broyden_maxiter x 6Np
  double *Sinv;          // per-filament inverse Schur complement (3Nw x 3Nw row-major) at soff[f]
  double *aux;           // per-filament D', F' blocks, tangents, P coefficient at aoff[f]
  long long *soff, *aoff;
  int max_nw, min_nw;  // longest and shortest filament
  // swimming drive (fs_set_swimming): per filament (alpha, beta, phase, wavenumber,
  // angular frequency); null when off. Spring links (fs_set_spring_links): bead
  // pairs and, per bead, its links in link order (entry 2 l + side).
  double *swim;
  double swim_curvature;
  int swim_sperm_decay;
  int nspring;
  int *spring_beads, *spring_off, *spring_ent;
  double spring_k, spring_l0;
  size_t spring_bytes, swim_bytes;  // device bytes of the spring-link arrays and the drive
  int barrier_mode;      // pair filter of the step's barrier (fs_set_barrier_mode)
  double *dots;          // broyden_maxiter partial dots
  double *partials;      // reduction scratch
  double *scalars;       // [0] = ||dE||
  int *flags;            // FLAG_COUNT ints
  int *flags_h;          // pinned host copy
  unsigned long long *maxerr_bits;
  fs_diag diag;
  size_t bytes;
  struct fs_mlp *mlp;    // learned warm start (fs_mlp.cu); null until fs_mlp_create
  // start of the implicit step (fs_set_start_order, fs_start.cu): 1 the reference's
  // first-bead extrapolation 2X - Xt, 2 quadratic, 3X - 3Xt + Xtt
  int start_order;
  // tension start of the next step (fs_set_tension_extrapolation, fs_start.cu): 2 the
  // reference's quadratic extrapolation after lambda_extrap_step, 1 linear (0: 2)
  int tension_order;
  // FP32 steps go on in FP64 after this many Broyden iterations (0: never;
  // fs_set_precision_escalation)
  int escalate_after;
  // Broyden memory across steps (fs_set_broyden_memory, fs_bmem.cu): J0 and up to
  // bmem_keep history columns continue after a step of fewer than bmem_thr
  // iterations; after a longer one its last bmem_carry columns start the next
  // step beside a new J0; a step on carried state that reaches bmem_restart
  // iterations drops it (0: never). bmem_cols = max(bmem_keep, bmem_carry), 0 when
  // off; bmem_cap: history columns allocated beyond broyden_maxiter; bmem_d: the
  // device state (BM_COUNT ints, fs_bmem.cu)
  int bmem_keep, bmem_carry, bmem_thr, bmem_restart, bmem_cols, bmem_cap;
  int *bmem_d;
  // velocity predictor (fs_set_velocity_predictor, fs_start.cu): the weight of its
  // update (0: off), V, W of the last two converged states (vp_V1, vp_W1 the
  // latest), the extrapolated V, W, and vp_ok (device): converged states recorded
  // since the last reset, up to 2
  double vpred_weight;
  double *vp_V1, *vp_W1, *vp_V2, *vp_W2, *vp_Vs, *vp_Ws;
  int *vp_ok;
  // positions two steps back (fs_start.cu), kept while the quadratic or the learned
  // start is on (3 max_beads doubles each); hist_ok (device): steps run since the
  // history was reset, up to 2 (hist_Xtt holds positions two steps back once it is
  // 1, all from this context's own steps at 2); hist_pX, hist_pXt: X, Xt before an upload
  double *hist_Xtt, *hist_pX, *hist_pXt;
  int *hist_ok;
  bool hist_cmp_pending;
  struct fs_graph *graph;  // captured steady step (fs_graph.cu); null until first used
  int graph_mode;        // 1: steady steps run as CUDA graphs with the Broyden loop on the device
  int graph_gen;         // bumped whenever captured graphs of this context become stale
  int *gemm_err;         // error word of fs_gemm_bf16 (allocated at its first call)
};

#define FS_CUDA(call)                                                         \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      fprintf(stderr, "filsim_gpu: %s failed: %s (%s:%d)\n", #call,          \
              cudaGetErrorString(e_), __FILE__, __LINE__);                    \
      return e_ == cudaErrorMemoryAllocation ? FS_ERR_OOM : FS_ERR_CUDA;      \
    }                                                                         \
  } while (0)

// kernels this library has launched in the process (every launch is followed by FS_LAUNCH_CHECK)
extern unsigned long long g_fs_kernel_launches;

#define FS_LAUNCH_CHECK()                                                     \
  do {                                                                        \
    __atomic_fetch_add(&g_fs_kernel_launches, 1ull, __ATOMIC_RELAXED);        \
    cudaError_t e_ = cudaGetLastError();                                      \
    if (e_ != cudaSuccess) {                                                  \
      fprintf(stderr, "filsim_gpu: launch failed: %s (%s:%d)\n",             \
              cudaGetErrorString(e_), __FILE__, __LINE__);                    \
      return FS_ERR_CUDA;                                                     \
    }                                                                         \
  } while (0)

#define FS_TRY(call)                   \
  do {                                 \
    fs_status s_ = (call);             \
    if (s_ != FS_OK) return s_;        \
  } while (0)

static inline int fs_blocks(long long n, int threads) { return (int)((n + threads - 1) / threads); }

// ---- stage timing (fs_capi.cu) ----
int prof_begin(fs_ctx *c, int stage);
void prof_end(fs_ctx *c, int slot);
void prof_flush(fs_ctx *c);
struct ProfScope {
  fs_ctx *c;
  int slot;
  ProfScope(fs_ctx *ctx, int stage) : c(ctx), slot(prof_begin(ctx, stage)) {}
  ~ProfScope() { prof_end(c, slot); }
};

// ---- entry points implemented across the .cu files (internal C++ linkage) ----
fs_status fs_sort_alloc(fs_sort *s, int nkeys, int max_items, size_t *bytes);
void fs_sort_free(fs_sort *s);
fs_status fs_sort_run(fs_sort *s, int n, cudaStream_t st);  // keys in s->key must be set

fs_status fcm_init(fs_ctx *c);
void fcm_free(fs_ctx *c);
fs_status fcm_mobility(fs_ctx *c, const double *Y, const double *F, const double *T, double *V, double *W, int np);
fs_status fcm_friction(fs_ctx *c, const double *F, const double *T, double *V, double *W, int np);
fs_status fcm_flow_solve_only(fs_ctx *c, const double *f, double *u);
fs_status fcm_spread_only(fs_ctx *c, const double *Y, const double *F, const double *T, int np, double *f);
fs_status fcm_interpolate_only(fs_ctx *c, const double *u, const double *Y, int np, double *V, double *W);
void slab_free(fs_ctx *c);

bool fft32_supported(const fs_ctx *c);
fs_status fft32_init(fs_ctx *c);
void fft32_free(fs_ctx *c);
fs_status fft32_flow_solve(fs_ctx *c);

fs_status cells_init(fs_ctx *c);
void cells_free(fs_ctx *c);
fs_status cells_link(fs_ctx *c, const double *Xs, int np);
fs_status cells_barrier(fs_ctx *c, const double *Y, double *F, int np, int nt, const int *fil_id, const int *seg_id,
                        int *pairs_d, int max_pairs, int *npairs_h, int mode = FS_BARRIER_ALL);

fs_status fil_initial_guess(fs_ctx *c);
fs_status fil_forces(fs_ctx *c, int nt);
fs_status fil_jacobian_build(fs_ctx *c, int nt, const int *keep = nullptr);
fs_status fil_jacobian_prepare(fs_ctx *c);  // after an upload: kernel attributes for the filament lengths
int fil_aux_size(int nw);
fs_status fil_jacobian_inverse(fs_ctx *c, int f, double *out_d);
fs_status fil_error_check(fs_ctx *c, const double *V, const double *W, double *err, int nt);
fs_status fil_broyden_apply(fs_ctx *c, const double *b, double *x, int iter, const int *iter_d = nullptr,
                            const int *off_d = nullptr);
fs_status fil_broyden_update(fs_ctx *c, int iter, const int *iter_d = nullptr, const int *off_d = nullptr);
fs_status fil_state_update(fs_ctx *c, const double *upd);
fs_status fil_step(fs_ctx *c, int nt);
fs_status fil_max_abs_err(fs_ctx *c, const double *err, double *out_h);

fs_status fcm_set_stream(fs_ctx *c, cudaStream_t st);  // creates the cuFFT plans the precision needs, binds them
fs_status step_barrier_mobility(fs_ctx *c, int nt);     // collision barrier + FCM (or friction) solve

// ---- graph-captured steps (fs_graph.cu) ----
bool graph_steady(const fs_ctx *c, int nt);
fs_status graph_launch_step(fs_ctx *c, int nt);
fs_status graph_flush(fs_ctx *c, int *iters_h);
void graph_invalidate(fs_ctx *c);
void graph_free(fs_ctx *c);

// ---- learned warm start (fs_mlp.cu) ----
fs_status learn_prepare_capture(fs_ctx *c);
bool learn_active(const fs_ctx *c);
bool learn_gate_choose(fs_ctx *c);
bool learn_gate_on(const fs_ctx *c);
void learn_gate_record(fs_ctx *c, bool learned, long long solves);
bool learn_recording(const fs_ctx *c);
fs_status learn_save_guess(fs_ctx *c);
fs_status learn_warm_start(fs_ctx *c, int nt, fs_status (*solve)(fs_ctx *, int));
fs_status learn_diag_apply(fs_ctx *c, const double *b, double *x);
fs_status learn_capture_targets(fs_ctx *c, int iters);
fs_status learn_end_step(fs_ctx *c);
// velocity predictor (fs_start.cu): the predicted update before a step's first
// residual; the shift of the velocity history after a committed step
fs_status vpred_step(fs_ctx *c, int nt);
fs_status vpred_end_step(fs_ctx *c);
void vpred_free(fs_ctx *c);
bool hist_wanted(const fs_ctx *c);
fs_status hist_ensure(fs_ctx *c);
void hist_free(fs_ctx *c);
fs_status hist_end_step(fs_ctx *c);
fs_status hist_before_upload(fs_ctx *c, bool same_layout);
fs_status hist_after_upload(fs_ctx *c);
// Broyden memory (fs_bmem.cu). Device state: BM_NCOL history columns in use
// (carried and this step's); BM_MOVE, BM_SRC the last carry's moved columns and
// first source; BM_KEEPJ nonzero: the step keeps the previous J0; BM_SKIPJ
// nonzero: the Jacobian build inside the iteration skips (zero at a restart);
// BM_CARRIED nonzero while the step runs on carried columns or a kept J0.
enum { BM_NCOL = 0, BM_MOVE, BM_SRC, BM_KEEPJ, BM_SKIPJ, BM_CARRIED, BM_COUNT = 8 };
// with the memory on the Broyden kernels take their column count from BM_NCOL
inline const int *bmem_off(const fs_ctx *c) { return c->bmem_cols > 0 ? c->bmem_d + BM_NCOL : nullptr; }
inline const int *bmem_keep(const fs_ctx *c) { return c->bmem_cols > 0 ? c->bmem_d + BM_KEEPJ : nullptr; }
// per iteration: the restart check (and J0 build at a restart) before the apply;
// the column count after the history update
fs_status bmem_iter_begin(fs_ctx *c, int nt, int iter, const int *iter_d);
fs_status bmem_iter_end(fs_ctx *c);
// after a committed step of its (its_d: on the device) iterations: the carry
fs_status bmem_end_step(fs_ctx *c, int its, const int *its_d);
fs_status bmem_reset(fs_ctx *c);
void bmem_free(fs_ctx *c);
// an upload that changes X or Xt drops the carried state (device side, k_hist_same)
__device__ inline void bmem_drop(int *m) { m[BM_NCOL] = m[BM_KEEPJ] = m[BM_CARRIED] = 0; }
fs_status learn_before_upload(fs_ctx *c, bool same_layout);
void mlp_free(fs_ctx *c);

// ordered bit patterns for atomicMin/Max on non-negative doubles
__device__ __forceinline__ unsigned long long fs_dbits(double x) { return (unsigned long long)__double_as_longlong(x); }
