// fs_capi.cu -- the extern "C" boundary of libfilsim_gpu and the implicit
// time-step driver (the loop body of main.cpp:284-754) that sequences the
// kernels on the context's stream. Host code here allocates, validates and
// launches; all arithmetic on bead and grid data runs in the sm_100a kernels.
#include <stdlib.h>
#include <algorithm>
#include <cmath>
#include <vector>
#include "fs_internal.cuh"

unsigned long long g_fs_kernel_launches = 0;

int prof_begin(fs_ctx *c, int stage) {
  if (!c->prof.on) return -1;
  if (c->prof.n == FS_PROF_SLOTS) prof_flush(c);
  const int s = c->prof.n++;
  c->prof.stage[s] = stage;
  cudaEventRecord(c->prof.ev[2 * s], c->stream);
  return s;
}

void prof_end(fs_ctx *c, int slot) {
  if (slot >= 0) cudaEventRecord(c->prof.ev[2 * slot + 1], c->stream);
}

void prof_flush(fs_ctx *c) {
  if (!c->prof.n) return;
  cudaStreamSynchronize(c->stream);
  for (int i = 0; i < c->prof.n; ++i) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c->prof.ev[2 * i], c->prof.ev[2 * i + 1]) == cudaSuccess) {
      c->prof.ms[c->prof.stage[i]] += ms;
      c->prof.calls[c->prof.stage[i]]++;
    }
  }
  c->prof.n = 0;
}

namespace {

fs_status validate_params(const fs_params *p) {
  const int n[3] = {p->npts_x, p->npts_y, p->npts_z};
  for (int d = 0; d < 3; ++d)
    if (n[d] < FS_TILE || n[d] % FS_TILE != 0) return FS_ERR_INVALID_ARG;  // grids are whole 16^3 tiles
  if (p->ngd < 2 || p->ngd > FS_NGD_MAX) return FS_ERR_INVALID_ARG;
  for (int d = 0; d < 3; ++d)
    if (n[d] < p->ngd) return FS_ERR_INVALID_ARG;  // a stencil never wraps onto itself
  if (!(p->dx > 0) || !(p->a > 0) || !(p->mu > 0) || !(p->sigma > 0) || !(p->sigma_dip > 0)) return FS_ERR_INVALID_ARG;
  if (!(p->cell_width > 0) || !(p->dt > 0) || !(p->dl > 0)) return FS_ERR_INVALID_ARG;
  if (p->broyden_maxiter < 1 || p->broyden_maxiter > 100000) return FS_ERR_INVALID_ARG;
  if (p->precision != FS_PREC_FP64 && p->precision != FS_PREC_FP32) return FS_ERR_INVALID_ARG;
  return FS_OK;
}

fs_status alloc_state(fs_ctx *c) {
  const size_t nb = (size_t)(c->max_beads > 0 ? c->max_beads : 1);
  const size_t nf = (size_t)(c->max_fil > 0 ? c->max_fil : 1);
  double **b3[] = {&c->X, &c->Xs, &c->Xt, &c->U, &c->Us, &c->Ut, &c->F, &c->TAU, &c->Y, &c->V, &c->W,
                   &c->lam, &c->lam1, &c->lam2};
  for (double **pp : b3) FS_CUDA(cudaMalloc(pp, sizeof(double) * 3 * nb));
  double **b4[] = {&c->q, &c->qs, &c->qt};
  for (double **pp : b4) FS_CUDA(cudaMalloc(pp, sizeof(double) * 4 * nb));
  double **b6[] = {&c->err, &c->newerr, &c->upd, &c->tmp, &c->dE};
  for (double **pp : b6) FS_CUDA(cudaMalloc(pp, sizeof(double) * 6 * nb));
  FS_CUDA(cudaMalloc(&c->kap, sizeof(double) * nf));
  FS_CUDA(cudaMalloc(&c->cc, sizeof(double) * nf));
  FS_CUDA(cudaMalloc(&c->fil_start, sizeof(int) * (nf + 1)));
  FS_CUDA(cudaMalloc(&c->fil_id, sizeof(int) * nb));
  FS_CUDA(cudaMalloc(&c->seg_id, sizeof(int) * nb));
  FS_CUDA(cudaMalloc(&c->soff, sizeof(long long) * (nf + 1)));
  FS_CUDA(cudaMalloc(&c->aoff, sizeof(long long) * (nf + 1)));
  const size_t hist = (size_t)c->p.broyden_maxiter * 6 * nb;
  FS_CUDA(cudaMalloc(&c->Cmat, sizeof(double) * hist));
  FS_CUDA(cudaMalloc(&c->Dmat, sizeof(double) * hist));
  FS_CUDA(cudaMalloc(&c->dots, sizeof(double) * c->p.broyden_maxiter));
  FS_CUDA(cudaMalloc(&c->partials, sizeof(double) * (size_t)c->p.broyden_maxiter * 296));
  FS_CUDA(cudaMalloc(&c->scalars, sizeof(double) * 8));
  FS_CUDA(cudaMalloc(&c->flags, sizeof(int) * FLAG_COUNT));
  FS_CUDA(cudaMemset(c->flags, 0, sizeof(int) * FLAG_COUNT));
  FS_CUDA(cudaMalloc(&c->maxerr_bits, sizeof(unsigned long long)));
  FS_CUDA(cudaHostAlloc(&c->flags_h, sizeof(int) * FLAG_COUNT, cudaHostAllocDefault));
  c->bytes += sizeof(double) * nb * (3 * 14 + 4 * 3 + 6 * 5) + sizeof(double) * 2 * hist +
              sizeof(int) * nb * 8 + sizeof(double) * (size_t)c->p.broyden_maxiter * 297;
  return FS_OK;
}

void free_state(fs_ctx *c) {
  void *ptrs[] = {c->X, c->Xs, c->Xt, c->U, c->Us, c->Ut, c->F, c->TAU, c->Y, c->V, c->W, c->lam, c->lam1,
                  c->lam2, c->q, c->qs, c->qt, c->err, c->newerr, c->upd, c->tmp, c->dE, c->kap, c->cc,
                  c->fil_start, c->fil_id, c->seg_id, c->soff, c->aoff, c->Cmat, c->Dmat, c->dots, c->partials,
                  c->scalars, c->flags, c->maxerr_bits, c->Sinv, c->aux, c->swim, c->spring_beads,
                  c->spring_off, c->spring_ent};
  for (void *p : ptrs) cudaFree(p);
  if (c->flags_h) cudaFreeHost(c->flags_h);
}

fs_status read_flags(fs_ctx *c) {
  FS_CUDA(cudaMemcpyAsync(c->flags_h, c->flags, sizeof(int) * FLAG_COUNT, cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaStreamSynchronize(c->stream));
  prof_flush(c);
  if (c->flags_h[FLAG_NONFINITE]) c->diag.nonfinite = 1;
  if (c->flags_h[FLAG_EXPLODE]) c->diag.explosion = 1;
  if (c->flags_h[FLAG_CAPACITY]) return FS_ERR_CAPACITY;
  return FS_OK;
}

fs_status barrier_and_mobility(fs_ctx *c, int nt) {
  if (c->barrier_mode != FS_BARRIER_OFF)
    FS_TRY(cells_barrier(c, c->Y, c->F, c->np, nt, c->fil_id, c->seg_id, nullptr, 0, nullptr, c->barrier_mode));
  if (nt > c->p.initial_friction_steps)
    FS_TRY(fcm_mobility(c, c->Y, c->F, c->TAU, c->V, c->W, c->np));
  else
    FS_TRY(fcm_friction(c, c->F, c->TAU, c->V, c->W, c->np));
  c->diag.mobility_solves++;
  return FS_OK;
}

}  // namespace

fs_status step_barrier_mobility(fs_ctx *c, int nt) { return barrier_and_mobility(c, nt); }

namespace {

// one implicit step (main.cpp:334-707); commit = false leaves out Filament::step
// (the gait-reset driver's trial solves); choice: the cost gate's start when the
// caller has already asked it (0 plain, 1 learned), -1 to ask here
fs_status step_implicit(fs_ctx *c, int nt, int *iters_out, bool commit = true, int choice = -1) {
  FS_TRY(fil_initial_guess(c));
  const bool learn_on = learn_active(c) && nt > c->p.initial_friction_steps;
  const bool learned = learn_on && (choice >= 0 ? choice == 1 : learn_gate_choose(c));
  const long long solves0 = c->diag.mobility_solves;
  if (learned || learn_recording(c)) FS_TRY(learn_save_guess(c));
  FS_TRY(fil_forces(c, nt));
  FS_TRY(fil_jacobian_build(c, nt, bmem_keep(c)));
  FS_TRY(cells_link(c, c->Xs, c->np));
  if (!learned) FS_TRY(vpred_step(c, nt));
  if (learned) {
    FS_TRY(learn_warm_start(c, nt, barrier_and_mobility));
  } else {
    FS_TRY(barrier_and_mobility(c, nt));
    FS_TRY(fil_error_check(c, c->V, c->W, c->err, nt));
  }
  FS_TRY(read_flags(c));
  if (c->flags_h[FLAG_PIVOT]) return FS_ERR_NONFINITE;
  int check = c->flags_h[FLAG_CHECK];
  int iter = 0;
  // precision escalation: an FP32 step past escalate_after iterations finishes in FP64
  struct Precision {
    fs_ctx *c;
    int prec;
    ~Precision() {
      if (c->precision != prec) {
        c->precision = prec;
        fcm_set_stream(c, c->stream);
      }
    }
  } restore{c, c->precision};
  const int esc = (c->precision == FS_PREC_FP32 && c->escalate_after > 0) ? c->escalate_after : 0;
  while (check && iter < c->p.broyden_maxiter) {
    if (esc > 0 && iter == esc) {
      c->precision = FS_PREC_FP64;
      FS_TRY(fcm_set_stream(c, c->stream));
    }
    if (c->precision != restore.prec) c->diag.escalated_iters++;
    // with the Broyden memory on the column count lives on the device
    const int *off = bmem_off(c);
    const int hit = off ? 0 : iter;
    FS_TRY(bmem_iter_begin(c, nt, iter, nullptr));
    FS_TRY(fil_broyden_apply(c, c->err, c->upd, hit, nullptr, off));
    FS_TRY(fil_state_update(c, c->upd));
    FS_TRY(fil_forces(c, nt));
    FS_TRY(barrier_and_mobility(c, nt));
    FS_TRY(fil_error_check(c, c->V, c->W, c->newerr, nt));
    FS_TRY(fil_broyden_update(c, hit, nullptr, off));
    FS_TRY(bmem_iter_end(c));
    std::swap(c->err, c->newerr);
    ++iter;
    FS_TRY(read_flags(c));
    if (c->flags_h[FLAG_PIVOT]) return FS_ERR_NONFINITE;  // a J0 built at a memory restart
    check = c->flags_h[FLAG_CHECK];
  }
  if (learn_recording(c)) FS_TRY(learn_capture_targets(c, iter));
  if (learn_on) learn_gate_record(c, learned, c->diag.mobility_solves - solves0);
  FS_TRY(learn_end_step(c));
  if (commit) {
    FS_TRY(hist_end_step(c));  // only a step that moves X to Xt shifts the history
    FS_TRY(bmem_end_step(c, iter, nullptr));  // and carries Broyden columns
    FS_TRY(vpred_end_step(c));
    FS_TRY(fil_step(c, nt));
  }
  c->diag.last_nt = nt;
  c->diag.last_iters = iter;
  c->diag.total_iters += iter;
  if (check) c->diag.not_converged_steps++;
  if (iters_out) *iters_out = iter;
  return FS_OK;
}

}  // namespace

extern "C" {

int fs_abi_version(void) { return FS_ABI_VERSION; }

unsigned long long fs_kernel_launches(void) { return __atomic_load_n(&g_fs_kernel_launches, __ATOMIC_RELAXED); }

const char *fs_status_string(fs_status s) {
  switch (s) {
    case FS_OK: return "ok";
    case FS_ERR_INVALID_ARG: return "invalid argument";
    case FS_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case FS_ERR_CUDA: return "CUDA runtime error";
    case FS_ERR_CUFFT: return "cuFFT error";
    case FS_ERR_OOM: return "device allocation failed";
    case FS_ERR_NOT_CONVERGED: return "Broyden iteration reached broyden_maxiter";
    case FS_ERR_NONFINITE: return "non-finite residual or singular Jacobian";
    case FS_ERR_CAPACITY: return "internal list capacity exceeded";
    case FS_ERR_STATE: return "call order violated";
    case FS_ERR_IO: return "file could not be opened, written or parsed";
    default: return "unknown status";
  }
}

void fs_params_default(fs_params *p, int nx, int ny, int nz) {
  memset(p, 0, sizeof *p);
  const double PI = FS_PI;
  p->npts_x = nx;
  p->npts_y = ny;
  p->npts_z = nz;
  p->ngd = 12;
  p->a = 1.0;
  p->ah = 1.0;
  p->mu = 1.0;
  p->sigma_dip = p->a / pow(36.0 * PI, 1.0 / 6.0);
  p->sigma = p->a / sqrt(PI);
  p->dx = p->sigma_dip / 1.5;
  p->dl = 2.2 * p->a;
  p->dt = 0.05;
  p->tol = 1e-6;
  p->broyden_maxiter = 300;
  p->impl_euler_steps = 1;
  p->initial_friction_steps = 0;
  p->precision = FS_PREC_FP64;
  p->barrier_fs_over_2a = 15 * PI;
  p->barrier_distance_cap = 2.0;
  p->cell_width = 2.5 * p->a;
  p->lambda_extrap_step = 12;
}

fs_status fs_create(const fs_params *p, int max_beads, int max_filaments, void *stream, fs_ctx **out) {
  if (!p || !out || max_beads < 0 || max_filaments < 0) return FS_ERR_INVALID_ARG;
  *out = nullptr;
  FS_TRY(validate_params(p));
  int dev = 0, ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return FS_ERR_NO_DEVICE;
  }
  FS_CUDA(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  FS_CUDA(cudaGetDeviceProperties(&prop, dev));
  if (prop.major != 10) return FS_ERR_NO_DEVICE;
  fs_ctx *c = (fs_ctx *)calloc(1, sizeof(fs_ctx));
  if (!c) return FS_ERR_OOM;
  c->p = *p;
  c->device = dev;
  c->num_sms = prop.multiProcessorCount;
  c->max_beads = max_beads;
  c->max_fil = max_filaments;
  c->precision = p->precision;
  c->start_order = 1;
  c->tension_order = 2;
  c->L[0] = p->npts_x * p->dx;
  c->L[1] = p->npts_y * p->dx;
  c->L[2] = p->npts_z * p->dx;
  fs_status st = FS_OK;
  if (stream) {
    c->stream = (cudaStream_t)stream;
  } else {
    // a blocking stream: work on it is ordered against the legacy default
    // stream, which callers' own copies (and torch's) use
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault) != cudaSuccess) st = FS_ERR_CUDA;
    c->own_stream = true;
  }
  if (st == FS_OK) st = alloc_state(c);
  if (st == FS_OK) st = fcm_init(c);
  if (st == FS_OK) st = cells_init(c);
  if (st == FS_OK && cudaStreamSynchronize(c->stream) != cudaSuccess) st = FS_ERR_CUDA;
  if (st != FS_OK) {
    fs_destroy(c);
    return st;
  }
  *out = c;
  return FS_OK;
}

fs_status fs_profile_enable(fs_ctx *c, int on) {
  if (!c) return FS_ERR_INVALID_ARG;
  if (on && !c->prof.created) {
    for (int i = 0; i < 2 * FS_PROF_SLOTS; ++i) FS_CUDA(cudaEventCreate(&c->prof.ev[i]));
    c->prof.created = true;
  }
  prof_flush(c);
  memset(c->prof.ms, 0, sizeof c->prof.ms);
  memset(c->prof.calls, 0, sizeof c->prof.calls);
  c->prof.on = on != 0;
  return FS_OK;
}

fs_status fs_profile_get(fs_ctx *c, fs_profile *out) {
  if (!c || !out) return FS_ERR_INVALID_ARG;
  prof_flush(c);
  FS_CUDA(cudaStreamSynchronize(c->stream));
  memcpy(out->ms, c->prof.ms, sizeof out->ms);
  memcpy(out->calls, c->prof.calls, sizeof out->calls);
  return FS_OK;
}

fs_status fs_destroy(fs_ctx *c) {
  if (!c) return FS_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->prof.created)
    for (int i = 0; i < 2 * FS_PROF_SLOTS; ++i) cudaEventDestroy(c->prof.ev[i]);
  graph_free(c);
  mlp_free(c);
  hist_free(c);
  bmem_free(c);
  vpred_free(c);
  cudaFree(c->gemm_err);
  fcm_free(c);
  slab_free(c);
  cells_free(c);
  free_state(c);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  free(c->fil_start_h);
  free(c);
  return FS_OK;
}

fs_status fs_get_params(const fs_ctx *c, fs_params *p_h) {
  if (!c || !p_h) return FS_ERR_INVALID_ARG;
  *p_h = c->p;
  p_h->precision = c->precision;
  return FS_OK;
}

fs_status fs_set_precision(fs_ctx *c, int precision) {
  if (!c || (precision != FS_PREC_FP64 && precision != FS_PREC_FP32)) return FS_ERR_INVALID_ARG;
  if (precision != c->precision) graph_invalidate(c);
  c->precision = precision;
  return FS_OK;
}

fs_status fs_synchronize(fs_ctx *c) {
  if (!c) return FS_ERR_INVALID_ARG;
  FS_CUDA(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_device_bytes(const fs_ctx *c, size_t *bytes_h) {
  if (!c || !bytes_h) return FS_ERR_INVALID_ARG;
  *bytes_h = c->bytes;
  return FS_OK;
}

fs_status fs_fcm_mobility(fs_ctx *c, const double *Y, const double *F, const double *T, double *V, double *W,
                          int np) {
  if (!c || np < 0 || np > c->max_beads || (np > 0 && (!Y || !F || !T || !V || !W))) return FS_ERR_INVALID_ARG;
  return fcm_mobility(c, Y, F, T, V, W, np);
}

fs_status fs_fcm_mobility_host(fs_ctx *c, const double *Y_h, const double *F_h, const double *T_h, double *V_h,
                               double *W_h, int np) {
  if (!c || np < 0 || np > c->max_beads || (np > 0 && (!Y_h || !F_h || !T_h || !V_h || !W_h)))
    return FS_ERR_INVALID_ARG;
  const size_t bytes = sizeof(double) * 3 * (size_t)np;
  // the context's own bead buffers stage the call
  FS_CUDA(cudaMemcpyAsync(c->Y, Y_h, bytes, cudaMemcpyHostToDevice, c->stream));
  FS_CUDA(cudaMemcpyAsync(c->F, F_h, bytes, cudaMemcpyHostToDevice, c->stream));
  FS_CUDA(cudaMemcpyAsync(c->TAU, T_h, bytes, cudaMemcpyHostToDevice, c->stream));
  FS_TRY(fcm_mobility(c, c->Y, c->F, c->TAU, c->V, c->W, np));
  FS_CUDA(cudaMemcpyAsync(V_h, c->V, bytes, cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaMemcpyAsync(W_h, c->W, bytes, cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_fcm_friction(fs_ctx *c, const double *F, const double *T, double *V, double *W, int np) {
  if (!c || np < 0 || (np > 0 && (!F || !T || !V || !W))) return FS_ERR_INVALID_ARG;
  return fcm_friction(c, F, T, V, W, np);
}

fs_status fs_fcm_spread(fs_ctx *c, const double *Y, const double *F, const double *T, int np, double *f) {
  if (!c || np < 0 || np > c->max_beads || !f || (np > 0 && (!Y || !F || !T))) return FS_ERR_INVALID_ARG;
  return fcm_spread_only(c, Y, F, T, np, f);
}

fs_status fs_fcm_get_grid(fs_ctx *c, double *grid_h, size_t count) {
  if (!c || !grid_h || count < 3 * c->N) return FS_ERR_INVALID_ARG;
  if (c->last_grid_prec != FS_PREC_FP64) return FS_ERR_STATE;
  FS_CUDA(cudaMemcpyAsync(grid_h, c->grid_real, sizeof(double) * 3 * c->N, cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_fcm_flow_solve(fs_ctx *c, const double *f, double *u) {
  if (!c || !f || !u) return FS_ERR_INVALID_ARG;
  return fcm_flow_solve_only(c, f, u);
}

fs_status fs_cells_dims(const fs_ctx *c, int *mxyz_h) {
  if (!c || !mxyz_h) return FS_ERR_INVALID_ARG;
  for (int d = 0; d < 3; ++d) mxyz_h[d] = c->M[d];
  return FS_OK;
}

fs_status fs_cells_link(fs_ctx *c, const double *Xs, int np) {
  if (!c || np < 0 || np > c->max_beads || (np > 0 && !Xs)) return FS_ERR_INVALID_ARG;
  FS_CUDA(cudaMemsetAsync(c->flags + FLAG_CAPACITY, 0, sizeof(int), c->stream));
  FS_TRY(cells_link(c, Xs, np));
  // a cell of 4096 beads or more does not fit the barrier's visiting-order key
  int cap = 0;
  FS_CUDA(cudaMemcpyAsync(&cap, c->flags + FLAG_CAPACITY, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaStreamSynchronize(c->stream));
  return cap ? FS_ERR_CAPACITY : FS_OK;
}

fs_status fs_cells_get_lists(fs_ctx *c, int *head_h, int *list_h, int *map_h) {
  if (!c) return FS_ERR_INVALID_ARG;
  if (c->cells_np < 0) return FS_ERR_STATE;
  if (head_h) FS_CUDA(cudaMemcpyAsync(head_h, c->head, sizeof(int) * c->ncell, cudaMemcpyDeviceToHost, c->stream));
  if (list_h && c->cells_np > 0)
    FS_CUDA(cudaMemcpyAsync(list_h, c->list, sizeof(int) * c->cells_np, cudaMemcpyDeviceToHost, c->stream));
  if (map_h) FS_CUDA(cudaMemcpyAsync(map_h, c->map, sizeof(int) * 13 * (size_t)c->ncell, cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

static fs_status resolve_ids(fs_ctx *c, int np, const int **fil_id, const int **seg_id) {
  if (*fil_id && *seg_id) return FS_OK;
  if (*fil_id || *seg_id) return FS_ERR_INVALID_ARG;
  if (!c->have_state || c->np != np) return FS_ERR_STATE;
  *fil_id = c->fil_id;
  *seg_id = c->seg_id;
  return FS_OK;
}

fs_status fs_collision_barrier(fs_ctx *c, const double *Y, double *F_inout, int np, int nt, const int *fil_id,
                               const int *seg_id, double *min_dist2_h) {
  if (!c || np < 0 || (np > 0 && (!Y || !F_inout))) return FS_ERR_INVALID_ARG;
  FS_TRY(resolve_ids(c, np, &fil_id, &seg_id));
  FS_TRY(cells_barrier(c, Y, F_inout, np, nt, fil_id, seg_id, nullptr, 0, nullptr));
  int cap = 0;
  unsigned long long bits;
  FS_CUDA(cudaMemcpyAsync(&cap, c->flags + FLAG_CAPACITY, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  if (min_dist2_h)
    FS_CUDA(cudaMemcpyAsync(&bits, c->min_dist2_bits, sizeof bits, cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaStreamSynchronize(c->stream));
  if (min_dist2_h) {
    memcpy(min_dist2_h, &bits, sizeof bits);
    c->diag.min_dist2 = *min_dist2_h;
  }
  return cap ? FS_ERR_CAPACITY : FS_OK;
}

fs_status fs_collision_pairs(fs_ctx *c, const double *Y, int np, int nt, const int *fil_id, const int *seg_id,
                             int *pairs_h, int max_pairs, int *npairs_h) {
  if (!c || np < 0 || !npairs_h || max_pairs < 0 || (max_pairs > 0 && !pairs_h) || (np > 0 && !Y))
    return FS_ERR_INVALID_ARG;
  FS_TRY(resolve_ids(c, np, &fil_id, &seg_id));
  int *pairs_d = nullptr;
  if (max_pairs > 0) FS_CUDA(cudaMalloc(&pairs_d, sizeof(int) * 2 * (size_t)max_pairs));
  fs_status st = cells_barrier(c, Y, nullptr, np, nt, fil_id, seg_id, pairs_d, max_pairs, npairs_h);
  if (st == FS_OK && max_pairs > 0) {
    int n = *npairs_h < max_pairs ? *npairs_h : max_pairs;
    if (n > 0 && cudaMemcpy(pairs_h, pairs_d, sizeof(int) * 2 * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess)
      st = FS_ERR_CUDA;
  }
  cudaFree(pairs_d);
  return st;
}

static fs_status upload_layout(fs_ctx *c, const fs_host_state *s);
static void spring_free(fs_ctx *c);
static void swim_free(fs_ctx *c);

// state arrays always; the filament layout (ids, offsets, Schur buffers) only
// when it differs from the previous upload's
fs_status fs_state_upload(fs_ctx *c, const fs_host_state *s) {
  if (!c || !s || !s->fil_start || s->nfil < 0 || s->np < 0) return FS_ERR_INVALID_ARG;
  if (s->np > c->max_beads || s->nfil > c->max_fil) return FS_ERR_INVALID_ARG;
  const int nf = s->nfil, np = s->np;
  if (s->fil_start[0] != 0 || s->fil_start[nf] != np) return FS_ERR_INVALID_ARG;
  cudaStream_t st = c->stream;
  const bool same_layout = c->have_state && c->fil_start_h && c->nfil == nf && c->np == np &&
                           memcmp(c->fil_start_h, s->fil_start, sizeof(int) * (nf + 1)) == 0;
  FS_TRY(learn_before_upload(c, same_layout));
  FS_TRY(hist_before_upload(c, same_layout));
  if (!same_layout) {
    graph_invalidate(c);
    FS_CUDA(cudaStreamSynchronize(st));
    // a swimming drive and spring links refer to the previous layout's filaments and beads
    swim_free(c);
    spring_free(c);
    FS_TRY(upload_layout(c, s));
  }
  struct F3 {
    double *d;
    const double *h;
    size_t n;
  } fields[] = {{c->X, s->X, 3}, {c->Xs, s->Xs, 3}, {c->Xt, s->Xt, 3}, {c->U, s->U, 3}, {c->Us, s->Us, 3},
                {c->Ut, s->Ut, 3}, {c->q, s->q, 4}, {c->qs, s->qs, 4}, {c->qt, s->qt, 4}, {c->F, s->F, 3},
                {c->TAU, s->TAU, 3}};
  for (auto &fl : fields) {
    if (fl.h) FS_CUDA(cudaMemcpyAsync(fl.d, fl.h, sizeof(double) * fl.n * np, cudaMemcpyHostToDevice, st));
    else FS_CUDA(cudaMemsetAsync(fl.d, 0, sizeof(double) * fl.n * np, st));
  }
  const size_t nl3 = sizeof(double) * 3 * (size_t)c->nlink;
  double *lams[] = {c->lam, c->lam1, c->lam2};
  double *lams_h[] = {s->lam, s->lam1, s->lam2};
  for (int i = 0; i < 3; ++i) {
    if (lams_h[i]) FS_CUDA(cudaMemcpyAsync(lams[i], lams_h[i], nl3, cudaMemcpyHostToDevice, st));
    else FS_CUDA(cudaMemsetAsync(lams[i], 0, nl3, st));
  }
  FS_TRY(hist_after_upload(c));
  if (s->kap) FS_CUDA(cudaMemcpyAsync(c->kap, s->kap, sizeof(double) * nf, cudaMemcpyHostToDevice, st));
  if (s->c) FS_CUDA(cudaMemcpyAsync(c->cc, s->c, sizeof(double) * nf, cudaMemcpyHostToDevice, st));
  if (!same_layout || !s->kap || !s->c) {
    std::vector<double> ones(nf > 0 ? nf : 1, 1.0);
    if (!s->kap) FS_CUDA(cudaMemcpyAsync(c->kap, ones.data(), sizeof(double) * nf, cudaMemcpyHostToDevice, st));
    if (!s->c) FS_CUDA(cudaMemcpyAsync(c->cc, ones.data(), sizeof(double) * nf, cudaMemcpyHostToDevice, st));
    FS_CUDA(cudaStreamSynchronize(st));
  } else {
    FS_CUDA(cudaStreamSynchronize(st));
  }
  c->have_state = true;
  return FS_OK;
}

// the filament layout of an upload: ids, offsets, Schur buffers (fs_state_upload)
static fs_status upload_layout(fs_ctx *c, const fs_host_state *s) {
  const int nf = s->nfil, np = s->np;
  std::vector<int> fid(np > 0 ? np : 1), sid(np > 0 ? np : 1);
  std::vector<long long> soff(nf + 1), aoff(nf + 1);
  int max_nw = 1, min_nw = nf > 0 ? 1 << 30 : 1;
  soff[0] = aoff[0] = 0;
  for (int f = 0; f < nf; ++f) {
    const int nw = s->fil_start[f + 1] - s->fil_start[f];
    if (nw < 1) return FS_ERR_INVALID_ARG;
    max_nw = std::max(max_nw, nw);
    min_nw = std::min(min_nw, nw);
    for (int i = 0; i < nw; ++i) {
      fid[s->fil_start[f] + i] = f;
      sid[s->fil_start[f] + i] = i;
    }
    soff[f + 1] = soff[f] + 9LL * nw * nw;
    aoff[f + 1] = aoff[f] + fil_aux_size(nw);
  }
  const int prev_max_nw = c->max_nw;
  c->max_nw = max_nw;
  if (fil_jacobian_prepare(c) != FS_OK) {  // the Schur complement of a filament lives in shared memory
    c->max_nw = prev_max_nw;
    return FS_ERR_INVALID_ARG;
  }
  c->min_nw = min_nw;
  c->nfil = nf;
  c->np = np;
  c->nlink = np - nf;
  cudaFree(c->Sinv);
  cudaFree(c->aux);
  c->Sinv = c->aux = nullptr;
  FS_CUDA(cudaMalloc(&c->Sinv, sizeof(double) * (size_t)(soff[nf] > 0 ? soff[nf] : 1)));
  FS_CUDA(cudaMalloc(&c->aux, sizeof(double) * (size_t)(aoff[nf] > 0 ? aoff[nf] : 1)));
  cudaStream_t st = c->stream;
  FS_CUDA(cudaMemcpyAsync(c->fil_start, s->fil_start, sizeof(int) * (nf + 1), cudaMemcpyHostToDevice, st));
  FS_CUDA(cudaMemcpyAsync(c->fil_id, fid.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st));
  FS_CUDA(cudaMemcpyAsync(c->seg_id, sid.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st));
  FS_CUDA(cudaMemcpyAsync(c->soff, soff.data(), sizeof(long long) * (nf + 1), cudaMemcpyHostToDevice, st));
  FS_CUDA(cudaMemcpyAsync(c->aoff, aoff.data(), sizeof(long long) * (nf + 1), cudaMemcpyHostToDevice, st));
  FS_CUDA(cudaStreamSynchronize(st));  // the host vectors above go out of scope
  free(c->fil_start_h);
  c->fil_start_h = (int *)malloc(sizeof(int) * (nf + 1));
  if (!c->fil_start_h) return FS_ERR_OOM;
  memcpy(c->fil_start_h, s->fil_start, sizeof(int) * (nf + 1));
  return FS_OK;
}

fs_status fs_state_download(fs_ctx *c, fs_host_state *s) {
  if (!c || !s) return FS_ERR_INVALID_ARG;
  if (!c->have_state || s->np != c->np || s->nfil != c->nfil) return FS_ERR_STATE;
  const int np = c->np;
  cudaStream_t st = c->stream;
  struct F3 {
    const double *d;
    double *h;
    size_t n;
  } fields[] = {{c->X, s->X, 3}, {c->Xs, s->Xs, 3}, {c->Xt, s->Xt, 3}, {c->U, s->U, 3}, {c->Us, s->Us, 3},
                {c->Ut, s->Ut, 3}, {c->q, s->q, 4}, {c->qs, s->qs, 4}, {c->qt, s->qt, 4}, {c->F, s->F, 3},
                {c->TAU, s->TAU, 3}};
  for (auto &fl : fields)
    if (fl.h) FS_CUDA(cudaMemcpyAsync(fl.h, fl.d, sizeof(double) * fl.n * np, cudaMemcpyDeviceToHost, st));
  const size_t nl3 = sizeof(double) * 3 * (size_t)c->nlink;
  if (s->lam) FS_CUDA(cudaMemcpyAsync(s->lam, c->lam, nl3, cudaMemcpyDeviceToHost, st));
  if (s->lam1) FS_CUDA(cudaMemcpyAsync(s->lam1, c->lam1, nl3, cudaMemcpyDeviceToHost, st));
  if (s->lam2) FS_CUDA(cudaMemcpyAsync(s->lam2, c->lam2, nl3, cudaMemcpyDeviceToHost, st));
  if (s->kap) FS_CUDA(cudaMemcpyAsync(s->kap, c->kap, sizeof(double) * c->nfil, cudaMemcpyDeviceToHost, st));
  if (s->c) FS_CUDA(cudaMemcpyAsync(s->c, c->cc, sizeof(double) * c->nfil, cudaMemcpyDeviceToHost, st));
  FS_CUDA(cudaStreamSynchronize(st));
  return FS_OK;
}

fs_status fs_state_device_ptr(fs_ctx *c, const char *which, double **ptr_h) {
  if (!c || !which || !ptr_h) return FS_ERR_INVALID_ARG;
  struct {
    const char *n;
    double *p;
  } tab[] = {{"Xs", c->Xs}, {"X", c->X},   {"Xt", c->Xt},   {"Us", c->Us},   {"U", c->U},   {"Ut", c->Ut},
             {"qs", c->qs}, {"q", c->q},   {"qt", c->qt},   {"F", c->F},     {"TAU", c->TAU}, {"Y", c->Y},
             {"V", c->V},   {"W", c->W},   {"lam", c->lam}, {"err", c->err}, {"update", c->upd}};
  for (auto &t : tab)
    if (!strcmp(t.n, which)) {
      *ptr_h = t.p;
      return FS_OK;
    }
  return FS_ERR_INVALID_ARG;
}

fs_status fs_initial_guess(fs_ctx *c) { return c ? fil_initial_guess(c) : FS_ERR_INVALID_ARG; }
fs_status fs_filament_forces(fs_ctx *c, int nt) { return c ? fil_forces(c, nt) : FS_ERR_INVALID_ARG; }

fs_status fs_set_swimming(fs_ctx *c, const double *swim_h, double curvature, int sperm_decay) {
  if (!c) return FS_ERR_INVALID_ARG;
  if (!c->have_state) return FS_ERR_STATE;
  graph_invalidate(c);
  FS_CUDA(cudaStreamSynchronize(c->stream));  // no queued step still reads the old parameters
  if (!swim_h) {
    swim_free(c);
    return FS_OK;
  }
  const size_t n = 5 * (size_t)c->nfil;
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(swim_h[i])) return FS_ERR_INVALID_ARG;
  if (!std::isfinite(curvature)) return FS_ERR_INVALID_ARG;
  if (!c->swim) {
    FS_CUDA(cudaMalloc(&c->swim, sizeof(double) * (n > 0 ? n : 1)));
    c->swim_bytes = sizeof(double) * n;
    c->bytes += c->swim_bytes;
  }
  FS_CUDA(cudaMemcpyAsync(c->swim, swim_h, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  FS_CUDA(cudaStreamSynchronize(c->stream));
  c->swim_curvature = curvature;
  c->swim_sperm_decay = sperm_decay ? 1 : 0;
  return FS_OK;
}

fs_status fs_set_barrier_mode(fs_ctx *c, int mode) {
  if (!c || mode < FS_BARRIER_ALL || mode > FS_BARRIER_OFF) return FS_ERR_INVALID_ARG;
  if (mode != c->barrier_mode) graph_invalidate(c);
  c->barrier_mode = mode;
  return FS_OK;
}

fs_status fs_step_gait_reset(fs_ctx *c, int nt, int *iters_h, double *vwf_h) {
  if (!c || !iters_h) return FS_ERR_INVALID_ARG;
  if (!c->have_state) return FS_ERR_STATE;
  memset(&c->diag, 0, sizeof c->diag);
  const int saved = c->barrier_mode;
  const int modes[3] = {FS_BARRIER_OFF, FS_BARRIER_NOT_SWIMMER, saved};
  const int nw0 = c->nfil > 0 ? c->fil_start_h[1] - c->fil_start_h[0] : 0;
  fs_status st = FS_OK;
  for (int pass = 0; pass < 3 && st == FS_OK; ++pass) {
    c->barrier_mode = modes[pass];
    st = step_implicit(c, nt, iters_h + pass, pass == 2);
    if (st == FS_OK && vwf_h && nw0 > 0) {
      // filament 0's beads: V, W, F of the solve (save_swimmer_velocity_data_to_file)
      std::vector<double> v(3 * (size_t)nw0), w(3 * (size_t)nw0), f(3 * (size_t)nw0);
      cudaError_t e = cudaMemcpyAsync(v.data(), c->V, sizeof(double) * 3 * nw0, cudaMemcpyDeviceToHost, c->stream);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(w.data(), c->W, sizeof(double) * 3 * nw0, cudaMemcpyDeviceToHost, c->stream);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(f.data(), c->F, sizeof(double) * 3 * nw0, cudaMemcpyDeviceToHost, c->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
      if (e != cudaSuccess) {
        st = FS_ERR_CUDA;
        break;
      }
      for (int b = 0; b < nw0; ++b)
        for (int d = 0; d < 3; ++d) {
          vwf_h[((size_t)pass * nw0 + b) * 9 + d] = v[3 * b + d];
          vwf_h[((size_t)pass * nw0 + b) * 9 + 3 + d] = w[3 * b + d];
          vwf_h[((size_t)pass * nw0 + b) * 9 + 6 + d] = f[3 * b + d];
        }
    }
  }
  c->barrier_mode = saved;
  FS_TRY(st);
  if (c->diag.nonfinite) return FS_ERR_NONFINITE;
  return c->diag.not_converged_steps ? FS_ERR_NOT_CONVERGED : FS_OK;
}

static void swim_free(fs_ctx *c) {
  cudaFree(c->swim);
  c->swim = nullptr;
  c->bytes -= c->swim_bytes;
  c->swim_bytes = 0;
}

static void spring_free(fs_ctx *c) {
  cudaFree(c->spring_beads);
  cudaFree(c->spring_off);
  cudaFree(c->spring_ent);
  c->spring_beads = c->spring_off = c->spring_ent = nullptr;
  c->nspring = 0;
  c->bytes -= c->spring_bytes;
  c->spring_bytes = 0;
}

fs_status fs_set_spring_links(fs_ctx *c, int nlinks, const int *beads_h, double k, double l0) {
  if (!c || nlinks < 0 || (nlinks > 0 && !beads_h)) return FS_ERR_INVALID_ARG;
  if (!c->have_state) return FS_ERR_STATE;
  if (!std::isfinite(k) || !std::isfinite(l0)) return FS_ERR_INVALID_ARG;
  for (int l = 0; l < nlinks; ++l) {
    const int a = beads_h[2 * l], b = beads_h[2 * l + 1];
    if (a < 0 || b < 0 || a >= c->np || b >= c->np || a == b) return FS_ERR_INVALID_ARG;
  }
  graph_invalidate(c);
  FS_CUDA(cudaStreamSynchronize(c->stream));
  spring_free(c);
  if (nlinks == 0) return FS_OK;
  // per bead, its links in link order: entry 2 l (first bead of link l) or 2 l + 1 (second)
  std::vector<int> off(c->np + 1, 0), ent(2 * (size_t)nlinks);
  for (int l = 0; l < nlinks; ++l) {
    off[beads_h[2 * l] + 1]++;
    off[beads_h[2 * l + 1] + 1]++;
  }
  for (int b = 0; b < c->np; ++b) off[b + 1] += off[b];
  std::vector<int> fill(off.begin(), off.end() - 1);
  for (int l = 0; l < nlinks; ++l) {
    ent[fill[beads_h[2 * l]]++] = 2 * l;
    ent[fill[beads_h[2 * l + 1]]++] = 2 * l + 1;
  }
  FS_CUDA(cudaMalloc(&c->spring_beads, sizeof(int) * 2 * (size_t)nlinks));
  FS_CUDA(cudaMalloc(&c->spring_off, sizeof(int) * (size_t)(c->np + 1)));
  FS_CUDA(cudaMalloc(&c->spring_ent, sizeof(int) * 2 * (size_t)nlinks));
  FS_CUDA(cudaMemcpyAsync(c->spring_beads, beads_h, sizeof(int) * 2 * (size_t)nlinks, cudaMemcpyHostToDevice,
                          c->stream));
  FS_CUDA(cudaMemcpyAsync(c->spring_off, off.data(), sizeof(int) * (size_t)(c->np + 1), cudaMemcpyHostToDevice,
                          c->stream));
  FS_CUDA(cudaMemcpyAsync(c->spring_ent, ent.data(), sizeof(int) * 2 * (size_t)nlinks, cudaMemcpyHostToDevice,
                          c->stream));
  FS_CUDA(cudaStreamSynchronize(c->stream));  // the host vectors go out of scope
  c->nspring = nlinks;
  c->spring_k = k;
  c->spring_l0 = l0;
  c->spring_bytes = sizeof(int) * (4 * (size_t)nlinks + (size_t)(c->np + 1));
  c->bytes += c->spring_bytes;
  return FS_OK;
}

fs_status fs_jacobian_build(fs_ctx *c, int nt) {
  if (!c) return FS_ERR_INVALID_ARG;
  FS_CUDA(cudaMemsetAsync(c->flags + FLAG_PIVOT, 0, sizeof(int), c->stream));
  return fil_jacobian_build(c, nt);
}

fs_status fs_jacobian_get_inverse(fs_ctx *c, int f, double *jinv_h, int n) {
  if (!c || !jinv_h || !c->have_state || f < 0 || f >= c->nfil) return FS_ERR_INVALID_ARG;
  double *out_d = nullptr;
  FS_CUDA(cudaMalloc(&out_d, sizeof(double) * (size_t)n * n));
  int fs_h[2];
  fs_status st = FS_OK;
  if (cudaMemcpy(fs_h, c->fil_start + f, 2 * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) st = FS_ERR_CUDA;
  if (st == FS_OK && 6 * (fs_h[1] - fs_h[0]) != n) st = FS_ERR_INVALID_ARG;
  if (st == FS_OK) st = fil_jacobian_inverse(c, f, out_d);
  if (st == FS_OK && cudaMemcpy(jinv_h, out_d, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToHost) != cudaSuccess)
    st = FS_ERR_CUDA;
  cudaFree(out_d);
  return st;
}

fs_status fs_error_check(fs_ctx *c, const double *V, const double *W, double *err, int nt, int *check_h) {
  if (!c || !V || !W || !err) return FS_ERR_INVALID_ARG;
  FS_TRY(fil_error_check(c, V, W, err, nt));
  FS_TRY(read_flags(c));
  if (check_h) *check_h = c->flags_h[FLAG_CHECK];
  return FS_OK;
}

fs_status fs_broyden_apply(fs_ctx *c, const double *b, double *x, int iter) {
  if (!c || !b || !x || iter < 0 || iter > c->p.broyden_maxiter) return FS_ERR_INVALID_ARG;
  return fil_broyden_apply(c, b, x, iter);
}

fs_status fs_broyden_set_cols(fs_ctx *c, const double *cc, const double *d, int iter) {
  if (!c || iter < 0 || iter >= c->p.broyden_maxiter || !c->have_state) return FS_ERR_INVALID_ARG;
  const size_t n6 = (size_t)6 * c->np;
  if (cc) FS_CUDA(cudaMemcpyAsync(c->Cmat + iter * n6, cc, sizeof(double) * n6, cudaMemcpyDeviceToDevice, c->stream));
  if (d) FS_CUDA(cudaMemcpyAsync(c->Dmat + iter * n6, d, sizeof(double) * n6, cudaMemcpyDeviceToDevice, c->stream));
  return FS_OK;
}

fs_status fs_state_update(fs_ctx *c, const double *update) {
  if (!c || !update) return FS_ERR_INVALID_ARG;
  return fil_state_update(c, update);
}

fs_status fs_step(fs_ctx *c, int nt) {
  if (!c) return FS_ERR_INVALID_ARG;
  if (!c->have_state) return FS_ERR_STATE;
  FS_TRY(learn_end_step(c));
  FS_TRY(hist_end_step(c));
  FS_TRY(vpred_end_step(c));
  return fil_step(c, nt);
}

static fs_status run_one(fs_ctx *c, int nt, int *iters_h, int choice = -1) {
  FS_CUDA(cudaMemsetAsync(c->flags, 0, sizeof(int) * FLAG_COUNT, c->stream));
  const int before = c->diag.not_converged_steps;
  int it = 0;
  FS_TRY(step_implicit(c, nt, &it, true, choice));
  if (iters_h) *iters_h = it;
  if (c->diag.nonfinite) return FS_ERR_NONFINITE;
  return c->diag.not_converged_steps > before ? FS_ERR_NOT_CONVERGED : FS_OK;
}

static bool use_graph(const fs_ctx *c, int nt) {
  return c->graph_mode && graph_steady(c, nt) && !learn_active(c) && !learn_recording(c);
}

// the learned start under its cost gate: a step the gate gives the plain start
// runs as the captured graph (flushed at once, so the gate sees its solves
// before its next choice); a learned-start step runs host-driven
static bool use_gated_graph(const fs_ctx *c, int nt) {
  return c->graph_mode && graph_steady(c, nt) && learn_active(c) && learn_gate_on(c) && !learn_recording(c);
}

static fs_status run_one_gated(fs_ctx *c, int nt, int *iters_h) {
  if (learn_gate_choose(c)) return run_one(c, nt, iters_h, 1);
  // the graph ends with hist_end_step and Filament::step (its start reads the
  // history, so it must not shift before the launch)
  FS_TRY(learn_end_step(c));
  FS_TRY(graph_launch_step(c, nt));
  int it = 0;
  fs_status s = graph_flush(c, &it);
  if (iters_h) *iters_h = it;
  if (s == FS_OK || s == FS_ERR_NOT_CONVERGED) learn_gate_record(c, false, (long long)it + 1);
  return s;
}

fs_status fs_step_implicit(fs_ctx *c, int nt, int *iters_h) {
  if (!c) return FS_ERR_INVALID_ARG;
  if (!c->have_state) return FS_ERR_STATE;
  memset(&c->diag, 0, sizeof c->diag);
  if (use_graph(c, nt)) {
    FS_TRY(graph_launch_step(c, nt));
    return graph_flush(c, iters_h);
  }
  if (use_gated_graph(c, nt)) return run_one_gated(c, nt, iters_h);
  return run_one(c, nt, iters_h);
}

fs_status fs_set_precision_escalation(fs_ctx *c, int after_iters) {
  if (!c || after_iters < 0) return FS_ERR_INVALID_ARG;
  c->escalate_after = after_iters;
  graph_invalidate(c);  // captured FP32 steps bake the second loop
  return FS_OK;
}

fs_status fs_set_graph_mode(fs_ctx *c, int on) {
  if (!c) return FS_ERR_INVALID_ARG;
  c->graph_mode = on ? 1 : 0;
  if (!on) graph_invalidate(c);
  return FS_OK;
}

fs_status fs_run_steps(fs_ctx *c, int nt_start, int nsteps, int *iters_h) {
  if (!c || nsteps < 0) return FS_ERR_INVALID_ARG;
  if (!c->have_state) return FS_ERR_STATE;
  memset(&c->diag, 0, sizeof c->diag);
  fs_status worst = FS_OK;
  int k = 0;
  while (k < nsteps) {
    if (use_graph(c, nt_start + k)) {
      // a run of graph launches, one synchronisation at its end
      const int k0 = k;
      int n = 0;
      while (k < nsteps && n < 4096 && use_graph(c, nt_start + k)) {
        FS_TRY(graph_launch_step(c, nt_start + k));
        ++k;
        ++n;
      }
      fs_status s = graph_flush(c, iters_h ? iters_h + k0 : nullptr);
      if (s != FS_OK && s != FS_ERR_NOT_CONVERGED) return s;
      if (s != FS_OK) worst = s;
      continue;
    }
    int it = 0;
    fs_status s = use_gated_graph(c, nt_start + k) ? run_one_gated(c, nt_start + k, &it)
                                                    : run_one(c, nt_start + k, &it);
    if (iters_h) iters_h[k] = it;
    if (s != FS_OK && s != FS_ERR_NOT_CONVERGED) return s;
    if (s != FS_OK) worst = s;
    ++k;
  }
  return worst;
}

fs_status fs_get_diag(fs_ctx *c, fs_diag *d_h) {
  if (!c || !d_h) return FS_ERR_INVALID_ARG;
  *d_h = c->diag;
  unsigned long long bits = 0, mbits = 0;
  FS_CUDA(cudaMemcpyAsync(&bits, c->maxerr_bits, sizeof bits, cudaMemcpyDeviceToHost, c->stream));
  if (c->min_dist2_valid)
    FS_CUDA(cudaMemcpyAsync(&mbits, c->min_dist2_bits, sizeof mbits, cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaStreamSynchronize(c->stream));
  memcpy(&d_h->last_max_abs_err, &bits, sizeof bits);
  if (c->min_dist2_valid) memcpy(&d_h->min_dist2, &mbits, sizeof mbits);
  return FS_OK;
}

}  // extern "C"
