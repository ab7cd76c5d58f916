// fs_start.cu -- the start of the implicit step's Broyden iteration beyond the
// reference's, and the positions two steps back that it needs. No reference
// counterpart.
//
// The reference starts every step from Xs = 2X - Xt for the first bead of each
// filament and Us = 2U - Ut for every bead (Filament::initialGuess,
// Filament.hpp:227-237, Bead.hpp:202-216). U is itself a per-step increment, so
// the orientations are extrapolated to second order, but the first bead's
// position to first order only, and the other beads follow it through the
// robot-arm construction: its error moves the whole filament. With start order 2
// the first bead starts from 3X - 3Xt + Xtt, Xtt the positions two steps back,
// once the context's history spans two steps it ran itself: not on the first two
// steps after creation, a layout change or an upload of other positions (an
// uploaded Xt need not be a step's: a suspension placed at rest has Xt = X, and
// extrapolating through the impulsive start overshoots). The Broyden loop and
// its convergence test are unchanged, so a step converges to the reference's
// tolerance from either start.
//
// The history is also the learned start's acceleration feature (fs_mlp.cu). It
// is kept while either needs it: before Filament::step moves X to Xt, Xtt <- Xt.
//
// Filament::step also starts the next step's tensions: constant before
// lambda_extrap_step, linear at it and quadratic, 3 lam - 3 lam1 + lam2, after it
// (main.cpp's lambda extrapolation). The converged tensions carry the Broyden
// tolerance's noise, which the quadratic extrapolation multiplies by up to 7;
// tension order 1 keeps the linear 2 lam - lam1 (noise up to 3) after
// lambda_extrap_step too.

#include "fs_internal.cuh"

namespace {

// hist_ok counts the steps since the history was last reset, up to 2
__global__ void k_hist_tick(int *ok) {
  if (*ok < 2) ++*ok;
}

// the history, the carried Broyden columns and the velocity history survive an
// upload only if X and Xt are unchanged
__global__ void k_hist_same(size_t n, const double *__restrict__ X, const double *__restrict__ Xt,
                            const double *__restrict__ pX, const double *__restrict__ pXt, int *__restrict__ ok,
                            int *__restrict__ carried, int *__restrict__ vp_ok) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && (X[i] != pX[i] || Xt[i] != pXt[i])) {
    *ok = 0;
    if (carried) bmem_drop(carried);
    if (vp_ok) *vp_ok = 0;
  }
}

// V*, W* = 2 V1 - V2, 2 W1 - W2 (rounded as written)
__global__ void k_vpred_extrap(size_t n, const double *__restrict__ V1, const double *__restrict__ V2,
                               const double *__restrict__ W1, const double *__restrict__ W2, double *__restrict__ Vs,
                               double *__restrict__ Ws) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Vs[i] = __dsub_rn(__dmul_rn(2.0, V1[i]), V2[i]);
  Ws[i] = __dsub_rn(__dmul_rn(2.0, W1[i]), W2[i]);
}

// the predicted residual times the weight; without two recorded states zero, so
// that the update is zero and leaves the state bitwise as it was
__global__ void k_vpred_gate(size_t n, const int *__restrict__ ok, double weight, double *__restrict__ err) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) err[i] = *ok < 2 ? 0.0 : weight * err[i];
}

}  // namespace

// ---- velocity predictor ------------------------------------------------------------
// The step's first residual needs a mobility solve at the initial guess. With the
// predictor on, the step first takes one Broyden update from the residual with the
// velocities extrapolated from the last two converged states, V* = 2 V1 - V2
// (W alike), no solve: x <- x - w H E(x; V*, W*), w the weight, H the iteration's
// current inverse Jacobian (J0^-1 and any carried Broyden columns), then the forces
// at the new iterate; the iteration proper starts there. The update adds no history
// column and counts as no iteration; the convergence test is unchanged.
fs_status vpred_step(fs_ctx *c, int nt) {
  if (c->vpred_weight == 0.0) return FS_OK;
  const size_t n3 = (size_t)3 * c->np, n6 = 2 * n3;
  if (n3 == 0) return FS_OK;
  k_vpred_extrap<<<fs_blocks((long long)n3, 256), 256, 0, c->stream>>>(n3, c->vp_V1, c->vp_V2, c->vp_W1, c->vp_W2,
                                                                      c->vp_Vs, c->vp_Ws);
  FS_LAUNCH_CHECK();
  FS_TRY(fil_error_check(c, c->vp_Vs, c->vp_Ws, c->err, nt));
  k_vpred_gate<<<fs_blocks((long long)n6, 256), 256, 0, c->stream>>>(n6, c->vp_ok, c->vpred_weight, c->err);
  FS_LAUNCH_CHECK();
  FS_TRY(fil_broyden_apply(c, c->err, c->upd, 0, nullptr, bmem_off(c)));
  FS_TRY(fil_state_update(c, c->upd));
  return fil_forces(c, nt);
}

// after a committed step (host-driven and captured): the converged state's V, W
fs_status vpred_end_step(fs_ctx *c) {
  if (c->vpred_weight == 0.0 || c->np == 0) return FS_OK;
  const size_t b = sizeof(double) * 3 * (size_t)c->np;
  FS_CUDA(cudaMemcpyAsync(c->vp_V2, c->vp_V1, b, cudaMemcpyDeviceToDevice, c->stream));
  FS_CUDA(cudaMemcpyAsync(c->vp_W2, c->vp_W1, b, cudaMemcpyDeviceToDevice, c->stream));
  FS_CUDA(cudaMemcpyAsync(c->vp_V1, c->V, b, cudaMemcpyDeviceToDevice, c->stream));
  FS_CUDA(cudaMemcpyAsync(c->vp_W1, c->W, b, cudaMemcpyDeviceToDevice, c->stream));
  k_hist_tick<<<1, 1, 0, c->stream>>>(c->vp_ok);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

void vpred_free(fs_ctx *c) {
  double **arrs[6] = {&c->vp_V1, &c->vp_W1, &c->vp_V2, &c->vp_W2, &c->vp_Vs, &c->vp_Ws};
  if (c->vp_V1) c->bytes -= 6 * sizeof(double) * 3 * (size_t)(c->max_beads > 0 ? c->max_beads : 1) + sizeof(int);
  for (double **a : arrs) {
    cudaFree(*a);
    *a = nullptr;
  }
  cudaFree(c->vp_ok);
  c->vp_ok = nullptr;
}

bool hist_wanted(const fs_ctx *c) { return c->mlp != nullptr || c->start_order == 2; }

fs_status hist_ensure(fs_ctx *c) {
  if (c->hist_Xtt) return FS_OK;
  const size_t n = (size_t)3 * (c->max_beads > 0 ? c->max_beads : 1);
  double **arrs[3] = {&c->hist_Xtt, &c->hist_pX, &c->hist_pXt};
  for (double **a : arrs) {
    const cudaError_t e = cudaMalloc(a, sizeof(double) * n);
    if (e != cudaSuccess) {
      hist_free(c);
      return e == cudaErrorMemoryAllocation ? FS_ERR_OOM : FS_ERR_CUDA;
    }
  }
  const cudaError_t e = cudaMalloc(&c->hist_ok, sizeof(int));
  if (e != cudaSuccess) {
    hist_free(c);
    return e == cudaErrorMemoryAllocation ? FS_ERR_OOM : FS_ERR_CUDA;
  }
  c->bytes += 3 * sizeof(double) * n + sizeof(int);
  c->hist_cmp_pending = false;
  FS_CUDA(cudaMemsetAsync(c->hist_ok, 0, sizeof(int), c->stream));
  return FS_OK;
}

void hist_free(fs_ctx *c) {
  if (c->hist_Xtt || c->hist_ok) {
    const size_t n = (size_t)3 * (c->max_beads > 0 ? c->max_beads : 1);
    c->bytes -= 3 * sizeof(double) * n + sizeof(int);
  }
  cudaFree(c->hist_Xtt);
  cudaFree(c->hist_pX);
  cudaFree(c->hist_pXt);
  cudaFree(c->hist_ok);
  c->hist_Xtt = c->hist_pX = c->hist_pXt = nullptr;
  c->hist_ok = nullptr;
  c->hist_cmp_pending = false;
}

// before Filament::step of every step (also in a captured step, whose graph ends
// with it): Xtt <- Xt, the positions two steps back once X has moved to Xt
fs_status hist_end_step(fs_ctx *c) {
  if (!c->hist_Xtt || !hist_wanted(c)) return FS_OK;
  if (c->np > 0)
    FS_CUDA(cudaMemcpyAsync(c->hist_Xtt, c->Xt, sizeof(double) * 3 * (size_t)c->np, cudaMemcpyDeviceToDevice,
                            c->stream));
  k_hist_tick<<<1, 1, 0, c->stream>>>(c->hist_ok);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

// around fs_state_upload: the history (and the carried Broyden columns) stay valid
// when the upload repeats X and Xt
fs_status hist_before_upload(fs_ctx *c, bool same_layout) {
  c->hist_cmp_pending = false;
  if (!c->hist_Xtt || (same_layout && c->np == 0)) return FS_OK;  // no beads: nothing to compare
  if (!same_layout) {
    FS_CUDA(cudaMemsetAsync(c->hist_ok, 0, sizeof(int), c->stream));
    if (c->vp_ok) FS_CUDA(cudaMemsetAsync(c->vp_ok, 0, sizeof(int), c->stream));
    return bmem_reset(c);
  }
  const size_t b = sizeof(double) * 3 * (size_t)c->np;
  FS_CUDA(cudaMemcpyAsync(c->hist_pX, c->X, b, cudaMemcpyDeviceToDevice, c->stream));
  FS_CUDA(cudaMemcpyAsync(c->hist_pXt, c->Xt, b, cudaMemcpyDeviceToDevice, c->stream));
  c->hist_cmp_pending = true;
  return FS_OK;
}

fs_status hist_after_upload(fs_ctx *c) {
  if (!c->hist_cmp_pending) return FS_OK;
  c->hist_cmp_pending = false;
  const size_t n = (size_t)3 * c->np;
  k_hist_same<<<fs_blocks((long long)n, 256), 256, 0, c->stream>>>(n, c->X, c->Xt, c->hist_pX, c->hist_pXt,
                                                                  c->hist_ok, c->bmem_d, c->vp_ok);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

extern "C" {

fs_status fs_set_start_order(fs_ctx *c, int order) {
  if (!c || (order != 1 && order != 2)) return FS_ERR_INVALID_ARG;
  if (order == 2) FS_TRY(hist_ensure(c));
  c->start_order = order;
  // a history no longer kept would go stale
  if (!hist_wanted(c) && c->hist_ok) FS_CUDA(cudaMemsetAsync(c->hist_ok, 0, sizeof(int), c->stream));
  graph_invalidate(c);  // captured steps bake the start
  return FS_OK;
}

fs_status fs_set_velocity_predictor(fs_ctx *c, double weight) {
  if (!c || !(weight >= 0.0 && weight <= 2.0)) return FS_ERR_INVALID_ARG;
  const bool on = weight > 0.0;
  if (on && !c->vp_V1) {
    const size_t n = (size_t)3 * (c->max_beads > 0 ? c->max_beads : 1);
    double **arrs[6] = {&c->vp_V1, &c->vp_W1, &c->vp_V2, &c->vp_W2, &c->vp_Vs, &c->vp_Ws};
    cudaError_t e = cudaSuccess;
    for (double **a : arrs)
      if (e == cudaSuccess) e = cudaMalloc(a, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&c->vp_ok, sizeof(int));
    if (e != cudaSuccess) {
      cudaGetLastError();
      for (double **a : arrs) {
        cudaFree(*a);
        *a = nullptr;
      }
      cudaFree(c->vp_ok);
      c->vp_ok = nullptr;
      return e == cudaErrorMemoryAllocation ? FS_ERR_OOM : FS_ERR_CUDA;
    }
    c->bytes += 6 * sizeof(double) * n + sizeof(int);
    FS_TRY(hist_ensure(c));  // an upload compares X and Xt
  }
  if (c->vp_ok) FS_CUDA(cudaMemsetAsync(c->vp_ok, 0, sizeof(int), c->stream));
  c->vpred_weight = weight;
  graph_invalidate(c);  // captured steps bake the predictor
  return FS_OK;
}

fs_status fs_set_tension_extrapolation(fs_ctx *c, int order) {
  if (!c || (order != 1 && order != 2)) return FS_ERR_INVALID_ARG;
  c->tension_order = order;
  graph_invalidate(c);  // captured steps bake Filament::step's extrapolation
  return FS_OK;
}

}  // extern "C"
