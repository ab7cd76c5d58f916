// fs_bmem.cu -- Broyden memory across steps (fs_set_broyden_memory). No reference
// counterpart.
//
// The reference starts every step's iteration from H = J0^-1, the approximate
// inverse Jacobian of the filaments alone (no hydrodynamic coupling between
// beads), and its "bad Broyden" updates add one rank-one term C_i D_i^T per
// iteration (main.cpp:640-663, FilamentJacobianSolver.hpp:49-73):
// H = J0^-1 + sum_i C_i D_i^T. What those terms learn about the coupling is
// dropped at the end of the step, and J0 is rebuilt (3 ms per 512^3 step). The
// memory hands them on:
//  - after a converged step of fewer than `threshold` iterations whose history
//    holds at most keep_columns columns, the next step keeps J0 and all of them:
//    its iteration continues the same H (the Jacobian kernels skip);
//  - after a converged step of `threshold` or more iterations, its last
//    carry_columns columns start the next step beside a new J0;
//  - otherwise (an unconverged step, or a history past keep_columns) the next
//    step starts afresh, as the reference's does;
//  - a step that runs on carried state and reaches restart_after iterations
//    drops it: J0 is built at the current iterate and the history restarts empty,
//    as if the step had started there.
// The convergence test is unchanged, so each step still ends within the
// tolerance; what changes is the path to it. The column count lives on the device
// (BM_NCOL), so host-driven and captured steps run the same kernels on the same
// data and give bitwise the same results.
#include "fs_internal.cuh"

namespace {

struct BmemPolicy {
  int keep, thr, carry;
};

// after a committed step of (its_d ? *its_d : its) iterations with m[BM_NCOL]
// columns in use: the next step's start
__global__ void k_bmem_plan(int *m, BmemPolicy p, int its, const int *its_d, const int *flags) {
  const int it = its_d ? *its_d : its;
  const int total = m[BM_NCOL];
  const bool conv = !(flags[FLAG_CHECK] || flags[FLAG_NONFINITE]);
  int ncol = 0, move = 0, keepj = 0;
  if (conv && p.keep > 0 && it < p.thr && total <= p.keep) {
    ncol = total;
    keepj = 1;
  } else if (conv && p.carry > 0 && it >= p.thr) {
    ncol = move = total < p.carry ? total : p.carry;
  }
  m[BM_MOVE] = move;
  m[BM_SRC] = move ? total - move : 0;
  m[BM_NCOL] = ncol;
  m[BM_KEEPJ] = keepj;
  m[BM_SKIPJ] = 1;
  m[BM_CARRIED] = (ncol > 0 || keepj) ? 1 : 0;
}

// columns [m[BM_SRC], + m[BM_MOVE]) of C and D move to [0, m[BM_MOVE]). A thread
// moves its element of every column in ascending order; the source column
// src + j lies above every destination written before it, so no source is
// overwritten before it is read.
__global__ void k_bmem_move(size_t n6, const int *__restrict__ m, double *C, double *D) {
  const int move = m[BM_MOVE], src = m[BM_SRC];
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (src == 0 || k >= n6) return;
  for (int j = 0; j < move; ++j) {
    C[(size_t)j * n6 + k] = C[(size_t)(src + j) * n6 + k];
    D[(size_t)j * n6 + k] = D[(size_t)(src + j) * n6 + k];
  }
}

// top of iteration (iter_d ? *iter_d : iter): the restart of a step on carried state
__global__ void k_bmem_restart(int *m, int restart, int iter, const int *iter_d) {
  const int it = iter_d ? *iter_d : iter;
  const bool now = m[BM_CARRIED] && it == restart;
  if (now) {
    m[BM_NCOL] = 0;
    m[BM_CARRIED] = 0;
  }
  m[BM_SKIPJ] = now ? 0 : 1;
}

// after the history update of an iteration: one more column in use
__global__ void k_bmem_next(int *m) { ++m[BM_NCOL]; }

}  // namespace

fs_status bmem_iter_begin(fs_ctx *c, int nt, int iter, const int *iter_d) {
  if (c->bmem_cols <= 0 || c->bmem_restart <= 0) return FS_OK;
  k_bmem_restart<<<1, 1, 0, c->stream>>>(c->bmem_d, c->bmem_restart, iter, iter_d);
  FS_LAUNCH_CHECK();
  return fil_jacobian_build(c, nt, c->bmem_d + BM_SKIPJ);
}

fs_status bmem_iter_end(fs_ctx *c) {
  if (c->bmem_cols <= 0) return FS_OK;
  k_bmem_next<<<1, 1, 0, c->stream>>>(c->bmem_d);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

fs_status bmem_end_step(fs_ctx *c, int its, const int *its_d) {
  if (c->bmem_cols <= 0) return FS_OK;
  const BmemPolicy p{c->bmem_keep, c->bmem_thr, c->bmem_carry};
  k_bmem_plan<<<1, 1, 0, c->stream>>>(c->bmem_d, p, its, its_d, c->flags);
  FS_LAUNCH_CHECK();
  const size_t n6 = (size_t)6 * c->np;
  if (c->bmem_carry > 0 && n6 > 0) {
    k_bmem_move<<<fs_blocks((long long)n6, 256), 256, 0, c->stream>>>(n6, c->bmem_d, c->Cmat, c->Dmat);
    FS_LAUNCH_CHECK();
  }
  return FS_OK;
}

fs_status bmem_reset(fs_ctx *c) {
  if (c->bmem_d) FS_CUDA(cudaMemsetAsync(c->bmem_d, 0, BM_COUNT * sizeof(int), c->stream));
  return FS_OK;
}

void bmem_free(fs_ctx *c) {
  if (c->bmem_d) c->bytes -= BM_COUNT * sizeof(int);
  cudaFree(c->bmem_d);
  c->bmem_d = nullptr;
}

extern "C" {

fs_status fs_set_broyden_memory(fs_ctx *c, int keep_columns, int carry_columns, int threshold, int restart_after) {
  if (!c || keep_columns < 0 || carry_columns < 0 || threshold < 0 || restart_after < 0 ||
      keep_columns > FS_BROYDEN_MEMORY_MAX || carry_columns > FS_BROYDEN_MEMORY_MAX)
    return FS_ERR_INVALID_ARG;
  const int cols = keep_columns > carry_columns ? keep_columns : carry_columns;
  if (cols > c->bmem_cap) {
    // the history grows to broyden_maxiter + cols columns (its contents are dropped)
    FS_CUDA(cudaStreamSynchronize(c->stream));
    const size_t ncols = (size_t)c->p.broyden_maxiter + cols;
    const size_t n6 = (size_t)6 * (c->max_beads > 0 ? c->max_beads : 1);
    double *C = nullptr, *D = nullptr, *dots = nullptr, *part = nullptr;
    cudaError_t e = cudaMalloc(&C, sizeof(double) * ncols * n6);
    if (e == cudaSuccess) e = cudaMalloc(&D, sizeof(double) * ncols * n6);
    if (e == cudaSuccess) e = cudaMalloc(&dots, sizeof(double) * ncols);
    if (e == cudaSuccess) e = cudaMalloc(&part, sizeof(double) * ncols * 296);
    if (e != cudaSuccess) {
      cudaFree(C);
      cudaFree(D);
      cudaFree(dots);
      cudaFree(part);
      cudaGetLastError();
      return e == cudaErrorMemoryAllocation ? FS_ERR_OOM : FS_ERR_CUDA;
    }
    cudaFree(c->Cmat);
    cudaFree(c->Dmat);
    cudaFree(c->dots);
    cudaFree(c->partials);
    c->Cmat = C;
    c->Dmat = D;
    c->dots = dots;
    c->partials = part;
    c->bytes += sizeof(double) * (size_t)(cols - c->bmem_cap) * (2 * n6 + 297);
    c->bmem_cap = cols;
  }
  if (cols > 0 && !c->bmem_d) {
    FS_CUDA(cudaMalloc(&c->bmem_d, BM_COUNT * sizeof(int)));
    c->bytes += BM_COUNT * sizeof(int);
  }
  if (cols > 0) FS_TRY(hist_ensure(c));  // an upload compares X and Xt (fs_start.cu)
  c->bmem_keep = keep_columns;
  c->bmem_carry = carry_columns;
  c->bmem_thr = threshold;
  c->bmem_restart = restart_after;
  c->bmem_cols = cols;
  FS_TRY(bmem_reset(c));
  graph_invalidate(c);  // captured steps bake the history's pointers and the policy
  return FS_OK;
}

}  // extern "C"
