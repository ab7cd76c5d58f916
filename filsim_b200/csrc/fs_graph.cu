// fs_graph.cu -- an implicit time step (main.cpp:284-754) as one CUDA graph with
// the Broyden loop on the device.
//
// A step in the steady regime (nt above the implicit-Euler, friction and
// lambda-extrapolation thresholds, where every nt-dependent branch of the
// kernels is fixed) is captured once: the start of the step (initial guess,
// forces, Jacobian, cell link, first barrier + mobility solve and residual), a
// conditional WHILE node whose body is one Broyden iteration (apply, update,
// forces, barrier + mobility, residual, history column, err <- newerr), and the
// end of the step (Filament::step). The loop condition is the reference's
// `check` (any |Err| > TOL) and iter < broyden_maxiter, set on the device by
// cudaGraphSetConditional; the iteration count lives in device memory and the
// Broyden kernels read it there. A run of steps is a sequence of graph launches
// with one host synchronisation at the end: per-step iteration counts and the
// non-finite / explosion / pivot / capacity flags are kept on the device.
// The arithmetic and its order are the host-driven step's, so trajectories are
// bitwise identical.
#include "fs_internal.cuh"

enum { GD_ITER = 0, GD_STEPS, GD_NONFIN, GD_EXPLODE, GD_NOTCONV, GD_PIVOT, GD_CAPACITY, GD_HDR = 8 };
constexpr int GRAPH_STEP_SLOTS = 4096;

struct fs_graph {
  cudaGraphExec_t exec = nullptr;
  cudaStream_t body_stream = nullptr;
  int *dev = nullptr;  // GD_HDR header ints, then the iteration count of each launched step
  int *host = nullptr;  // pinned copy
  unsigned long long kpre = 0, kbody = 0;  // kernels per launch outside / inside the loop
  int precision = -1, np = -1, nfil = -1, pending = 0;
};

namespace {

__global__ void k_loop_head(int *__restrict__ gd, const int *__restrict__ flags, int maxiter,
                            cudaGraphConditionalHandle h) {
  gd[GD_ITER] = 0;
  gd[GD_NONFIN] |= flags[FLAG_NONFINITE];
  gd[GD_EXPLODE] |= flags[FLAG_EXPLODE];
  gd[GD_PIVOT] |= flags[FLAG_PIVOT];
  cudaGraphSetConditional(h, (flags[FLAG_CHECK] && maxiter > 0) ? 1u : 0u);
}

__global__ void k_loop_tail(int *__restrict__ gd, const int *__restrict__ flags, int maxiter,
                            cudaGraphConditionalHandle h) {
  const int it = gd[GD_ITER] + 1;
  gd[GD_ITER] = it;
  gd[GD_NONFIN] |= flags[FLAG_NONFINITE];
  gd[GD_EXPLODE] |= flags[FLAG_EXPLODE];
  cudaGraphSetConditional(h, (flags[FLAG_CHECK] && it < maxiter) ? 1u : 0u);
}

__global__ void k_step_done(int *__restrict__ gd, const int *__restrict__ flags, int slots) {
  const int k = gd[GD_STEPS];
  if (k < slots) gd[GD_HDR + k] = gd[GD_ITER];
  gd[GD_STEPS] = k + 1;
  if (flags[FLAG_CHECK]) gd[GD_NOTCONV] += 1;
  gd[GD_CAPACITY] |= flags[FLAG_CAPACITY];
}

// the start, loop and end of one step, captured on c->stream
fs_status capture_step(fs_ctx *c, int nt, fs_graph *g, cudaGraph_t *out) {
  const int maxiter = c->p.broyden_maxiter;
  FS_CUDA(cudaMemsetAsync(c->flags, 0, sizeof(int) * FLAG_COUNT, c->stream));
  FS_TRY(fil_initial_guess(c));
  FS_TRY(fil_forces(c, nt));
  FS_TRY(fil_jacobian_build(c, nt));
  FS_TRY(cells_link(c, c->Xs, c->np));
  FS_TRY(step_barrier_mobility(c, nt));
  FS_TRY(fil_error_check(c, c->V, c->W, c->err, nt));
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  FS_CUDA(cudaStreamGetCaptureInfo(c->stream, &cs, nullptr, &cg, &deps, &nd));
  cudaGraphConditionalHandle h;
  FS_CUDA(cudaGraphConditionalHandleCreate(&h, cg, 0, 0));
  k_loop_head<<<1, 1, 0, c->stream>>>(g->dev, c->flags, maxiter, h);
  FS_LAUNCH_CHECK();
  FS_CUDA(cudaStreamGetCaptureInfo(c->stream, &cs, nullptr, &cg, &deps, &nd));
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  FS_CUDA(cudaGraphAddNode(&cnode, cg, deps, nd, &cp));
  FS_CUDA(cudaStreamUpdateCaptureDependencies(c->stream, &cnode, 1, cudaStreamSetCaptureDependencies));
  // one Broyden iteration (main.cpp:572-673), captured into the loop body
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  cudaStream_t main_stream = c->stream;
  const unsigned long long k0 = __atomic_load_n(&g_fs_kernel_launches, __ATOMIC_RELAXED);
  FS_CUDA(cudaStreamBeginCaptureToGraph(g->body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  c->stream = g->body_stream;
  fs_status st = fcm_set_stream(c, c->stream);
  const int *iter_d = g->dev + GD_ITER;
  if (st == FS_OK) st = fil_broyden_apply(c, c->err, c->upd, 0, iter_d);
  if (st == FS_OK) st = fil_state_update(c, c->upd);
  if (st == FS_OK) st = fil_forces(c, nt);
  if (st == FS_OK) st = step_barrier_mobility(c, nt);
  if (st == FS_OK) st = fil_error_check(c, c->V, c->W, c->newerr, nt);
  if (st == FS_OK) st = fil_broyden_update(c, 0, iter_d);
  if (st == FS_OK && cudaMemcpyAsync(c->err, c->newerr, sizeof(double) * 6 * (size_t)c->np, cudaMemcpyDeviceToDevice,
                                     c->stream) != cudaSuccess)
    st = FS_ERR_CUDA;
  if (st == FS_OK) {
    k_loop_tail<<<1, 1, 0, c->stream>>>(g->dev, c->flags, maxiter, h);
    if (cudaGetLastError() != cudaSuccess) st = FS_ERR_CUDA;
    __atomic_fetch_add(&g_fs_kernel_launches, 1ull, __ATOMIC_RELAXED);
  }
  cudaGraph_t body_out = body;
  const cudaError_t e_end = cudaStreamEndCapture(g->body_stream, &body_out);
  c->stream = main_stream;
  const fs_status st2 = fcm_set_stream(c, c->stream);
  g->kbody = __atomic_load_n(&g_fs_kernel_launches, __ATOMIC_RELAXED) - k0;
  FS_TRY(st);
  FS_TRY(st2);
  FS_CUDA(e_end);
  FS_TRY(learn_end_step(c));
  FS_TRY(fil_step(c, nt));
  k_step_done<<<1, 1, 0, c->stream>>>(g->dev, c->flags, GRAPH_STEP_SLOTS);
  FS_LAUNCH_CHECK();
  (void)out;
  return FS_OK;
}

}  // namespace

bool graph_steady(const fs_ctx *c, int nt) {
  return nt > c->p.impl_euler_steps && nt > c->p.initial_friction_steps && nt > c->p.lambda_extrap_step;
}

void graph_free(fs_ctx *c) {
  fs_graph *g = c->graph;
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->body_stream) cudaStreamDestroy(g->body_stream);
  cudaFree(g->dev);
  if (g->host) cudaFreeHost(g->host);
  delete g;
  c->graph = nullptr;
}

void graph_invalidate(fs_ctx *c) {
  if (c->graph && c->graph->exec) {
    cudaGraphExecDestroy(c->graph->exec);
    c->graph->exec = nullptr;
  }
}

static fs_status graph_build(fs_ctx *c, int nt) {
  fs_graph *g = c->graph;
  if (!g) {
    g = new fs_graph();
    c->graph = g;
    FS_CUDA(cudaStreamCreateWithFlags(&g->body_stream, cudaStreamNonBlocking));
    FS_CUDA(cudaMalloc(&g->dev, sizeof(int) * (GD_HDR + GRAPH_STEP_SLOTS)));
    FS_CUDA(cudaMallocHost(&g->host, sizeof(int) * (GD_HDR + GRAPH_STEP_SLOTS)));
    FS_CUDA(cudaMemsetAsync(g->dev, 0, sizeof(int) * GD_HDR, c->stream));
  }
  graph_invalidate(c);
  // everything the captured work touches must exist before the capture
  FS_TRY(fcm_set_stream(c, c->stream));
  FS_TRY(learn_prepare_capture(c));
  const bool prof = c->prof.on;
  c->prof.on = false;
  const fs_diag diag = c->diag;  // the capture runs nothing; its host-side counters are undone
  const unsigned long long k0 = __atomic_load_n(&g_fs_kernel_launches, __ATOMIC_RELAXED);
  FS_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  fs_status st = capture_step(c, nt, g, nullptr);
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
  c->prof.on = prof;
  c->diag = diag;
  // captured kernels were counted once; launches are counted per graph launch instead
  const unsigned long long captured = __atomic_load_n(&g_fs_kernel_launches, __ATOMIC_RELAXED) - k0;
  __atomic_fetch_sub(&g_fs_kernel_launches, captured, __ATOMIC_RELAXED);
  g->kpre = captured - g->kbody;
  if (st != FS_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  FS_CUDA(e);
  const cudaError_t ei = cudaGraphInstantiate(&g->exec, graph, 0);
  cudaGraphDestroy(graph);
  FS_CUDA(ei);
  g->precision = c->precision;
  g->np = c->np;
  g->nfil = c->nfil;
  return FS_OK;
}

// Synchronises and folds the launched steps into the diagnostics; iters_h gets
// their iteration counts. Returns the status the host-driven steps would have.
fs_status graph_flush(fs_ctx *c, int *iters_h) {
  fs_graph *g = c->graph;
  if (!g || g->pending == 0) return FS_OK;
  const int n = g->pending;
  g->pending = 0;
  FS_CUDA(cudaMemcpyAsync(g->host, g->dev, sizeof(int) * (GD_HDR + (n < GRAPH_STEP_SLOTS ? n : GRAPH_STEP_SLOTS)),
                          cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaStreamSynchronize(c->stream));
  FS_CUDA(cudaMemsetAsync(g->dev, 0, sizeof(int) * GD_HDR, c->stream));
  long long its = 0;
  for (int k = 0; k < n; ++k) {
    const int it = g->host[GD_HDR + k];
    its += it;
    if (iters_h) iters_h[k] = it;
  }
  c->diag.total_iters += its;
  c->diag.last_iters = g->host[GD_HDR + n - 1];
  c->diag.mobility_solves += n + its;
  c->diag.not_converged_steps += g->host[GD_NOTCONV];
  __atomic_fetch_add(&g_fs_kernel_launches, (unsigned long long)n * g->kpre + (unsigned long long)its * g->kbody,
                     __ATOMIC_RELAXED);
  if (g->host[GD_NONFIN]) c->diag.nonfinite = 1;
  if (g->host[GD_EXPLODE]) c->diag.explosion = 1;
  if (g->host[GD_CAPACITY]) return FS_ERR_CAPACITY;
  if (g->host[GD_PIVOT]) return FS_ERR_NONFINITE;
  if (c->diag.nonfinite) return FS_ERR_NONFINITE;
  return g->host[GD_NOTCONV] ? FS_ERR_NOT_CONVERGED : FS_OK;
}

// Launches step nt as a graph (capturing it first if needed). The caller
// flushes before reading results and every GRAPH_STEP_SLOTS launches.
fs_status graph_launch_step(fs_ctx *c, int nt) {
  fs_graph *g = c->graph;
  if (!g || !g->exec || g->precision != c->precision || g->np != c->np || g->nfil != c->nfil) {
    FS_TRY(graph_build(c, nt));
    g = c->graph;
  }
  if (g->pending >= GRAPH_STEP_SLOTS) return FS_ERR_CAPACITY;
  FS_CUDA(cudaGraphLaunch(g->exec, c->stream));
  g->pending++;
  c->diag.last_nt = nt;
  return FS_OK;
}
