// fs_graph.cu -- an implicit time step (main.cpp:284-754) as one CUDA graph with
// the Broyden loop on the device.
//
// A step in the steady regime (nt above the implicit-Euler, friction and
// lambda-extrapolation thresholds, where every nt-dependent branch of the
// kernels is fixed; no swimming drive, whose strain twist depends on nt) is
// captured once: the start of the step (initial guess,
// forces, Jacobian, cell link, first barrier + mobility solve and residual), a
// conditional WHILE node whose body is one Broyden iteration (apply, update,
// forces, barrier + mobility, residual, history column, err <- newerr), and the
// end of the step (Filament::step). With precision escalation an FP32 step has a
// second WHILE node after the first, its body captured with the FP64 chain. The
// loop condition is the reference's
// `check` (any |Err| > TOL) and iter < broyden_maxiter, set on the device by
// cudaGraphSetConditional; the iteration count lives in device memory and the
// Broyden kernels read it there. A run of steps is a sequence of graph launches
// with one host synchronisation at the end: per-step iteration counts and the
// non-finite / explosion / pivot / capacity flags are kept on the device.
// The arithmetic and its order are the host-driven step's, so trajectories are
// bitwise identical.
#include <vector>
#include "fs_internal.cuh"

enum { GD_ITER = 0, GD_STEPS, GD_NONFIN, GD_EXPLODE, GD_NOTCONV, GD_PIVOT, GD_CAPACITY, GD_ESC, GD_HDR = 8 };
constexpr int GRAPH_STEP_SLOTS = 4096;

struct fs_graph {
  cudaGraphExec_t exec = nullptr;
  cudaStream_t body_stream = nullptr;
  int *dev = nullptr;  // GD_HDR header ints, then the iteration count of each launched step
  int *host = nullptr;  // pinned copy
  unsigned long long *ts = nullptr;  // per launched step: device clock (ns) at its start and end (batches)
  unsigned long long kpre = 0, kbody = 0;  // kernels per launch outside / inside the loop
  unsigned long long kbody64 = 0;          // kernels per iteration of the escalated FP64 loop
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
                            cudaGraphConditionalHandle h, int escalated) {
  const int it = gd[GD_ITER] + 1;
  gd[GD_ITER] = it;
  if (escalated) gd[GD_ESC] += 1;
  gd[GD_NONFIN] |= flags[FLAG_NONFINITE];
  gd[GD_EXPLODE] |= flags[FLAG_EXPLODE];
  cudaGraphSetConditional(h, (flags[FLAG_CHECK] && it < maxiter) ? 1u : 0u);
}

// between the FP32 loop and the escalated FP64 loop: go on while unconverged
__global__ void k_loop_mid(const int *__restrict__ gd, const int *__restrict__ flags, int maxiter,
                           cudaGraphConditionalHandle h) {
  cudaGraphSetConditional(h, (flags[FLAG_CHECK] && gd[GD_ITER] < maxiter) ? 1u : 0u);
}

__global__ void k_step_done(int *__restrict__ gd, const int *__restrict__ flags, int slots) {
  const int k = gd[GD_STEPS];
  if (k < slots) gd[GD_HDR + k] = gd[GD_ITER];
  gd[GD_STEPS] = k + 1;
  if (flags[FLAG_CHECK]) gd[GD_NOTCONV] += 1;
  gd[GD_CAPACITY] |= flags[FLAG_CAPACITY];
}

__global__ void k_stamp(const int *__restrict__ gd, unsigned long long *__restrict__ ts, int which, int slots) {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  const int k = gd[GD_STEPS] - which;  // the end stamp follows k_step_done's increment
  if (k >= 0 && k < slots) ts[2 * k + which] = t;
}

// one Broyden iteration (main.cpp:572-673) captured into the conditional node's
// body graph on g->body_stream, ending with the loop condition (limit: the last
// iteration count it may reach)
fs_status capture_body(fs_ctx *c, int nt, fs_graph *g, cudaGraph_t body, cudaGraphConditionalHandle h, int limit,
                       bool escalated, unsigned long long *kernels) {
  cudaStream_t main_stream = c->stream;
  const unsigned long long k0 = __atomic_load_n(&g_fs_kernel_launches, __ATOMIC_RELAXED);
  FS_CUDA(cudaStreamBeginCaptureToGraph(g->body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  c->stream = g->body_stream;
  fs_status st = fcm_set_stream(c, c->stream);
  // with the Broyden memory on the column count lives on the device (fs_bmem.cu)
  const int *off = bmem_off(c);
  const int *iter_d = off ? nullptr : g->dev + GD_ITER;
  if (st == FS_OK) st = bmem_iter_begin(c, nt, 0, g->dev + GD_ITER);
  if (st == FS_OK) st = fil_broyden_apply(c, c->err, c->upd, 0, iter_d, off);
  if (st == FS_OK) st = fil_state_update(c, c->upd);
  if (st == FS_OK) st = fil_forces(c, nt);
  if (st == FS_OK) st = step_barrier_mobility(c, nt);
  if (st == FS_OK) st = fil_error_check(c, c->V, c->W, c->newerr, nt);
  if (st == FS_OK) st = fil_broyden_update(c, 0, iter_d, off);
  if (st == FS_OK) st = bmem_iter_end(c);
  if (st == FS_OK && cudaMemcpyAsync(c->err, c->newerr, sizeof(double) * 6 * (size_t)c->np, cudaMemcpyDeviceToDevice,
                                     c->stream) != cudaSuccess)
    st = FS_ERR_CUDA;
  if (st == FS_OK) {
    k_loop_tail<<<1, 1, 0, c->stream>>>(g->dev, c->flags, limit, h, escalated ? 1 : 0);
    if (cudaGetLastError() != cudaSuccess) st = FS_ERR_CUDA;
    __atomic_fetch_add(&g_fs_kernel_launches, 1ull, __ATOMIC_RELAXED);
  }
  cudaGraph_t body_out = body;
  const cudaError_t e_end = cudaStreamEndCapture(g->body_stream, &body_out);
  c->stream = main_stream;
  const fs_status st2 = fcm_set_stream(c, c->stream);
  *kernels = __atomic_load_n(&g_fs_kernel_launches, __ATOMIC_RELAXED) - k0;
  FS_TRY(st);
  FS_TRY(st2);
  FS_CUDA(e_end);
  return FS_OK;
}

// a conditional handle of the graph being captured on c->stream
fs_status new_cond_handle(fs_ctx *c, cudaGraphConditionalHandle *h) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  FS_CUDA(cudaStreamGetCaptureInfo(c->stream, &cs, nullptr, &cg, &deps, &nd));
  FS_CUDA(cudaGraphConditionalHandleCreate(h, cg, 0, 0));
  return FS_OK;
}

// a conditional WHILE node after the capture's current dependencies; its body graph
fs_status add_while_node(fs_ctx *c, cudaGraphConditionalHandle h, cudaGraph_t *body) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  FS_CUDA(cudaStreamGetCaptureInfo(c->stream, &cs, nullptr, &cg, &deps, &nd));
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  FS_CUDA(cudaGraphAddNode(&cnode, cg, deps, nd, &cp));
  FS_CUDA(cudaStreamUpdateCaptureDependencies(c->stream, &cnode, 1, cudaStreamSetCaptureDependencies));
  *body = cp.conditional.phGraph_out[0];
  return FS_OK;
}

// the start, loop(s) and end of one step, captured on c->stream. With precision
// escalation (fs_set_precision_escalation) an FP32 step runs two loops: the FP32
// iterations up to the escalation count, then, while unconverged, the rest with
// the FP64 chain.
fs_status capture_step(fs_ctx *c, int nt, fs_graph *g, cudaGraph_t *out) {
  const int maxiter = c->p.broyden_maxiter;
  const int esc = (c->precision == FS_PREC_FP32 && c->escalate_after > 0) ? c->escalate_after : 0;
  const int limit1 = esc > 0 && esc < maxiter ? esc : maxiter;
  FS_CUDA(cudaMemsetAsync(c->flags, 0, sizeof(int) * FLAG_COUNT, c->stream));
  FS_TRY(fil_initial_guess(c));
  FS_TRY(fil_forces(c, nt));
  FS_TRY(fil_jacobian_build(c, nt, bmem_keep(c)));
  FS_TRY(cells_link(c, c->Xs, c->np));
  FS_TRY(vpred_step(c, nt));
  FS_TRY(step_barrier_mobility(c, nt));
  FS_TRY(fil_error_check(c, c->V, c->W, c->err, nt));
  cudaGraphConditionalHandle h;
  FS_TRY(new_cond_handle(c, &h));
  k_loop_head<<<1, 1, 0, c->stream>>>(g->dev, c->flags, limit1, h);
  FS_LAUNCH_CHECK();
  cudaGraph_t body;
  FS_TRY(add_while_node(c, h, &body));
  FS_TRY(capture_body(c, nt, g, body, h, limit1, false, &g->kbody));
  g->kbody64 = 0;
  if (esc > 0 && limit1 < maxiter) {
    cudaGraphConditionalHandle h2;
    FS_TRY(new_cond_handle(c, &h2));
    k_loop_mid<<<1, 1, 0, c->stream>>>(g->dev, c->flags, maxiter, h2);
    FS_LAUNCH_CHECK();
    cudaGraph_t body2;
    FS_TRY(add_while_node(c, h2, &body2));
    c->precision = FS_PREC_FP64;
    const fs_status st = capture_body(c, nt, g, body2, h2, maxiter, true, &g->kbody64);
    c->precision = FS_PREC_FP32;
    FS_TRY(st);
    FS_TRY(fcm_set_stream(c, c->stream));
  }
  FS_TRY(learn_end_step(c));
  FS_TRY(hist_end_step(c));
  FS_TRY(bmem_end_step(c, 0, g->dev + GD_ITER));
  FS_TRY(vpred_end_step(c));
  FS_TRY(fil_step(c, nt));
  k_step_done<<<1, 1, 0, c->stream>>>(g->dev, c->flags, GRAPH_STEP_SLOTS);
  FS_LAUNCH_CHECK();
  (void)out;
  return FS_OK;
}

}  // namespace

bool graph_steady(const fs_ctx *c, int nt) {
  // a swimming drive makes the forces depend on nt, which a captured step bakes in
  return nt > c->p.impl_euler_steps && nt > c->p.initial_friction_steps && nt > c->p.lambda_extrap_step &&
         !c->swim;
}

void graph_free(fs_ctx *c) {
  fs_graph *g = c->graph;
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->body_stream) cudaStreamDestroy(g->body_stream);
  cudaFree(g->dev);
  cudaFree(g->ts);
  if (g->host) cudaFreeHost(g->host);
  delete g;
  c->graph = nullptr;
}

void graph_invalidate(fs_ctx *c) {
  c->graph_gen++;
  if (c->graph && c->graph->exec) {
    cudaGraphExecDestroy(c->graph->exec);
    c->graph->exec = nullptr;
  }
}

// buffers of the graph state, cuFFT plans and learn buffers: everything the
// captured work touches must exist before a capture
static fs_status graph_prepare(fs_ctx *c) {
  fs_graph *g = c->graph;
  if (!g) {
    g = new fs_graph();
    c->graph = g;
    FS_CUDA(cudaStreamCreateWithFlags(&g->body_stream, cudaStreamNonBlocking));
    FS_CUDA(cudaMalloc(&g->dev, sizeof(int) * (GD_HDR + GRAPH_STEP_SLOTS)));
    FS_CUDA(cudaMallocHost(&g->host, sizeof(int) * (GD_HDR + GRAPH_STEP_SLOTS)));
    FS_CUDA(cudaMalloc(&g->ts, sizeof(unsigned long long) * 2 * GRAPH_STEP_SLOTS));
    FS_CUDA(cudaMemsetAsync(g->dev, 0, sizeof(int) * GD_HDR, c->stream));
  }
  FS_TRY(fcm_set_stream(c, c->stream));
  if (c->precision == FS_PREC_FP32 && c->escalate_after > 0) {
    // the escalated loop's FP64 plans must exist before a capture
    c->precision = FS_PREC_FP64;
    const fs_status st = fcm_set_stream(c, c->stream);
    c->precision = FS_PREC_FP32;
    FS_TRY(st);
  }
  return learn_prepare_capture(c);
}

static fs_status graph_build(fs_ctx *c, int nt) {
  FS_TRY(graph_prepare(c));
  fs_graph *g = c->graph;
  graph_invalidate(c);
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
  g->kpre = captured - g->kbody - g->kbody64;
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
  const long long esc_its = g->host[GD_ESC];  // iterations of the escalated FP64 loop
  c->diag.escalated_iters += esc_its;
  __atomic_fetch_add(&g_fs_kernel_launches,
                     (unsigned long long)n * g->kpre + (unsigned long long)(its - esc_its) * g->kbody +
                         (unsigned long long)esc_its * g->kbody64,
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

// ---- ensembles: one graph launch advances every box by one step ------------------
struct fs_batch {
  int n = 0;
  fs_ctx **ctx = nullptr;
  int *gen = nullptr;  // each box's graph_gen when the batch graph was captured
  cudaStream_t origin = nullptr;
  cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
  cudaEvent_t *join = nullptr;
  cudaGraphExec_t exec = nullptr;
};

static fs_status batch_build(fs_batch *b, int nt) {
  for (int i = 0; i < b->n; ++i) {
    fs_ctx *c = b->ctx[i];
    if (!c->have_state || !graph_steady(c, nt)) return FS_ERR_STATE;
    FS_TRY(graph_prepare(c));
    FS_TRY(graph_flush(c, nullptr));
  }
  std::vector<fs_diag> diag(b->n);
  std::vector<bool> prof(b->n);
  for (int i = 0; i < b->n; ++i) {
    diag[i] = b->ctx[i]->diag;
    prof[i] = b->ctx[i]->prof.on;
    b->ctx[i]->prof.on = false;
  }
  FS_CUDA(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
  fs_status st = FS_OK;
  unsigned long long captured = 0;
  // every box forks from the same point and joins at the end: the boxes' steps are
  // independent branches of the graph
  if (cudaEventRecord(b->fork, b->origin) != cudaSuccess) st = FS_ERR_CUDA;
  for (int i = 0; i < b->n && st == FS_OK; ++i) {
    fs_ctx *c = b->ctx[i];
    fs_graph *g = c->graph;
    const unsigned long long k0 = __atomic_load_n(&g_fs_kernel_launches, __ATOMIC_RELAXED);
    if (cudaStreamWaitEvent(c->stream, b->fork, 0) != cudaSuccess) {
      st = FS_ERR_CUDA;
      break;
    }
    k_stamp<<<1, 1, 0, c->stream>>>(g->dev, g->ts, 0, GRAPH_STEP_SLOTS);
    __atomic_fetch_add(&g_fs_kernel_launches, 1ull, __ATOMIC_RELAXED);
    st = capture_step(c, nt, g, nullptr);
    if (st != FS_OK) break;
    k_stamp<<<1, 1, 0, c->stream>>>(g->dev, g->ts, 1, GRAPH_STEP_SLOTS);
    __atomic_fetch_add(&g_fs_kernel_launches, 1ull, __ATOMIC_RELAXED);
    if (cudaGetLastError() != cudaSuccess || cudaEventRecord(b->join[i], c->stream) != cudaSuccess) st = FS_ERR_CUDA;
    const unsigned long long kb = __atomic_load_n(&g_fs_kernel_launches, __ATOMIC_RELAXED) - k0;
    g->kpre = kb - g->kbody - g->kbody64;
    captured += kb;
  }
  for (int i = 0; i < b->n && st == FS_OK; ++i)
    if (cudaStreamWaitEvent(b->origin, b->join[i], 0) != cudaSuccess) st = FS_ERR_CUDA;
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->origin, &graph);
  __atomic_fetch_sub(&g_fs_kernel_launches, captured, __ATOMIC_RELAXED);
  for (int i = 0; i < b->n; ++i) b->gen[i] = b->ctx[i]->graph_gen;
  for (int i = 0; i < b->n; ++i) {
    b->ctx[i]->diag = diag[i];
    b->ctx[i]->prof.on = prof[i];
  }
  if (st != FS_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  FS_CUDA(e);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&b->exec, graph, 0);
  cudaGraphDestroy(graph);
  FS_CUDA(ei);
  return FS_OK;
}

extern "C" {

fs_status fs_batch_create(fs_ctx *const *ctxs, int n, fs_batch **out) {
  if (!ctxs || n <= 0 || !out) return FS_ERR_INVALID_ARG;
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (!ctxs[i]) return FS_ERR_INVALID_ARG;
    for (int j = 0; j < i; ++j)
      if (ctxs[j] == ctxs[i] || ctxs[j]->stream == ctxs[i]->stream) return FS_ERR_INVALID_ARG;
  }
  fs_batch *b = new fs_batch();
  b->n = n;
  b->ctx = new fs_ctx *[n];
  b->gen = new int[n]();
  b->join = new cudaEvent_t[n]();
  for (int i = 0; i < n; ++i) b->ctx[i] = ctxs[i];
  fs_status st = FS_OK;
  if (cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&b->t0) != cudaSuccess || cudaEventCreate(&b->t1) != cudaSuccess)
    st = FS_ERR_CUDA;
  for (int i = 0; i < n && st == FS_OK; ++i)
    if (cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) != cudaSuccess) st = FS_ERR_CUDA;
  if (st != FS_OK) {
    fs_batch_destroy(b);
    return st;
  }
  *out = b;
  return FS_OK;
}

fs_status fs_batch_destroy(fs_batch *b) {
  if (!b) return FS_OK;
  if (b->origin) cudaStreamSynchronize(b->origin);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (int i = 0; i < b->n; ++i)
    if (b->join && b->join[i]) cudaEventDestroy(b->join[i]);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->t0) cudaEventDestroy(b->t0);
  if (b->t1) cudaEventDestroy(b->t1);
  if (b->origin) cudaStreamDestroy(b->origin);
  delete[] b->join;
  delete[] b->gen;
  delete[] b->ctx;
  delete b;
  return FS_OK;
}

fs_status fs_batch_run(fs_batch *b, int nt_start, int nsteps, int *iters_h, float *box_ms_h, float *total_ms_h) {
  if (!b || nsteps < 0 || nsteps > GRAPH_STEP_SLOTS) return FS_ERR_INVALID_ARG;
  if (nsteps == 0) return FS_OK;
  bool stale = !b->exec;
  for (int i = 0; i < b->n; ++i) stale = stale || b->gen[i] != b->ctx[i]->graph_gen;
  if (stale) FS_TRY(batch_build(b, nt_start));
  for (int i = 0; i < b->n; ++i) {
    fs_ctx *c = b->ctx[i];
    if (!graph_steady(c, nt_start)) return FS_ERR_STATE;
    memset(&c->diag, 0, sizeof c->diag);
    // the boxes' own streams finish their earlier work before the batch starts
    FS_CUDA(cudaEventRecord(b->join[i], c->stream));
    FS_CUDA(cudaStreamWaitEvent(b->origin, b->join[i], 0));
  }
  FS_CUDA(cudaEventRecord(b->t0, b->origin));
  for (int k = 0; k < nsteps; ++k) FS_CUDA(cudaGraphLaunch(b->exec, b->origin));
  FS_CUDA(cudaEventRecord(b->t1, b->origin));
  FS_CUDA(cudaStreamSynchronize(b->origin));
  if (total_ms_h) FS_CUDA(cudaEventElapsedTime(total_ms_h, b->t0, b->t1));
  fs_status worst = FS_OK;
  std::vector<int> its(nsteps);
  std::vector<unsigned long long> ts(2 * (size_t)nsteps);
  for (int i = 0; i < b->n; ++i) {
    fs_ctx *c = b->ctx[i];
    fs_graph *g = c->graph;
    g->pending = nsteps;
    if (box_ms_h) {
      FS_CUDA(cudaMemcpy(ts.data(), g->ts, sizeof(unsigned long long) * 2 * nsteps, cudaMemcpyDeviceToHost));
      for (int k = 0; k < nsteps; ++k) box_ms_h[(size_t)k * b->n + i] = (float)((ts[2 * k + 1] - ts[2 * k]) * 1e-6);
    }
    fs_status s = graph_flush(c, its.data());
    c->diag.last_nt = nt_start + nsteps - 1;
    if (iters_h)
      for (int k = 0; k < nsteps; ++k) iters_h[(size_t)k * b->n + i] = its[k];
    if (s != FS_OK && s != FS_ERR_NOT_CONVERGED) return s;
    if (s != FS_OK) worst = s;
  }
  return worst;
}

}  // extern "C"
