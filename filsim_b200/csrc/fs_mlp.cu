// fs_mlp.cu -- learned Broyden warm start: a per-filament MLP trained and run
// on the tensor cores by this library's own kernels (no reference counterpart;
// the reference always starts Broyden from the extrapolated guess of
// Filament::initialGuess, Filament.hpp:227-237, with J0^-1 as the initial
// inverse Jacobian, main.cpp:556-566).
//
// Network: features (19 per bead, 9 per link, log K_B) -> 3 x (Linear 256 + SiLU) -> Linear
// to 12 nw outputs: the update from the extrapolated guess to the converged
// state in the solver's own coordinates [X0 | U | lambda] (6 nw) and a
// correction to the diagonal of the initial inverse Jacobian (6 nw). Linear
// layers are BF16 GEMMs with FP32 accumulation (fs_gemm.cuh); activations are
// stored in BF16 (and their transposes, for the weight gradients), the
// pre-activations in FP32; FP32 master weights with Adam.
//
// In a step (step_implicit): features of the state before the step -> MLP ->
// candidate start. Both starts are evaluated (one mobility solve each); every
// filament whose learned-start residual (max |E| over its rows) is larger than
// its plain-start residual is put back to the plain start, and the residual is
// recomputed when any filament was put back. The Broyden iteration then runs
// unchanged to the reference's tolerance test.
#include <algorithm>
#include <mutex>
#include <vector>
#include "fs_internal.cuh"
#include "fs_gemm.cuh"
#include <cudaTypedefs.h>

struct fs_mlp {
  int nw, nfeat, k_in, hidden, ntgt, k_out, cap;
  int dims[5];
  float *W[4], *b[4], *mW[4], *vW[4], *mb[4], *vb[4], *dW[4], *db[4];
  fs_bf16 *Wb[4], *WTb[4];
  float *in_mu, *in_sd, *out_mu, *out_sd;
  fs_bf16 *X, *XT;
  float *Z[3];
  fs_bf16 *H[3], *HT[3], *dZ[3], *dZT[3];
  float *Y, *T;
  fs_bf16 *dY, *dYT;
  float *outbuf;  // denormalised outputs [cap x ntgt]
  double *loss;
  int *err;
  int adam_t;
  // warm start state
  int mode;            // 0 off, 1 learned iterate, 2 learned iterate + inverse-Jacobian diagonal
  bool record;
  double *gXs, *gUs, *gqs, *glam;  // the plain (extrapolated) guess of the current step
  double *updl, *jdiag;            // 6 Np
  float *feat, *pred, *tgt;        // [nfil x nfeat], [nfil x ntgt], [nfil x ntgt]
  float *rP, *rL;                  // per filament residuals
  int *plain_next;                 // per filament: take the plain start until the next comparison step
  // carried bound (fs_warm_start_bound): between comparison steps the learned
  // start alone is solved and checked against rP of the last comparison step
  int bound_refresh;               // 0: compare with the plain start every step
  int bound_age;                   // learned steps since rP was measured
  bool bound_ok;                   // rP holds a comparison step's plain residuals
  int *count;                      // [0] filaments put back to the plain start
  int *count_h;
  int nfil_alloc, np_alloc;
  bool jdiag_on;                   // jdiag holds this step's diagonal
  bool have_targets;
  bool override_next;              // the next warm start uses pred as given (fs_learn_override)
  long long learned_total, fallback_total;
  // cost gate of the learned start (fs_warm_start_gate): per start, the running
  // mean of mobility solves per step; the cheaper start (the learned one only
  // when it saves gate_margin solves per step) runs and the other one is probed after
  // gate_interval steps. The interval starts at gate_period and
  // doubles (up to GATE_BACKOFF_MAX x gate_period) after each probe that leaves
  // the choice unchanged; a probe that changes it restores gate_period.
  int gate_period;                 // 0: off (the learned start runs every step)
  int gate_interval;
  double gate_margin = 0.25;       // solves per step the learned start must save (fs_warm_start_gate_margin)
  double gate_solves[2];           // [0] plain start, [1] learned start
  int gate_have[2];
  int gate_since;
  int gate_probe_best = -1;        // -1: no probe pending; else the best start when the probe was chosen
  long long gate_steps[2];
};

namespace {

constexpr int RND = 128;
// normalised inputs and targets are clipped to +-NORM_CLIP standard deviations:
// the targets are heavy-tailed (collision events) and the mean-square loss
// would otherwise be set by a few outliers
constexpr float NORM_CLIP = 10.f;
int round_up(int x, int m) { return (x + m - 1) / m * m; }

// ---- small kernels ---------------------------------------------------------------
// Features of one filament (one warp): per bead i, 19 values [X_i - centroid (3), q_i (4),
// (X_i - Xt_i)/dt (3), U_i/dt (3), Ut_i/dt (3), (X_i - 2 Xt_i + Xtt_i)/dt^2 (3)]; per
// link j, 9 values [lambda_j, lambda1_j, lambda2_j]; then log K_B. The
// extrapolated guess is built from the same history (Filament::initialGuess,
// Filament.hpp:227-237; Filament::step's lambda extrapolation, :455-478); the
// acceleration (zero until two steps of history exist) is what the linear
// position extrapolation leaves out.
__global__ void k_features(int nfil, const int *__restrict__ fil_start, int nw_model, const double *__restrict__ X,
                           const double *__restrict__ Xt, const double *__restrict__ Xtt, const int *__restrict__ xtt_ok,
                           const double *__restrict__ q, const double *__restrict__ U,
                           const double *__restrict__ Ut, const double *__restrict__ lam,
                           const double *__restrict__ lam1, const double *__restrict__ lam2,
                           const double *__restrict__ kap, double inv_dt, int nfeat, float *__restrict__ out) {
  const int f = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (f >= nfil) return;
  const int b0 = fil_start[f], nw = fil_start[f + 1] - b0;
  float *o = out + (size_t)f * nfeat;
  if (nw != nw_model) {
    for (int t = lane; t < nfeat; t += 32) o[t] = 0.f;
    return;
  }
  double c[3] = {0, 0, 0};
  for (int i = lane; i < nw; i += 32)
    for (int d = 0; d < 3; ++d) c[d] += X[3 * (b0 + i) + d];
  for (int d = 0; d < 3; ++d)
    for (int m = 16; m >= 1; m >>= 1) c[d] += __shfl_xor_sync(0xffffffffu, c[d], m);
  const bool hist = *xtt_ok != 0;
  for (int i = lane; i < nw; i += 32) {
    const int b = b0 + i;
    float *oi = o + 19 * i;
    for (int d = 0; d < 3; ++d) {
      const double x = X[3 * b + d], xt = Xt[3 * b + d];
      oi[d] = (float)(x - c[d] / nw);
      oi[7 + d] = (float)((x - xt) * inv_dt);
      oi[10 + d] = (float)(U[3 * b + d] * inv_dt);
      oi[13 + d] = (float)(Ut[3 * b + d] * inv_dt);
      oi[16 + d] = hist ? (float)((x - 2 * xt + Xtt[3 * b + d]) * inv_dt * inv_dt) : 0.f;
    }
    for (int d = 0; d < 4; ++d) oi[3 + d] = (float)q[4 * b + d];
  }
  const int l0 = b0 - f;
  for (int j = lane; j < nw - 1; j += 32) {
    float *oj = o + 19 * nw + 9 * j;
    for (int d = 0; d < 3; ++d) {
      oj[d] = (float)lam[3 * (l0 + j) + d];
      oj[3 + d] = (float)lam1[3 * (l0 + j) + d];
      oj[6 + d] = (float)lam2[3 * (l0 + j) + d];
    }
  }
  if (lane == 0) o[nfeat - 1] = (float)log(kap[f]);
}

// normalised BF16 inputs [cap x k_in] and (optionally) their transpose [k_in x cap]
__global__ void k_prep_input(const float *__restrict__ raw, int n, int cap, int nfeat, int k_in,
                             const float *__restrict__ mu, const float *__restrict__ sd, fs_bf16 *__restrict__ X,
                             fs_bf16 *__restrict__ XT) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)cap * k_in) return;
  const int row = (int)(idx % cap), col = (int)(idx / cap);
  float v = (row < n && col < nfeat) ? (raw[(size_t)row * nfeat + col] - mu[col]) / sd[col] : 0.f;
  v = isfinite(v) ? fminf(fmaxf(v, -NORM_CLIP), NORM_CLIP) : 0.f;
  const fs_bf16 h = __float2bfloat16_rn(v);
  X[(size_t)row * k_in + col] = h;
  if (XT) XT[idx] = h;
}

__global__ void k_prep_target(const float *__restrict__ raw, int n, int cap, int ntgt, int k_out,
                              const float *__restrict__ mu, const float *__restrict__ sd, float *__restrict__ T) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)cap * k_out) return;
  const int row = (int)(idx / k_out), col = (int)(idx % k_out);
  const float v = (row < n && col < ntgt) ? (raw[(size_t)row * ntgt + col] - mu[col]) / sd[col] : 0.f;
  T[idx] = isfinite(v) ? fminf(fmaxf(v, -NORM_CLIP), NORM_CLIP) : 0.f;
}

// mean-square loss over the valid rows and targets; dY = d loss / d Y in BF16 and transposed
__global__ void k_loss_grad(const float *__restrict__ Y, const float *__restrict__ T, int n, int cap, int ntgt,
                            int k_out, float scale, fs_bf16 *__restrict__ dY, fs_bf16 *__restrict__ dYT,
                            double *__restrict__ loss) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double sq = 0.0;
  if (idx < (size_t)cap * k_out) {
    const int row = (int)(idx % cap), col = (int)(idx / cap);
    float d = 0.f;
    if (row < n && col < ntgt) d = Y[(size_t)row * k_out + col] - T[(size_t)row * k_out + col];
    const fs_bf16 g = __float2bfloat16_rn(2.f * d * scale);
    dY[(size_t)row * k_out + col] = g;
    dYT[idx] = g;
    sq = (double)d * d;
  }
  for (int m = 16; m >= 1; m >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, m);
  __shared__ double part[8];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += part[w];
    atomicAdd(loss, s * scale);
  }
}

// out[r] = sum_m MT[r][m] (bias gradients from the transposed layer gradients)
__global__ void k_rowsum(const fs_bf16 *__restrict__ MT, int rows, int cap, float *__restrict__ out) {
  const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (r >= rows) return;
  float s = 0.f;
  for (int m = lane; m < cap; m += 32) s += __bfloat162float(MT[(size_t)r * cap + m]);
  for (int k = 16; k >= 1; k >>= 1) s += __shfl_xor_sync(0xffffffffu, s, k);
  if (lane == 0) out[r] = s;
}

// Adam step; refreshes the BF16 copy [rows x cols] and its transpose
__global__ void k_adam(float *__restrict__ P, const float *__restrict__ G, float *__restrict__ m, float *__restrict__ v,
                       int n, float lr, float b1, float b2, float eps, float bc1, float bc2, int rows, int cols,
                       fs_bf16 *__restrict__ Pb, fs_bf16 *__restrict__ PTb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = isfinite(G[i]) ? G[i] : 0.f;
  const float mi = b1 * m[i] + (1.f - b1) * g, vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float p = P[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  P[i] = p;
  if (Pb) {
    const fs_bf16 h = __float2bfloat16_rn(p);
    Pb[i] = h;
    PTb[(size_t)(i % cols) * rows + i / cols] = h;
  }
}

__global__ void k_bf16_copies(const float *__restrict__ P, int rows, int cols, fs_bf16 *__restrict__ Pb,
                              fs_bf16 *__restrict__ PTb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const fs_bf16 h = __float2bfloat16_rn(P[i]);
  Pb[i] = h;
  PTb[(size_t)(i % cols) * rows + i / cols] = h;
}

// denormalised outputs of the first n rows
__global__ void k_denorm(const float *__restrict__ Y, int n, int ntgt, int k_out, const float *__restrict__ mu,
                         const float *__restrict__ sd, float *__restrict__ out) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)n * ntgt) return;
  const int row = (int)(idx / ntgt), col = (int)(idx % ntgt);
  out[idx] = Y[(size_t)row * k_out + col] * sd[col] + mu[col];
}

// learned start: upd = -delta (state -= upd), jdiag = diagonal correction
// (plain: per filament, nonzero = keep the plain start this step, or NULL)
__global__ void k_learn_apply(int nfil, const int *__restrict__ fil_start, int nw_model, int ntgt,
                              const float *__restrict__ pred, const int *__restrict__ plain,
                              double *__restrict__ upd, double *__restrict__ jdiag) {
  const int f = blockIdx.x;
  const int b0 = fil_start[f], nw = fil_start[f + 1] - b0;
  const bool model = nw == nw_model && !(plain && plain[f]);
  for (int t = threadIdx.x; t < 6 * nw; t += blockDim.x) {
    const float u = model ? pred[(size_t)f * ntgt + t] : 0.f;
    upd[6 * (size_t)b0 + t] = isfinite(u) ? -(double)u : 0.0;  // a non-finite output is no update
    if (jdiag) {
      const float d = model ? pred[(size_t)f * ntgt + 6 * nw + t] : 0.f;
      jdiag[6 * (size_t)b0 + t] = isfinite(d) ? (double)d : 0.0;
    }
  }
}

// per-filament max |E| (non-finite counts as infinite)
__global__ void k_fil_maxabs(int nfil, const int *__restrict__ fil_start, const double *__restrict__ err,
                             float *__restrict__ r) {
  const int f = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (f >= nfil) return;
  const int b0 = fil_start[f], nw = fil_start[f + 1] - b0;
  double mx = 0.0;
  for (int t = lane; t < 6 * nw; t += 32) {
    const double e = fabs(err[6 * (size_t)b0 + t]);
    mx = (e > mx || e != e) ? (e != e ? INFINITY : e) : mx;
  }
  for (int m = 16; m >= 1; m >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, m));
  if (lane == 0) r[f] = (float)mx;
}

// carried steps: a filament whose learned first residual exceeds the carried
// plain one takes the plain start from the next step on; counts those that
// started plain this step
__global__ void k_flag_worse(int nfil, const int *__restrict__ fil_start, int nw_model, const float *__restrict__ rP,
                             const float *__restrict__ rL, int *__restrict__ plain, int *__restrict__ count) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nfil || fil_start[f + 1] - fil_start[f] != nw_model) return;
  if (plain[f]) atomicAdd(count, 1);
  else if (rL[f] > rP[f]) plain[f] = 1;
}

// filaments whose learned start is worse go back to the plain guess
__global__ void k_fallback(int nfil, const int *__restrict__ fil_start, int nw_model, const float *__restrict__ rP,
                           const float *__restrict__ rL, const double *__restrict__ gXs, const double *__restrict__ gUs,
                           const double *__restrict__ gqs, const double *__restrict__ glam, double *__restrict__ Xs,
                           double *__restrict__ Us, double *__restrict__ qs, double *__restrict__ lam,
                           int *__restrict__ count) {
  const int f = blockIdx.x;
  const int b0 = fil_start[f], nw = fil_start[f + 1] - b0, l0 = b0 - f;
  if (nw != nw_model || !(rL[f] > rP[f])) return;
  for (int t = threadIdx.x; t < 3 * nw; t += blockDim.x) {
    Xs[3 * (size_t)b0 + t] = gXs[3 * (size_t)b0 + t];
    Us[3 * (size_t)b0 + t] = gUs[3 * (size_t)b0 + t];
  }
  for (int t = threadIdx.x; t < 4 * nw; t += blockDim.x) qs[4 * (size_t)b0 + t] = gqs[4 * (size_t)b0 + t];
  for (int t = threadIdx.x; t < 3 * (nw - 1); t += blockDim.x) lam[3 * (size_t)l0 + t] = glam[3 * (size_t)l0 + t];
  if (threadIdx.x == 0) atomicAdd(count, 1);
}

// training targets of the converged step: the update from the guess in the
// solver's coordinates and the diagonal of the accumulated Broyden correction
__global__ void k_targets(int nfil, const int *__restrict__ fil_start, int nw_model, int ntgt,
                          const double *__restrict__ Xs, const double *__restrict__ Us, const double *__restrict__ lam,
                          const double *__restrict__ gXs, const double *__restrict__ gUs,
                          const double *__restrict__ glam, const double *__restrict__ C, const double *__restrict__ D,
                          int iters, const int *__restrict__ off, size_t n6, float *__restrict__ tgt) {
  const int f = blockIdx.x;
  const int b0 = fil_start[f], nw = fil_start[f + 1] - b0, l0 = b0 - f;
  for (int t = threadIdx.x; t < ntgt; t += blockDim.x) {
    float v = 0.f;
    if (nw == nw_model) {
      if (t < 3) {
        v = (float)(Xs[3 * (size_t)b0 + t] - gXs[3 * (size_t)b0 + t]);
      } else if (t < 3 + 3 * nw) {
        v = (float)(Us[3 * (size_t)b0 + t - 3] - gUs[3 * (size_t)b0 + t - 3]);
      } else if (t < 6 * nw) {
        const size_t j = 3 * (size_t)l0 + (t - 3 - 3 * nw);
        v = (float)(lam[j] - glam[j]);
      } else if (t < 12 * nw) {
        const size_t r = 6 * (size_t)b0 + (t - 6 * nw);
        double s = 0.0;
        const int ncol = iters + (off ? *off : 0);  // off: the column count with the Broyden memory on
        for (int i = 0; i < ncol; ++i) s += C[(size_t)i * n6 + r] * D[(size_t)i * n6 + r];
        v = (float)s;
      }
    }
    tgt[(size_t)f * ntgt + t] = v;
  }
}

__global__ void k_diag_axpy(size_t n, const double *__restrict__ d, const double *__restrict__ b, double *__restrict__ x) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += d[i] * b[i];
}

// ---- helpers -------------------------------------------------------------------------
template <typename T>
fs_status dalloc(T **p, size_t n, size_t *bytes) {
  FS_CUDA(cudaMalloc(p, sizeof(T) * (n > 0 ? n : 1)));
  *bytes += sizeof(T) * n;
  return FS_OK;
}

// TMA descriptor of a row-major BF16 matrix [rows x cols] (leading dimension ld
// elements) read in 64-column x 128-row boxes with the 128-byte swizzle; the
// encoder comes from the CUDA driver API through the runtime (no link against libcuda).
// A descriptor is a function of (address, rows, cols, ld) only, so encoded ones
// are kept in a small process-wide cache (the MLP's GEMMs reuse the same
// operands every call; encoding costs tens of microseconds on the host).
struct TmaCacheEntry {
  const void *ptr;
  int rows, cols, ld;
  CUtensorMap map;
};
constexpr int TMA_CACHE_SIZE = 128;

fs_status tma_map_bf16(CUtensorMap *map, const fs_bf16 *ptr, int rows, int cols, int ld) {
  static std::mutex mu;
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  static std::vector<TmaCacheEntry> cache;
  static size_t next_slot = 0;
  if (((uintptr_t)ptr & 15) || ((size_t)ld * sizeof(fs_bf16)) % 16) return FS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(mu);
  for (const TmaCacheEntry &e : cache)
    if (e.ptr == ptr && e.rows == rows && e.cols == cols && e.ld == ld) {
      *map = e.map;
      return FS_OK;
    }
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return FS_ERR_CUDA;
    encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(fs_bf16)};
  const cuuint32_t box[2] = {(cuuint32_t)fsg::BK, 128u};
  const cuuint32_t estr[2] = {1u, 1u};
  if (encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<fs_bf16 *>(ptr), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return FS_ERR_CUDA;
  const TmaCacheEntry e{ptr, rows, cols, ld, *map};
  if ((int)cache.size() < TMA_CACHE_SIZE) {
    cache.push_back(e);
  } else {
    cache[next_slot] = e;
    next_slot = (next_slot + 1) % TMA_CACHE_SIZE;
  }
  return FS_OK;
}

template <int EPI>
fs_status gemm(cudaStream_t st, const GemmArgs &g) {
  if (g.M % fsg::BM || g.N % 128 || g.K % fsg::BK || g.K <= 0) return FS_ERR_INVALID_ARG;
  CUtensorMap ta, tb;
  FS_TRY(tma_map_bf16(&ta, g.A, g.M, g.K, g.lda));
  FS_TRY(tma_map_bf16(&tb, g.B, g.N, g.K, g.ldb));
  dim3 grid(g.M / fsg::BM, g.N / 128);
  fsg::k_gemm_bf16<128, EPI><<<grid, fsg::THREADS, fsg::smem_bytes<128>(), st>>>(g, ta, tb);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

GemmArgs gargs(const fs_bf16 *A, int lda, const fs_bf16 *B, int ldb, int M, int N, int K, int *err) {
  GemmArgs g;
  memset(&g, 0, sizeof g);
  g.A = A;
  g.B = B;
  g.lda = lda;
  g.ldb = ldb;
  g.M = M;
  g.N = N;
  g.K = K;
  g.err = err;
  return g;
}

fs_status gemm_attrs() {
  const int s = fsg::smem_bytes<128>();
  FS_CUDA(cudaFuncSetAttribute(fsg::k_gemm_bf16<128, GEMM_EPI_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, s));
  FS_CUDA(cudaFuncSetAttribute(fsg::k_gemm_bf16<128, GEMM_EPI_SILU>, cudaFuncAttributeMaxDynamicSharedMemorySize, s));
  FS_CUDA(cudaFuncSetAttribute(fsg::k_gemm_bf16<128, GEMM_EPI_DSILU>, cudaFuncAttributeMaxDynamicSharedMemorySize, s));
  return FS_OK;
}

uint64_t splitmix(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

fs_status check_err(fs_ctx *c) {
  int e = 0;
  FS_CUDA(cudaMemcpyAsync(&e, c->mlp->err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaStreamSynchronize(c->stream));
  return e ? FS_ERR_CUDA : FS_OK;
}

// forward pass of rows [0, n) of m->X (already prepared); train: keep transposes
fs_status forward(fs_ctx *c, int n_rows, bool train) {
  fs_mlp *m = c->mlp;
  const int cap = m->cap;
  (void)n_rows;
  const fs_bf16 *in = m->X;
  int kin = m->k_in;
  for (int l = 0; l < 3; ++l) {
    GemmArgs g = gargs(in, kin, m->Wb[l], kin, cap, m->hidden, kin, m->err);
    g.bias = m->b[l];
    g.aux = m->Z[l];
    g.ldx = m->hidden;
    g.outH = m->H[l];
    g.ldh = m->hidden;
    g.outT = train ? m->HT[l] : nullptr;
    g.ldt = cap;
    FS_TRY(gemm<GEMM_EPI_SILU>(c->stream, g));
    in = m->H[l];
    kin = m->hidden;
  }
  GemmArgs g = gargs(in, kin, m->Wb[3], kin, cap, m->k_out, kin, m->err);
  g.bias = m->b[3];
  g.outF = m->Y;
  g.ldo = m->k_out;
  return gemm<GEMM_EPI_F32>(c->stream, g);
}

// gradients of the mean-square loss for the prepared batch (m->X, m->XT, m->T)
fs_status backward(fs_ctx *c, int n) {
  fs_mlp *m = c->mlp;
  const int cap = m->cap, h = m->hidden;
  FS_CUDA(cudaMemsetAsync(m->loss, 0, sizeof(double), c->stream));
  const float scale = 1.0f / ((float)n * (float)m->ntgt);
  k_loss_grad<<<fs_blocks((long long)cap * m->k_out, 256), 256, 0, c->stream>>>(m->Y, m->T, n, cap, m->ntgt, m->k_out,
                                                                               scale, m->dY, m->dYT, m->loss);
  FS_LAUNCH_CHECK();
  // layer 4
  {
    GemmArgs g = gargs(m->dYT, cap, m->HT[2], cap, m->k_out, h, cap, m->err);
    g.outF = m->dW[3];
    g.ldo = h;
    FS_TRY(gemm<GEMM_EPI_F32>(c->stream, g));
    k_rowsum<<<fs_blocks(m->k_out, 8), 256, 0, c->stream>>>(m->dYT, m->k_out, cap, m->db[3]);
    FS_LAUNCH_CHECK();
  }
  const fs_bf16 *gin = m->dY;
  int kg = m->k_out;
  for (int l = 2; l >= 0; --l) {
    // dZ_l = (g_{l+1} W_{l+1}) * silu'(Z_l)
    GemmArgs g = gargs(gin, kg, m->WTb[l + 1], kg, cap, h, kg, m->err);
    g.aux = m->Z[l];
    g.ldx = h;
    g.outH = m->dZ[l];
    g.ldh = h;
    g.outT = m->dZT[l];
    g.ldt = cap;
    FS_TRY(gemm<GEMM_EPI_DSILU>(c->stream, g));
    // dW_l = dZ_l^T x input_l
    const fs_bf16 *inT = l == 0 ? m->XT : m->HT[l - 1];
    const int kin = l == 0 ? m->k_in : h;
    GemmArgs gw = gargs(m->dZT[l], cap, inT, cap, h, kin, cap, m->err);
    gw.outF = m->dW[l];
    gw.ldo = kin;
    FS_TRY(gemm<GEMM_EPI_F32>(c->stream, gw));
    k_rowsum<<<fs_blocks(h, 8), 256, 0, c->stream>>>(m->dZT[l], h, cap, m->db[l]);
    FS_LAUNCH_CHECK();
    gin = m->dZ[l];
    kg = h;
  }
  return FS_OK;
}

fs_status prepare(fs_ctx *c, const float *feat, const float *tgt, int n, bool train) {
  fs_mlp *m = c->mlp;
  k_prep_input<<<fs_blocks((long long)m->cap * m->k_in, 256), 256, 0, c->stream>>>(
      feat, n, m->cap, m->nfeat, m->k_in, m->in_mu, m->in_sd, m->X, train ? m->XT : nullptr);
  FS_LAUNCH_CHECK();
  if (tgt) {
    k_prep_target<<<fs_blocks((long long)m->cap * m->k_out, 256), 256, 0, c->stream>>>(
        tgt, n, m->cap, m->ntgt, m->k_out, m->out_mu, m->out_sd, m->T);
    FS_LAUNCH_CHECK();
  }
  return FS_OK;
}

// predictions (denormalised) for n rows of raw features, in chunks of the capacity
fs_status predict(fs_ctx *c, const float *feat, int n, float *out) {
  fs_mlp *m = c->mlp;
  for (int r0 = 0; r0 < n; r0 += m->cap) {
    const int rows = n - r0 < m->cap ? n - r0 : m->cap;
    FS_TRY(prepare(c, feat + (size_t)r0 * m->nfeat, nullptr, rows, false));
    FS_TRY(forward(c, rows, false));
    k_denorm<<<fs_blocks((long long)rows * m->ntgt, 256), 256, 0, c->stream>>>(m->Y, rows, m->ntgt, m->k_out,
                                                                               m->out_mu, m->out_sd,
                                                                               out + (size_t)r0 * m->ntgt);
    FS_LAUNCH_CHECK();
  }
  return FS_OK;
}

size_t param_count(const fs_mlp *m) {
  size_t n = 0;
  for (int l = 0; l < 4; ++l) n += (size_t)m->dims[l + 1] * m->dims[l] + m->dims[l + 1];
  return n;
}

fs_status ensure_step_buffers(fs_ctx *c) {
  fs_mlp *m = c->mlp;
  if (m->nfil_alloc >= c->nfil && m->np_alloc >= c->np && m->gXs) return FS_OK;
  cudaFree(m->gXs);
  cudaFree(m->gUs);
  cudaFree(m->gqs);
  cudaFree(m->glam);
  cudaFree(m->updl);
  cudaFree(m->jdiag);
  cudaFree(m->feat);
  cudaFree(m->pred);
  cudaFree(m->tgt);
  cudaFree(m->rP);
  cudaFree(m->rL);
  cudaFree(m->plain_next);
  const size_t np = c->max_beads, nf = c->max_fil;
  size_t b = 0;
  FS_TRY(dalloc(&m->gXs, 3 * np, &b));
  FS_TRY(dalloc(&m->gUs, 3 * np, &b));
  FS_TRY(dalloc(&m->gqs, 4 * np, &b));
  FS_TRY(dalloc(&m->glam, 3 * np, &b));
  FS_TRY(dalloc(&m->updl, 6 * np, &b));
  FS_TRY(dalloc(&m->jdiag, 6 * np, &b));
  FS_TRY(dalloc(&m->feat, nf * m->nfeat, &b));
  FS_TRY(dalloc(&m->pred, nf * m->ntgt, &b));
  FS_TRY(dalloc(&m->tgt, nf * m->ntgt, &b));
  FS_TRY(dalloc(&m->rP, nf, &b));
  FS_TRY(dalloc(&m->rL, nf, &b));
  FS_TRY(dalloc(&m->plain_next, nf, &b));
  m->bound_ok = false;
  m->nfil_alloc = (int)nf;
  m->np_alloc = (int)np;
  c->bytes += b;
  return FS_OK;
}

}  // namespace

// ---- internal entry points used by the step driver -----------------------------------
bool learn_active(const fs_ctx *c) { return c->mlp && c->mlp->mode > 0; }

// the start of this step under the cost gate (true: learned)
constexpr int GATE_BACKOFF_MAX = 16;
// the learned start is chosen only when its running mean is at least gate_margin
// mobility solves per step below the plain start's (its inference and its
// host-driven step cost about a quarter of a 512^3 solve): a tie goes to the
// reference's start, which also runs as a captured step graph; and only once
// its mean rests on at least this many steps (one early step says little)
constexpr long long GATE_MIN_STEPS = 2;

int gate_best(const fs_mlp *m) {
  return m->gate_steps[1] >= GATE_MIN_STEPS && m->gate_solves[1] + m->gate_margin <= m->gate_solves[0] ? 1 : 0;
}

bool learn_gate_on(const fs_ctx *c) { return c->mlp && c->mlp->gate_period > 0; }

bool learn_gate_choose(fs_ctx *c) {
  fs_mlp *m = c->mlp;
  if (!m->gate_period) return true;
  if (!m->gate_have[0]) return false;
  if (!m->gate_have[1]) {  // first learned step: a probe against the plain start
    m->gate_since = 0;
    m->gate_probe_best = 0;
    return true;
  }
  const int best = gate_best(m);
  if (++m->gate_since >= m->gate_interval) {
    m->gate_since = 0;
    m->gate_probe_best = best;
    return best == 0;
  }
  return best == 1;
}

void learn_gate_record(fs_ctx *c, bool learned, long long solves) {
  fs_mlp *m = c->mlp;
  const int i = learned ? 1 : 0;
  m->gate_solves[i] = m->gate_have[i] ? 0.7 * m->gate_solves[i] + 0.3 * (double)solves : (double)solves;
  m->gate_have[i] = 1;
  m->gate_steps[i]++;
  if (m->gate_probe_best >= 0) {
    const bool kept = gate_best(m) == m->gate_probe_best;
    m->gate_interval = kept ? std::min(2 * m->gate_interval, GATE_BACKOFF_MAX * m->gate_period) : m->gate_period;
    m->gate_probe_best = -1;
  }
}
bool learn_recording(const fs_ctx *c) { return c->mlp && c->mlp->record; }

// after fil_initial_guess: keep the plain guess (for the fallback and the targets)
fs_status learn_save_guess(fs_ctx *c) {
  fs_mlp *m = c->mlp;
  FS_TRY(ensure_step_buffers(c));
  FS_CUDA(cudaMemcpyAsync(m->gXs, c->Xs, sizeof(double) * 3 * c->np, cudaMemcpyDeviceToDevice, c->stream));
  FS_CUDA(cudaMemcpyAsync(m->gUs, c->Us, sizeof(double) * 3 * c->np, cudaMemcpyDeviceToDevice, c->stream));
  FS_CUDA(cudaMemcpyAsync(m->gqs, c->qs, sizeof(double) * 4 * c->np, cudaMemcpyDeviceToDevice, c->stream));
  if (c->nlink > 0)
    FS_CUDA(cudaMemcpyAsync(m->glam, c->lam, sizeof(double) * 3 * c->nlink, cudaMemcpyDeviceToDevice, c->stream));
  return FS_OK;
}

fs_status learn_features(fs_ctx *c, float *out) {
  fs_mlp *m = c->mlp;
  FS_TRY(ensure_step_buffers(c));
  k_features<<<fs_blocks(c->nfil, 8), 256, 0, c->stream>>>(c->nfil, c->fil_start, m->nw, c->X, c->Xt, c->hist_Xtt, c->hist_ok,
                                                           c->q, c->U, c->Ut, c->lam, c->lam1, c->lam2, c->kap,
                                                           1.0 / c->p.dt, m->nfeat, out);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

// The start of the Broyden iteration: on return c->err holds the residual of the
// chosen start and c->flags its tolerance test (main.cpp:556-566 for the plain start).
fs_status learn_warm_start(fs_ctx *c, int nt, fs_status (*solve)(fs_ctx *, int)) {
  fs_mlp *m = c->mlp;
  {
    ProfScope ps(c, FS_STAGE_LEARN);
    if (m->override_next) {
      m->override_next = false;
    } else {
      FS_TRY(learn_features(c, m->feat));
      FS_TRY(predict(c, m->feat, c->nfil, m->pred));
    }
  }
  const bool carried = m->bound_refresh > 0 && m->bound_ok && m->bound_age < m->bound_refresh;
  {
    ProfScope ps(c, FS_STAGE_LEARN);
    k_learn_apply<<<c->nfil, 128, 0, c->stream>>>(c->nfil, c->fil_start, m->nw, m->ntgt, m->pred,
                                                  carried ? m->plain_next : nullptr, m->updl,
                                                  m->mode == 2 ? m->jdiag : nullptr);
    FS_LAUNCH_CHECK();
    m->jdiag_on = m->mode == 2;
  }
  if (carried) {
    // one solve: the learned start (the plain guess for the flagged filaments),
    // checked per filament against rP, the plain start's residual of the last
    // comparison step; a filament found worse takes the plain start from the
    // next step on, and its residual stands for this step
    ++m->bound_age;
    FS_TRY(fil_state_update(c, m->updl));
    FS_TRY(fil_forces(c, nt));
    FS_TRY(solve(c, nt));
    FS_TRY(fil_error_check(c, c->V, c->W, c->err, nt));
    k_fil_maxabs<<<fs_blocks(c->nfil, 8), 256, 0, c->stream>>>(c->nfil, c->fil_start, c->err, m->rL);
    FS_LAUNCH_CHECK();
    FS_CUDA(cudaMemsetAsync(m->count, 0, sizeof(int), c->stream));
    k_flag_worse<<<fs_blocks(c->nfil, 128), 128, 0, c->stream>>>(c->nfil, c->fil_start, m->nw, m->rP, m->rL,
                                                                 m->plain_next, m->count);
    FS_LAUNCH_CHECK();
    FS_CUDA(cudaMemcpyAsync(m->count_h, m->count, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FS_CUDA(cudaStreamSynchronize(c->stream));
    int nmodel = 0;
    for (int f = 0; f < c->nfil; ++f) nmodel += (c->fil_start_h[f + 1] - c->fil_start_h[f]) == m->nw;
    const int back = *m->count_h;
    m->fallback_total += back;
    m->learned_total += nmodel - back;
    c->diag.learned_filaments += nmodel - back;
    c->diag.fallback_filaments += back;
    return FS_OK;
  }
  {
    // plain start, measured: the comparison of this step and the bound of the next ones
    FS_TRY(solve(c, nt));
    FS_TRY(fil_error_check(c, c->V, c->W, c->err, nt));
    k_fil_maxabs<<<fs_blocks(c->nfil, 8), 256, 0, c->stream>>>(c->nfil, c->fil_start, c->err, m->rP);
    FS_LAUNCH_CHECK();
    if (m->bound_refresh > 0) {
      m->bound_ok = true;
      m->bound_age = 0;
      FS_CUDA(cudaMemsetAsync(m->plain_next, 0, sizeof(int) * c->nfil, c->stream));
    }
  }
  // learned start
  FS_TRY(fil_state_update(c, m->updl));
  FS_TRY(fil_forces(c, nt));
  FS_TRY(solve(c, nt));
  FS_TRY(fil_error_check(c, c->V, c->W, c->newerr, nt));
  k_fil_maxabs<<<fs_blocks(c->nfil, 8), 256, 0, c->stream>>>(c->nfil, c->fil_start, c->newerr, m->rL);
  FS_LAUNCH_CHECK();
  FS_CUDA(cudaMemsetAsync(m->count, 0, sizeof(int), c->stream));
  k_fallback<<<c->nfil, 128, 0, c->stream>>>(c->nfil, c->fil_start, m->nw, m->rP, m->rL, m->gXs, m->gUs, m->gqs,
                                             m->glam, c->Xs, c->Us, c->qs, c->lam, m->count);
  FS_LAUNCH_CHECK();
  FS_CUDA(cudaMemcpyAsync(m->count_h, m->count, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaStreamSynchronize(c->stream));
  int nmodel = 0;
  for (int f = 0; f < c->nfil; ++f) nmodel += (c->fil_start_h[f + 1] - c->fil_start_h[f]) == m->nw;
  const int back = *m->count_h;
  m->fallback_total += back;
  m->learned_total += nmodel - back;
  c->diag.learned_filaments += nmodel - back;
  c->diag.fallback_filaments += back;
  if (back == 0) {
    std::swap(c->err, c->newerr);  // the learned start's residual and flags stand
    return FS_OK;
  }
  // some filaments went back: residual of the mixed start
  FS_TRY(fil_forces(c, nt));
  FS_TRY(solve(c, nt));
  return fil_error_check(c, c->V, c->W, c->err, nt);
}

// before a graph capture: the learn module's per-step work must not allocate.
// A captured step is a plain-start step (with the learned start on, the cost
// gate's plain steps); it holds no learned-start work, and recording steps,
// which capture targets per step, are never captured.
fs_status learn_prepare_capture(fs_ctx *c) {
  if (!c->mlp) return FS_OK;
  if (c->mlp->record || c->mlp->jdiag_on) return FS_ERR_STATE;
  return ensure_step_buffers(c);
}

fs_status learn_diag_apply(fs_ctx *c, const double *b, double *x) {
  fs_mlp *m = c->mlp;
  if (!m || !m->jdiag_on) return FS_OK;
  const size_t n6 = (size_t)6 * c->np;
  k_diag_axpy<<<fs_blocks((long long)n6, 256), 256, 0, c->stream>>>(n6, m->jdiag, b, x);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

fs_status learn_capture_targets(fs_ctx *c, int iters) {
  fs_mlp *m = c->mlp;
  k_targets<<<c->nfil, 128, 0, c->stream>>>(c->nfil, c->fil_start, m->nw, m->ntgt, c->Xs, c->Us, c->lam, m->gXs,
                                            m->gUs, m->glam, c->Cmat, c->Dmat, bmem_off(c) ? 0 : iters, bmem_off(c),
                                            (size_t)6 * c->np, m->tgt);
  FS_LAUNCH_CHECK();
  m->have_targets = true;
  return FS_OK;
}

// before Filament::step of every step (also before a captured plain-start step,
// whose graph ends with it); the position history is kept by hist_end_step
fs_status learn_end_step(fs_ctx *c) {
  fs_mlp *m = c->mlp;
  if (!m) return FS_OK;
  m->jdiag_on = false;
  return FS_OK;
}

// before fs_state_upload: carried residuals are per filament, so another layout drops them
fs_status learn_before_upload(fs_ctx *c, bool same_layout) {
  fs_mlp *m = c->mlp;
  if (m && !same_layout) m->bound_ok = false;
  return FS_OK;
}

void mlp_free(fs_ctx *c) {
  fs_mlp *m = c->mlp;
  if (!m) return;
  for (int l = 0; l < 4; ++l) {
    cudaFree(m->W[l]);
    cudaFree(m->b[l]);
    cudaFree(m->mW[l]);
    cudaFree(m->vW[l]);
    cudaFree(m->mb[l]);
    cudaFree(m->vb[l]);
    cudaFree(m->dW[l]);
    cudaFree(m->db[l]);
    cudaFree(m->Wb[l]);
    cudaFree(m->WTb[l]);
  }
  for (int l = 0; l < 3; ++l) {
    cudaFree(m->Z[l]);
    cudaFree(m->H[l]);
    cudaFree(m->HT[l]);
    cudaFree(m->dZ[l]);
    cudaFree(m->dZT[l]);
  }
  void *rest[] = {m->in_mu, m->in_sd, m->out_mu, m->out_sd, m->X,   m->XT,   m->Y,    m->T,     m->dY,
                  m->dYT,   m->outbuf, m->loss, m->err,    m->gXs, m->gUs,  m->gqs,  m->glam,  m->updl,
                  m->jdiag, m->feat,  m->pred,  m->tgt,    m->rP,  m->rL,   m->count};
  for (void *p : rest) cudaFree(p);
  if (m->count_h) cudaFreeHost(m->count_h);
  delete m;
  c->mlp = nullptr;
}

// ---- C-ABI ----------------------------------------------------------------------------
extern "C" {

fs_status fs_mlp_create(fs_ctx *c, int nw, int hidden, int batch_capacity, unsigned long long seed) {
  if (!c || nw < 2 || hidden <= 0 || hidden % 128 || batch_capacity <= 0) return FS_ERR_INVALID_ARG;
  mlp_free(c);
  fs_mlp *m = new fs_mlp();
  c->mlp = m;
  m->nw = nw;
  m->nfeat = 19 * nw + 9 * (nw - 1) + 1;
  m->k_in = round_up(m->nfeat, RND);
  m->hidden = hidden;
  m->ntgt = 12 * nw;
  m->k_out = round_up(m->ntgt, RND);
  m->cap = round_up(batch_capacity, RND);
  const int d[5] = {m->k_in, hidden, hidden, hidden, m->k_out};
  for (int i = 0; i < 5; ++i) m->dims[i] = d[i];
  size_t b = 0;
  const int cap = m->cap;
  for (int l = 0; l < 4; ++l) {
    const size_t nW = (size_t)d[l + 1] * d[l], nb = d[l + 1];
    FS_TRY(dalloc(&m->W[l], nW, &b));
    FS_TRY(dalloc(&m->b[l], nb, &b));
    FS_TRY(dalloc(&m->mW[l], nW, &b));
    FS_TRY(dalloc(&m->vW[l], nW, &b));
    FS_TRY(dalloc(&m->mb[l], nb, &b));
    FS_TRY(dalloc(&m->vb[l], nb, &b));
    FS_TRY(dalloc(&m->dW[l], nW, &b));
    FS_TRY(dalloc(&m->db[l], nb, &b));
    FS_TRY(dalloc(&m->Wb[l], nW, &b));
    FS_TRY(dalloc(&m->WTb[l], nW, &b));
    FS_CUDA(cudaMemsetAsync(m->mW[l], 0, sizeof(float) * nW, c->stream));
    FS_CUDA(cudaMemsetAsync(m->vW[l], 0, sizeof(float) * nW, c->stream));
    FS_CUDA(cudaMemsetAsync(m->mb[l], 0, sizeof(float) * nb, c->stream));
    FS_CUDA(cudaMemsetAsync(m->vb[l], 0, sizeof(float) * nb, c->stream));
  }
  for (int l = 0; l < 3; ++l) {
    FS_TRY(dalloc(&m->Z[l], (size_t)cap * hidden, &b));
    FS_TRY(dalloc(&m->H[l], (size_t)cap * hidden, &b));
    FS_TRY(dalloc(&m->HT[l], (size_t)cap * hidden, &b));
    FS_TRY(dalloc(&m->dZ[l], (size_t)cap * hidden, &b));
    FS_TRY(dalloc(&m->dZT[l], (size_t)cap * hidden, &b));
  }
  FS_TRY(dalloc(&m->in_mu, m->k_in, &b));
  FS_TRY(dalloc(&m->in_sd, m->k_in, &b));
  FS_TRY(dalloc(&m->out_mu, m->k_out, &b));
  FS_TRY(dalloc(&m->out_sd, m->k_out, &b));
  FS_TRY(dalloc(&m->X, (size_t)cap * m->k_in, &b));
  FS_TRY(dalloc(&m->XT, (size_t)cap * m->k_in, &b));
  FS_TRY(dalloc(&m->Y, (size_t)cap * m->k_out, &b));
  FS_TRY(dalloc(&m->T, (size_t)cap * m->k_out, &b));
  FS_TRY(dalloc(&m->dY, (size_t)cap * m->k_out, &b));
  FS_TRY(dalloc(&m->dYT, (size_t)cap * m->k_out, &b));
  FS_TRY(dalloc(&m->loss, 1, &b));
  FS_TRY(dalloc(&m->err, 1, &b));
  FS_TRY(dalloc(&m->count, 1, &b));
  FS_CUDA(cudaMallocHost(&m->count_h, sizeof(int)));
  FS_CUDA(cudaMemsetAsync(m->err, 0, sizeof(int), c->stream));
  c->bytes += b;
  FS_TRY(hist_ensure(c));  // the features' acceleration needs the positions two steps back
  graph_invalidate(c);     // captured steps must now keep that history
  // identity normalisation until the caller sets the data's
  std::vector<float> zeros(m->k_in > m->k_out ? m->k_in : m->k_out, 0.f), ones(zeros.size(), 1.f);
  FS_CUDA(cudaMemcpy(m->in_mu, zeros.data(), sizeof(float) * m->k_in, cudaMemcpyHostToDevice));
  FS_CUDA(cudaMemcpy(m->in_sd, ones.data(), sizeof(float) * m->k_in, cudaMemcpyHostToDevice));
  FS_CUDA(cudaMemcpy(m->out_mu, zeros.data(), sizeof(float) * m->k_out, cudaMemcpyHostToDevice));
  FS_CUDA(cudaMemcpy(m->out_sd, ones.data(), sizeof(float) * m->k_out, cudaMemcpyHostToDevice));
  // Linear-layer initialisation: uniform in +-1/sqrt(fan_in) (seeded splitmix64)
  uint64_t s = seed;
  std::vector<float> hbuf;
  for (int l = 0; l < 4; ++l) {
    const size_t nW = (size_t)d[l + 1] * d[l];
    const float bound = 1.0f / sqrtf((float)(l == 0 ? m->nfeat : d[l]));
    hbuf.resize(nW);
    for (size_t i = 0; i < nW; ++i) {
      const int col = (int)(i % d[l]);
      const double u = (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
      hbuf[i] = (l == 0 && col >= m->nfeat) ? 0.f : (float)((2 * u - 1) * bound);
    }
    FS_CUDA(cudaMemcpy(m->W[l], hbuf.data(), sizeof(float) * nW, cudaMemcpyHostToDevice));
    hbuf.resize(d[l + 1]);
    for (int i = 0; i < d[l + 1]; ++i) {
      const double u = (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
      hbuf[i] = (float)((2 * u - 1) * bound);
    }
    FS_CUDA(cudaMemcpy(m->b[l], hbuf.data(), sizeof(float) * d[l + 1], cudaMemcpyHostToDevice));
    k_bf16_copies<<<fs_blocks((long long)nW, 256), 256, 0, c->stream>>>(m->W[l], d[l + 1], d[l], m->Wb[l], m->WTb[l]);
    FS_LAUNCH_CHECK();
  }
  FS_TRY(gemm_attrs());
  FS_CUDA(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_mlp_dims(const fs_ctx *c, int *dims_h) {
  if (!c || !c->mlp || !dims_h) return FS_ERR_INVALID_ARG;
  const fs_mlp *m = c->mlp;
  const int v[8] = {m->nw, m->nfeat, m->k_in, m->hidden, m->ntgt, m->k_out, m->cap, (int)param_count(m)};
  memcpy(dims_h, v, sizeof v);
  return FS_OK;
}

fs_status fs_mlp_set_normalization(fs_ctx *c, const float *in_mean_h, const float *in_std_h, const float *out_mean_h,
                                   const float *out_std_h) {
  if (!c || !c->mlp || !in_mean_h || !in_std_h || !out_mean_h || !out_std_h) return FS_ERR_INVALID_ARG;
  fs_mlp *m = c->mlp;
  FS_CUDA(cudaMemcpy(m->in_mu, in_mean_h, sizeof(float) * m->nfeat, cudaMemcpyHostToDevice));
  FS_CUDA(cudaMemcpy(m->in_sd, in_std_h, sizeof(float) * m->nfeat, cudaMemcpyHostToDevice));
  FS_CUDA(cudaMemcpy(m->out_mu, out_mean_h, sizeof(float) * m->ntgt, cudaMemcpyHostToDevice));
  FS_CUDA(cudaMemcpy(m->out_sd, out_std_h, sizeof(float) * m->ntgt, cudaMemcpyHostToDevice));
  return FS_OK;
}

// flat parameters [W1 b1 W2 b2 W3 b3 W4 b4], W_l row-major [out x in] with the padded widths
fs_status fs_mlp_get_params(fs_ctx *c, float *params_h, size_t count) {
  if (!c || !c->mlp || !params_h || count < param_count(c->mlp)) return FS_ERR_INVALID_ARG;
  fs_mlp *m = c->mlp;
  FS_CUDA(cudaStreamSynchronize(c->stream));
  size_t o = 0;
  for (int l = 0; l < 4; ++l) {
    const size_t nW = (size_t)m->dims[l + 1] * m->dims[l];
    FS_CUDA(cudaMemcpy(params_h + o, m->W[l], sizeof(float) * nW, cudaMemcpyDeviceToHost));
    o += nW;
    FS_CUDA(cudaMemcpy(params_h + o, m->b[l], sizeof(float) * m->dims[l + 1], cudaMemcpyDeviceToHost));
    o += m->dims[l + 1];
  }
  return FS_OK;
}

fs_status fs_mlp_set_params(fs_ctx *c, const float *params_h, size_t count) {
  if (!c || !c->mlp || !params_h || count < param_count(c->mlp)) return FS_ERR_INVALID_ARG;
  fs_mlp *m = c->mlp;
  size_t o = 0;
  for (int l = 0; l < 4; ++l) {
    const size_t nW = (size_t)m->dims[l + 1] * m->dims[l];
    FS_CUDA(cudaMemcpy(m->W[l], params_h + o, sizeof(float) * nW, cudaMemcpyHostToDevice));
    o += nW;
    FS_CUDA(cudaMemcpy(m->b[l], params_h + o, sizeof(float) * m->dims[l + 1], cudaMemcpyHostToDevice));
    o += m->dims[l + 1];
    k_bf16_copies<<<fs_blocks((long long)nW, 256), 256, 0, c->stream>>>(m->W[l], m->dims[l + 1], m->dims[l], m->Wb[l],
                                                                        m->WTb[l]);
    FS_LAUNCH_CHECK();
  }
  m->adam_t = 0;
  for (int l = 0; l < 4; ++l) {
    const size_t nW = (size_t)m->dims[l + 1] * m->dims[l];
    FS_CUDA(cudaMemsetAsync(m->mW[l], 0, sizeof(float) * nW, c->stream));
    FS_CUDA(cudaMemsetAsync(m->vW[l], 0, sizeof(float) * nW, c->stream));
    FS_CUDA(cudaMemsetAsync(m->mb[l], 0, sizeof(float) * m->dims[l + 1], c->stream));
    FS_CUDA(cudaMemsetAsync(m->vb[l], 0, sizeof(float) * m->dims[l + 1], c->stream));
  }
  FS_CUDA(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_mlp_forward(fs_ctx *c, const float *features_d, int n, float *out_d) {
  if (!c || !c->mlp || !features_d || !out_d || n < 0) return FS_ERR_INVALID_ARG;
  FS_TRY(predict(c, features_d, n, out_d));
  return check_err(c);
}

// gradients (flat, the layout of fs_mlp_get_params) and loss of one batch; no update
fs_status fs_mlp_gradients(fs_ctx *c, const float *features_d, const float *targets_d, int n, float *grads_h,
                           size_t count, double *loss_h) {
  if (!c || !c->mlp || !features_d || !targets_d || n <= 0 || n > c->mlp->cap) return FS_ERR_INVALID_ARG;
  fs_mlp *m = c->mlp;
  if (grads_h && count < param_count(m)) return FS_ERR_INVALID_ARG;
  FS_TRY(prepare(c, features_d, targets_d, n, true));
  FS_TRY(forward(c, n, true));
  FS_TRY(backward(c, n));
  FS_TRY(check_err(c));
  if (grads_h) {
    size_t o = 0;
    for (int l = 0; l < 4; ++l) {
      const size_t nW = (size_t)m->dims[l + 1] * m->dims[l];
      FS_CUDA(cudaMemcpy(grads_h + o, m->dW[l], sizeof(float) * nW, cudaMemcpyDeviceToHost));
      o += nW;
      FS_CUDA(cudaMemcpy(grads_h + o, m->db[l], sizeof(float) * m->dims[l + 1], cudaMemcpyDeviceToHost));
      o += m->dims[l + 1];
    }
  }
  if (loss_h) FS_CUDA(cudaMemcpy(loss_h, m->loss, sizeof(double), cudaMemcpyDeviceToHost));
  return FS_OK;
}

// one Adam step on a batch of raw features and targets (device arrays, n rows)
fs_status fs_mlp_train_step(fs_ctx *c, const float *features_d, const float *targets_d, int n, float lr,
                            double *loss_h) {
  if (!c || !c->mlp || !features_d || !targets_d || n <= 0 || n > c->mlp->cap || !(lr > 0)) return FS_ERR_INVALID_ARG;
  fs_mlp *m = c->mlp;
  {
    ProfScope ps(c, FS_STAGE_LEARN);
    FS_TRY(prepare(c, features_d, targets_d, n, true));
    FS_TRY(forward(c, n, true));
    FS_TRY(backward(c, n));
    m->adam_t++;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float bc1 = 1.f - powf(b1, (float)m->adam_t), bc2 = 1.f - powf(b2, (float)m->adam_t);
    for (int l = 0; l < 4; ++l) {
      const int rows = m->dims[l + 1], cols = m->dims[l];
      k_adam<<<fs_blocks((long long)rows * cols, 256), 256, 0, c->stream>>>(
          m->W[l], m->dW[l], m->mW[l], m->vW[l], rows * cols, lr, b1, b2, eps, bc1, bc2, rows, cols, m->Wb[l], m->WTb[l]);
      FS_LAUNCH_CHECK();
      k_adam<<<fs_blocks(rows, 256), 256, 0, c->stream>>>(m->b[l], m->db[l], m->mb[l], m->vb[l], rows, lr, b1, b2, eps,
                                                          bc1, bc2, rows, 1, nullptr, nullptr);
      FS_LAUNCH_CHECK();
    }
  }
  if (loss_h) {
    FS_CUDA(cudaMemcpyAsync(loss_h, m->loss, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    FS_CUDA(cudaStreamSynchronize(c->stream));
    return check_err(c);
  }
  return FS_OK;
}

fs_status fs_learn_features(fs_ctx *c, float *features_d) {
  if (!c || !c->mlp || !features_d) return FS_ERR_INVALID_ARG;
  if (!c->have_state) return FS_ERR_STATE;
  return learn_features(c, features_d);
}

fs_status fs_learn_record(fs_ctx *c, int on) {
  if (!c || !c->mlp) return FS_ERR_INVALID_ARG;
  c->mlp->record = on != 0;
  if (on && c->have_state) FS_TRY(ensure_step_buffers(c));
  return FS_OK;
}

fs_status fs_learn_targets(fs_ctx *c, float *targets_d) {
  if (!c || !c->mlp || !targets_d) return FS_ERR_INVALID_ARG;
  if (!c->mlp->have_targets) return FS_ERR_STATE;
  FS_CUDA(cudaMemcpyAsync(targets_d, c->mlp->tgt, sizeof(float) * c->nfil * c->mlp->ntgt, cudaMemcpyDeviceToDevice,
                          c->stream));
  return FS_OK;
}

fs_status fs_learn_override(fs_ctx *c, const float *pred_d) {
  if (!c || !c->mlp || !pred_d) return FS_ERR_INVALID_ARG;
  if (!c->have_state) return FS_ERR_STATE;
  FS_TRY(ensure_step_buffers(c));
  FS_CUDA(cudaMemcpyAsync(c->mlp->pred, pred_d, sizeof(float) * c->nfil * c->mlp->ntgt, cudaMemcpyDeviceToDevice,
                          c->stream));
  c->mlp->override_next = true;
  return FS_OK;
}

fs_status fs_set_warm_start(fs_ctx *c, int mode) {
  if (!c || mode < 0 || mode > 2) return FS_ERR_INVALID_ARG;
  if (mode > 0 && !c->mlp) return FS_ERR_STATE;
  if (c->mlp) c->mlp->mode = mode;
  return FS_OK;
}

fs_status fs_warm_start_bound(fs_ctx *c, int refresh) {
  if (!c || refresh < 0) return FS_ERR_INVALID_ARG;
  if (!c->mlp) return refresh ? FS_ERR_STATE : FS_OK;
  c->mlp->bound_refresh = refresh;
  c->mlp->bound_ok = false;
  c->mlp->bound_age = 0;
  return FS_OK;
}

fs_status fs_warm_start_gate(fs_ctx *c, int period) {
  if (!c || period < 0) return FS_ERR_INVALID_ARG;
  if (!c->mlp) return period ? FS_ERR_STATE : FS_OK;
  fs_mlp *m = c->mlp;
  m->gate_period = period;
  m->gate_interval = period;
  m->gate_have[0] = m->gate_have[1] = 0;
  m->gate_since = 0;
  m->gate_probe_best = -1;
  m->gate_steps[0] = m->gate_steps[1] = 0;
  return FS_OK;
}

fs_status fs_warm_start_gate_margin(fs_ctx *c, double margin) {
  if (!c || !(margin >= 0.0) || margin > 1e6) return FS_ERR_INVALID_ARG;
  if (!c->mlp) return FS_ERR_STATE;
  c->mlp->gate_margin = margin;
  return FS_OK;
}

fs_status fs_warm_start_gate_stats(fs_ctx *c, long long *steps_h, double *solves_h) {
  if (!c || !steps_h || !solves_h) return FS_ERR_INVALID_ARG;
  for (int i = 0; i < 2; ++i) {
    steps_h[i] = c->mlp ? c->mlp->gate_steps[i] : 0;
    solves_h[i] = (c->mlp && c->mlp->gate_have[i]) ? c->mlp->gate_solves[i] : 0.0;
  }
  return FS_OK;
}

fs_status fs_gemm_bf16(fs_ctx *c, const void *A, const void *B, float *D, int M, int N, int K) {
  if (!c || !A || !B || !D || M <= 0 || N <= 0 || K <= 0) return FS_ERR_INVALID_ARG;
  if (M % fsg::BM || N % 128 || K % fsg::BK) return FS_ERR_INVALID_ARG;
  if (!c->gemm_err) {  // first call: the error word and the kernels' shared-memory limits
    FS_TRY(gemm_attrs());
    FS_CUDA(cudaMalloc(&c->gemm_err, sizeof(int)));
  }
  int *err_d = c->gemm_err;
  FS_CUDA(cudaMemsetAsync(err_d, 0, sizeof(int), c->stream));
  GemmArgs g = gargs((const fs_bf16 *)A, K, (const fs_bf16 *)B, K, M, N, K, err_d);
  g.outF = D;
  g.ldo = N;
  fs_status st = gemm<GEMM_EPI_F32>(c->stream, g);
  int e = 0;
  if (st == FS_OK && cudaMemcpyAsync(&e, err_d, sizeof(int), cudaMemcpyDeviceToHost, c->stream) == cudaSuccess &&
      cudaStreamSynchronize(c->stream) == cudaSuccess && e)
    st = FS_ERR_CUDA;
  return st;
}

}  // extern "C"
