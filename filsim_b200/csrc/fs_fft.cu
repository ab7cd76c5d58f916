// fs_fft.cu -- FP32 periodic Stokes solve on power-of-two grids for sm_100a:
// the forward real 3-D transform, the projection of flow_solve
// (FCMfunctions.cpp:648-736) and the inverse real transform in five passes
// over HBM, replacing cuFFT R2C + projection + C2R in the mixed-precision path.
//
//   f[c][x][y][z] (real)  --z_r2c-->    A[c][kz][x][y]   z lines, real-to-half-complex
//                                                        (two real lines as one complex line)
//                         --y_fwd-->    B[c][kz][ky][x]  y lines, written transposed
//                         --x_project-> B (in place)     x lines: forward, Stokes
//                                                        projection, inverse, with the
//                                                        three components in registers
//                         --y_inv-->    A[c][kz][x][y]
//                         --z_c2r-->    u[c][x][y][z] (real)
// Each pass reads and writes the grid once with 128-byte rows. Every line is
// transformed by one warp in registers: N = 32*M points, M per lane, an
// M-point radix-2 DFT per lane, a transpose through a padded per-warp shared
// buffer, a second M-point DFT and log2(32/M) radix-2 stages across lanes with
// shuffles. Transforms are unnormalised; the projection divides by Nx*Ny*Nz as
// the reference does. The half-complex inverse along z takes only the real part
// of the kz = 0 and kz = Nz/2 coefficients after the complex inverse transforms
// along x and y, the semantics of the reference's multi-dimensional real
// inverse transform. Along z a warp transforms its two real lines a, b as one
// complex line a + i b and separates (or assembles) their half spectra.
#include "fs_internal.cuh"
#include "fs_f32x2.cuh"

namespace {

constexpr int FFT_WARPS = 8;
constexpr int FFT_THREADS = 32 * FFT_WARPS;
constexpr int FFT_TILE = 16;             // lines per transposing tile (16 complex = 128 bytes)
constexpr int FFT_TS = FFT_TILE + 1;     // padded tile row (conflict-free column access)
constexpr int TW_FULL = 1024;            // tw[j] = exp(-2 pi i j / 1024)
#define FULL_MASK 0xffffffffu

// Row of spectrum index k in a shared buffer that receives a warp's output in
// register order (k = c + M k' + M^2 t across lanes): k + (k / M^2) (16 / G)
// spreads the lanes of each half-warp over distinct banks.
template <int N>
__host__ __device__ constexpr int prow(int k) {
  return N == 32 ? k + (k >> 4) : k + (k / ((N / 32) * (N / 32))) * (16 / (32 / (N / 32)));
}

template <int N>
struct Fft {
  static constexpr int M = N / 32;                       // points per lane
  static constexpr int G = 32 / M;                       // lanes per column in the second stage
  static constexpr int RS = 32 + (G < 16 ? G : 0);       // padded transpose row
  static constexpr int PEXT = prow<N>(N - 1) + 1;        // rows of a swizzled N-point buffer
  static constexpr int SW = (PEXT > M * RS ? PEXT : M * RS);  // per-warp scratch (float2)
  static constexpr int LANE_TAB = TW_FULL + N - 32;      // offset of the per-lane twiddle table
};

__host__ __device__ constexpr int bitrev_c(int i, int n) {
  int r = 0;
  for (int b = 1, rb = n >> 1; b < n; b <<= 1, rb >>= 1)
    if (i & b) r |= rb;
  return r;
}

// complex add / subtract as one packed f32x2 instruction on the (re, im) pair
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  return f2_unpack(f2_add(f2_pack(a.x, a.y), f2_pack(b.x, b.y)));
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return f2_unpack(f2_sub(f2_pack(a.x, a.y), f2_pack(b.x, b.y)));
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// table twiddle for direction D (+1 forward, -1 inverse)
template <int D>
__device__ __forceinline__ float2 twd(const float2 *__restrict__ tw, int j) {
  float2 w = __ldg(tw + j);
  if (D < 0) w.y = -w.y;
  return w;
}

// a * exp(-D 2 pi i j / 16) for j in [0, 8); j is a compile-time constant after unrolling
__device__ __forceinline__ float cos16(int j) {
  switch (j) {
    case 1: return 0.92387953251128676f;
    case 2: return 0.70710678118654752f;
    case 3: return 0.38268343236508977f;
    case 5: return -0.38268343236508977f;
    case 6: return -0.70710678118654752f;
    case 7: return -0.92387953251128676f;
    default: return 0.f;
  }
}
__device__ __forceinline__ float sin16(int j) {
  switch (j) {
    case 1: case 7: return 0.38268343236508977f;
    case 2: case 6: return 0.70710678118654752f;
    case 3: case 5: return 0.92387953251128676f;
    default: return 0.f;
  }
}
// exp(-2 pi i k / 32), k in [0, 16); k is a compile-time constant after unrolling
__device__ __forceinline__ float2 w32(int k) {
  switch (k) {
    case 1: return make_float2(0.98078528040323043f, -0.19509032201612826f);
    case 2: return make_float2(0.92387953251128674f, -0.38268343236508978f);
    case 3: return make_float2(0.83146961230254524f, -0.55557023301960218f);
    case 4: return make_float2(0.70710678118654752f, -0.70710678118654752f);
    case 5: return make_float2(0.55557023301960218f, -0.83146961230254524f);
    case 6: return make_float2(0.38268343236508978f, -0.92387953251128674f);
    case 7: return make_float2(0.19509032201612826f, -0.98078528040323043f);
    case 8: return make_float2(0.f, -1.f);
    case 9: return make_float2(-0.19509032201612826f, -0.98078528040323043f);
    case 10: return make_float2(-0.38268343236508978f, -0.92387953251128674f);
    case 11: return make_float2(-0.55557023301960218f, -0.83146961230254524f);
    case 12: return make_float2(-0.70710678118654752f, -0.70710678118654752f);
    case 13: return make_float2(-0.83146961230254524f, -0.55557023301960218f);
    case 14: return make_float2(-0.92387953251128674f, -0.38268343236508978f);
    case 15: return make_float2(-0.98078528040323043f, -0.19509032201612826f);
    default: return make_float2(1.f, 0.f);
  }
}

template <int D>
__device__ __forceinline__ float2 tw16(float2 a, int j) {
  if (j == 0) return a;
  if (j == 4) return D > 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
  const float c = cos16(j), s = D > 0 ? sin16(j) : -sin16(j);
  return make_float2(a.x * c + a.y * s, a.y * c - a.x * s);
}

// M-point decimation in frequency: natural input, bit-reversed output
template <int M, int D>
__device__ __forceinline__ void dif_reg(float2 (&v)[M]) {
#pragma unroll
  for (int span = M / 2; span >= 1; span >>= 1) {
#pragma unroll
    for (int i = 0; i < M; ++i) {
      if ((i & span) == 0) {
        const float2 a = v[i], b = v[i + span];
        v[i] = cadd(a, b);
        v[i + span] = tw16<D>(csub(a, b), (i & (span - 1)) * (8 / span));
      }
    }
  }
}
// M-point decimation in time: bit-reversed input, natural output (the inverse
// of dif_reg<M, -D> up to the factor M)
template <int M, int D>
__device__ __forceinline__ void dit_reg(float2 (&v)[M]) {
#pragma unroll
  for (int span = 1; span < M; span <<= 1) {
#pragma unroll
    for (int i = 0; i < M; ++i) {
      if ((i & span) == 0) {
        const float2 t = tw16<D>(v[i + span], (i & (span - 1)) * (8 / span));
        const float2 u = v[i];
        v[i] = cadd(u, t);
        v[i + span] = csub(u, t);
      }
    }
  }
}

// 8-byte asynchronous global->shared copies (no register staging), so a CTA has
// its whole tile of loads in flight at once
__device__ __forceinline__ void cp_async8(float2 *smem, const float2 *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ float2 shfl_xor2(float2 a, int m) {
  return make_float2(__shfl_xor_sync(FULL_MASK, a.x, m), __shfl_xor_sync(FULL_MASK, a.y, m));
}

template <int N>
__device__ __forceinline__ int lane_bitrev_g(int h) {
  constexpr int G = Fft<N>::G;
  constexpr int LG = G == 2 ? 1 : G == 4 ? 2 : G == 8 ? 3 : G == 16 ? 4 : 5;
  return (int)(__brev((unsigned)h) >> (32 - LG));
}
// second-stage twiddles exp(-D 2 pi i h k' / 32) of register i (k' = bitrev(i));
// with two lanes per column (N = 512) they are constants selected by h
template <int N, int D>
__device__ __forceinline__ void stage2_twiddle(float2 (&v)[Fft<N>::M], const float2 *__restrict__ tw, int h) {
  constexpr int M = Fft<N>::M, G = Fft<N>::G;
#pragma unroll
  for (int i = 1; i < M; ++i) {
    float2 w;
    if (G == 2) {
      w = w32(bitrev_c(i, M));
      if (D < 0) w.y = -w.y;
      if (h == 0) w = make_float2(1.f, 0.f);
    } else {
      w = twd<D>(tw, h * bitrev_c(i, M) * (TW_FULL / 32));
    }
    v[i] = cmul(v[i], w);
  }
}

__device__ __forceinline__ float2 add_signed(float2 o, float sgn, float2 v) {
  return f2_unpack(f2_fma(f2_pack(sgn, sgn), f2_pack(v.x, v.y), f2_pack(o.x, o.y)));
}

// index of register i of this lane after fft_n2p (and before fft_p2n)
template <int N>
__device__ __forceinline__ int out_index(int lane, int i) {
  constexpr int M = Fft<N>::M, G = Fft<N>::G;
  const int c = lane / G, h = lane & (G - 1);
  return c + M * (bitrev_c(i, M) + M * lane_bitrev_g<N>(h));
}

// N-point DFT of one line held by a warp. Input v[m] = x[lane + 32 m];
// output v[i] = X[out_index<N>(lane, i)]. D = +1: exp(-2 pi i jk/N); D = -1: the
// unnormalised inverse. S: this warp's scratch (Fft<N>::SW float2).
template <int N, int D>
__device__ __forceinline__ void fft_n2p(float2 (&v)[Fft<N>::M], float2 *S, const float2 *__restrict__ tw, int lane) {
  constexpr int M = Fft<N>::M, G = Fft<N>::G, RS = Fft<N>::RS;
  dif_reg<M, D>(v);
#pragma unroll
  for (int i = 1; i < M; ++i) v[i] = cmul(v[i], twd<D>(tw + Fft<N>::LANE_TAB, bitrev_c(i, M) * 32 + lane));
  const int c = lane / G, h = lane & (G - 1);
  if (M > 1) {
#pragma unroll
    for (int i = 0; i < M; ++i) S[bitrev_c(i, M) * RS + lane] = v[i];
    __syncwarp();
#pragma unroll
    for (int j = 0; j < M; ++j) v[j] = S[c * RS + h + G * j];
    __syncwarp();
  }
  dif_reg<M, D>(v);
  stage2_twiddle<N, D>(v, tw, h);
  // radix-2 stages across lanes: lower lane a + b, upper lane (a - b) w
#pragma unroll
  for (int span = G / 2; span >= 1; span >>= 1) {
    const bool upper = (h & span) != 0;
    const float sgn = upper ? -1.f : 1.f;
    float2 w = make_float2(1.f, 0.f);
    if (span > 1 && upper) w = twd<D>(tw, (h & (span - 1)) * (TW_FULL / (2 * span)));
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const float2 t = add_signed(shfl_xor2(v[i], span), sgn, v[i]);
      v[i] = span > 1 ? cmul(t, w) : t;
    }
  }
}

// The adjoint pipeline: input v[i] = X[out_index<N>(lane, i)], output
// v[m] = x[lane + 32 m]; fft_p2n<N, -1> inverts fft_n2p<N, +1> up to the factor N.
template <int N, int D>
__device__ __forceinline__ void fft_p2n(float2 (&v)[Fft<N>::M], float2 *S, const float2 *__restrict__ tw, int lane) {
  constexpr int M = Fft<N>::M, G = Fft<N>::G, RS = Fft<N>::RS;
  const int c = lane / G, h = lane & (G - 1);
  // radix-2 stages across lanes: the upper lane scales its value by w, then
  // lower lane a + w b, upper lane a - w b
#pragma unroll
  for (int span = 1; span < G; span <<= 1) {
    const bool upper = (h & span) != 0;
    const float sgn = upper ? -1.f : 1.f;
    float2 w = make_float2(1.f, 0.f);
    if (span > 1 && upper) w = twd<D>(tw, (h & (span - 1)) * (TW_FULL / (2 * span)));
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const float2 z = span > 1 ? cmul(v[i], w) : v[i];
      v[i] = add_signed(shfl_xor2(z, span), sgn, z);
    }
  }
  stage2_twiddle<N, D>(v, tw, h);
  dit_reg<M, D>(v);
  if (M > 1) {
#pragma unroll
    for (int j = 0; j < M; ++j) S[c * RS + h + G * j] = v[j];
    __syncwarp();
#pragma unroll
    for (int i = 0; i < M; ++i) v[i] = S[bitrev_c(i, M) * RS + lane];
    __syncwarp();
  }
#pragma unroll
  for (int i = 1; i < M; ++i) v[i] = cmul(v[i], twd<D>(tw + Fft<N>::LANE_TAB, bitrev_c(i, M) * 32 + lane));
  dit_reg<M, D>(v);
}

// ---- lines of any supported length --------------------------------------------
// N = 2^p (32..512) runs the pipelines above. N = 3P, P = 2^p (96, 192, 384) adds a
// radix-3 step: a lane's registers m, m + P/32, m + 2P/32 hold the points n, n + P,
// n + 2P (n = lane + 32 m); one 3-point DFT across them, the twiddles
// exp(-D 2 pi i n k3 / N) (k3 = 1, 2), then the three P-point warp transforms, so
// that register k3 P/32 + i holds X[3 index_P(i) + k3] (decimation in frequency;
// the adjoint runs the steps backwards). The twiddles come from a per-N table of
// exp(-2 pi i j / N), j < 2P, after the power-of-two tables.
constexpr int TW3_BASE = TW_FULL + 512 - 32 + 512;
constexpr int TW3_LEN = 64 + 128 + 256;  // 2P for N = 96, 192, 384
template <int N>
__host__ __device__ constexpr int tw3_off() {
  return TW3_BASE + (N == 96 ? 0 : N == 192 ? 64 : 192);
}
// Row of spectrum index k in a natural-order buffer. For N = 3P a warp writes
// register i to X = 3 index_P(lane, i) + k3, i.e. 3c + 48h + K (P = 128 and 32:
// c < 4 or c = 0, h the lane's bit-reversed column, K < 48 the same for all lanes)
// or 3c + 12h + K (P = 64, c < 2, K < 12); k + 4 floor(k / 48), resp. k + floor(k / 12),
// puts the 32 lanes on 16 distinct 8-byte bank pairs, two each (the minimum), and
// keeps consecutive k on consecutive rows apart from one skip per block.
template <int N>
__host__ __device__ constexpr int xf_row(int k) {
  if constexpr (N == 192) return k + k / 12;
  else if constexpr (N % 3 == 0) return k + 4 * (k / 48);
  else return prow<N>(k);
}
template <int N>
__host__ __device__ constexpr int xf_rows() {
  if constexpr (N % 3 == 0) return xf_row<N>(N - 1) + 1;
  else return Fft<N>::PEXT;
}
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }
template <int N>
__host__ __device__ constexpr int xf_sw() {  // per-warp scratch (float2): sub-transforms, natural-order rows, N values
  if constexpr (N % 3 == 0) return cmax(cmax(Fft<N / 3>::SW, xf_rows<N>()), N);
  else return Fft<N>::SW;
}

// spectrum index held in register i after xf_fwd
template <int N>
__device__ __forceinline__ int xf_index(int lane, int i) {
  if constexpr (N % 3 == 0) {
    constexpr int MP = N / 96;
    return 3 * out_index<N / 3>(lane, i % MP) + i / MP;
  } else {
    return out_index<N>(lane, i);
  }
}

// 3-point DFT of (a, b, c) with kernel exp(-D 2 pi i jk / 3)
template <int D>
__device__ __forceinline__ void radix3(float2 &a, float2 &b, float2 &c) {
  constexpr float S3 = 0.86602540378443865f;  // sin(2 pi / 3)
  const float2 t1 = cadd(b, c), t2 = csub(b, c);
  const float2 mm = make_float2(a.x - 0.5f * t1.x, a.y - 0.5f * t1.y);
  const float2 r = D > 0 ? make_float2(S3 * t2.y, -S3 * t2.x) : make_float2(-S3 * t2.y, S3 * t2.x);  // -i D s t2
  a = cadd(a, t1);
  b = cadd(mm, r);
  c = csub(mm, r);
}

template <int N, int D>
__device__ __forceinline__ void xf_fwd(float2 (&v)[N / 32], float2 *S, const float2 *__restrict__ tw, int lane) {
  if constexpr (N % 3 == 0) {
    constexpr int P = N / 3, MP = P / 32;
    const float2 *t3 = tw + tw3_off<N>();
#pragma unroll
    for (int m = 0; m < MP; ++m) {
      radix3<D>(v[m], v[m + MP], v[m + 2 * MP]);
      const int n = lane + 32 * m;
      v[m + MP] = cmul(v[m + MP], twd<D>(t3, n));
      v[m + 2 * MP] = cmul(v[m + 2 * MP], twd<D>(t3, 2 * n));
    }
#pragma unroll
    for (int k3 = 0; k3 < 3; ++k3) {
      float2 u[MP];
#pragma unroll
      for (int i = 0; i < MP; ++i) u[i] = v[k3 * MP + i];
      fft_n2p<P, D>(u, S, tw, lane);
#pragma unroll
      for (int i = 0; i < MP; ++i) v[k3 * MP + i] = u[i];
    }
  } else {
    fft_n2p<N, D>(v, S, tw, lane);
  }
}

// the adjoint of xf_fwd: register-order input, natural output; xf_inv<N, -1>
// inverts xf_fwd<N, +1> up to the factor N
template <int N, int D>
__device__ __forceinline__ void xf_inv(float2 (&v)[N / 32], float2 *S, const float2 *__restrict__ tw, int lane) {
  if constexpr (N % 3 == 0) {
    constexpr int P = N / 3, MP = P / 32;
    const float2 *t3 = tw + tw3_off<N>();
#pragma unroll
    for (int k3 = 0; k3 < 3; ++k3) {
      float2 u[MP];
#pragma unroll
      for (int i = 0; i < MP; ++i) u[i] = v[k3 * MP + i];
      fft_p2n<P, D>(u, S, tw, lane);
#pragma unroll
      for (int i = 0; i < MP; ++i) v[k3 * MP + i] = u[i];
    }
#pragma unroll
    for (int m = 0; m < MP; ++m) {
      const int n = lane + 32 * m;
      v[m + MP] = cmul(v[m + MP], twd<D>(t3, n));
      v[m + 2 * MP] = cmul(v[m + 2 * MP], twd<D>(t3, 2 * n));
      radix3<D>(v[m], v[m + MP], v[m + 2 * MP]);
    }
  } else {
    fft_p2n<N, D>(v, S, tw, lane);
  }
}

// ---- pass 2: forward y, written transposed -----------------------------------
// CTA: (c, kz) plane, 16 consecutive x lines; output rows of 16 x values per ky.
template <int NY>
__global__ void __launch_bounds__(FFT_THREADS) k_fft_y_fwd(const float2 *__restrict__ A, float2 *__restrict__ B,
                                                           int nx, const float2 *__restrict__ tw) {
  constexpr int M = (NY / 32), SW = xf_sw<NY>();
  extern __shared__ float2 fft_smem[];
  float2 *T = fft_smem;  // xf_rows<NY>() swizzled rows x FFT_TS
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2 *S = fft_smem + xf_rows<NY>() * FFT_TS + warp * SW;
  const int nxt = nx / FFT_TILE;
  const int xt = blockIdx.x % nxt;
  const size_t ckz = blockIdx.x / nxt;
#pragma unroll 1
  for (int r = 0; r < FFT_TILE / FFT_WARPS; ++r) {
    const int wx = warp + FFT_WARPS * r;
    const float2 *line = A + (ckz * nx + (size_t)xt * FFT_TILE + wx) * NY;
    float2 v[M];
#pragma unroll
    for (int m = 0; m < M; ++m) v[m] = __ldg(line + lane + 32 * m);
    xf_fwd<NY, 1>(v, S, tw, lane);
#pragma unroll
    for (int i = 0; i < M; ++i) T[xf_row<NY>(xf_index<NY>(lane, i)) * FFT_TS + wx] = v[i];
  }
  __syncthreads();
  float2 *out = B + ckz * NY * nx + (size_t)xt * FFT_TILE;
  for (int idx = threadIdx.x; idx < NY * FFT_TILE; idx += FFT_THREADS) {
    const int ky = idx / FFT_TILE, j = idx % FFT_TILE;
    out[(size_t)ky * nx + j] = T[xf_row<NY>(ky) * FFT_TS + j];
  }
}

__device__ __forceinline__ float wavenumber_f(int i, int n, float ff) { return (float)((i <= n / 2) ? i : i - n) * ff; }

// ---- pass 3: x lines: forward, projection, inverse ---------------------------------
// Three warps per (kz, ky), one per component. After the forward transforms each
// warp leaves its spectrum in its scratch in register order (the same
// lane/register -> kx map for all three), every warp reads the three values of
// its modes and keeps its own projected component. Arithmetic of the projection
// as in flow_solve (FCMfunctions.cpp:668-722): norm = 1/(|q|^2 + 1e-18),
// u = norm (f - q (q.f) norm) / (Nx Ny Nz); the k = 0 mode is zeroed. The
// reciprocal is the fast one (2 ulp), well inside the FP32 chain's error.
constexpr int XP_PAIRS = 1;                    // (kz, ky) lines per CTA (1: 5% faster than 2 at 512^3)
constexpr int XP_THREADS = 3 * 32 * XP_PAIRS;  // one warp per component and line
template <int NX>
__global__ void __launch_bounds__(XP_THREADS) k_fft_x_project(float2 *__restrict__ B, int ny, int nzh,
                                                              size_t cstride, float ffx, float ffy, float ffz,
                                                              float inv_total, const float2 *__restrict__ tw) {
  constexpr int M = (NX / 32), SW = xf_sw<NX>();
  __shared__ float2 Sall[3 * XP_PAIRS * SW];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int comp = warp % 3, pl = warp / 3;
  float2 *S = Sall + warp * SW;
  const int pair = blockIdx.x * XP_PAIRS + pl;
  const bool active = pair < nzh * ny;  // warp-uniform; inactive warps still reach the barriers
  const int kz = pair / ny, ky = pair % ny;
  float2 *line = B + comp * cstride + (size_t)pair * NX;
  float2 v[M];
  if (active) {
#pragma unroll
    for (int m = 0; m < M; ++m) v[m] = line[lane + 32 * m];
    xf_fwd<NX, 1>(v, S, tw, lane);
#pragma unroll
    for (int i = 0; i < M; ++i) S[lane + 32 * i] = v[i];
  }
  __syncthreads();
  if (active) {
    const float2 *S0 = Sall + (3 * pl) * SW, *S1 = S0 + SW, *S2 = S1 + SW;
    const float q2 = wavenumber_f(ky, ny, ffy), q3 = (float)kz * ffz;
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int kx = xf_index<NX>(lane, i);
      const float q1 = wavenumber_f(kx, NX, ffx);
      const float qq = q2 * q2 + q1 * q1 + 1e-18f;
      const float norm = __fdividef(1.0f, qq + q3 * q3);
      const float2 a = S0[lane + 32 * i], b = S1[lane + 32 * i], d = S2[lane + 32 * i];
      const float kfr = (q1 * a.x + q2 * b.x + q3 * d.x) * norm;
      const float kfi = (q1 * a.y + q2 * b.y + q3 * d.y) * norm;
      const float qc = comp == 0 ? q1 : comp == 1 ? q2 : q3;
      const float sc = (kx | ky | kz) == 0 ? 0.f : norm * inv_total;
      v[i] = make_float2(sc * (v[i].x - qc * kfr), sc * (v[i].y - qc * kfi));
    }
  }
  __syncthreads();
  if (active) {
    xf_inv<NX, -1>(v, S, tw, lane);
#pragma unroll
    for (int m = 0; m < M; ++m) line[lane + 32 * m] = v[m];
  }
}

// ---- pass 4: inverse y, read transposed ---------------------------------------
template <int NY>
__global__ void __launch_bounds__(FFT_THREADS) k_fft_y_inv(const float2 *__restrict__ B, float2 *__restrict__ A,
                                                           int nx, const float2 *__restrict__ tw) {
  constexpr int M = (NY / 32), SW = xf_sw<NY>();
  extern __shared__ float2 fft_smem[];
  float2 *T = fft_smem;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2 *S = fft_smem + NY * FFT_TS + warp * SW;
  const int nxt = nx / FFT_TILE;
  const int xt = blockIdx.x % nxt;
  const size_t ckz = blockIdx.x / nxt;
  const float2 *in = B + ckz * NY * nx + (size_t)xt * FFT_TILE;
  for (int idx = threadIdx.x; idx < NY * FFT_TILE; idx += FFT_THREADS) {
    const int ky = idx / FFT_TILE, j = idx % FFT_TILE;
    cp_async8(T + ky * FFT_TS + j, in + (size_t)ky * nx + j);
  }
  cp_async_wait_all();
  __syncthreads();
#pragma unroll 1
  for (int r = 0; r < FFT_TILE / FFT_WARPS; ++r) {
    const int wx = warp + FFT_WARPS * r;
    float2 v[M];
#pragma unroll
    for (int m = 0; m < M; ++m) v[m] = T[(lane + 32 * m) * FFT_TS + wx];
    xf_fwd<NY, -1>(v, S, tw, lane);
    float2 *line = A + (ckz * nx + (size_t)xt * FFT_TILE + wx) * NY;
    if constexpr (NY % 3 == 0) {  // register order scatters at stride 3: store in natural order
#pragma unroll
      for (int i = 0; i < M; ++i) S[xf_row<NY>(xf_index<NY>(lane, i))] = v[i];
      __syncwarp();
#pragma unroll
      for (int m = 0; m < M; ++m) line[lane + 32 * m] = S[xf_row<NY>(lane + 32 * m)];
      __syncwarp();
    } else {
#pragma unroll
      for (int i = 0; i < M; ++i) line[xf_index<NY>(lane, i)] = v[i];
    }
  }
}

// ---- passes 1 and 5: z lines in pairs -------------------------------------------
// Warp w transforms its two real z lines a = y-line w and b = y-line w + 8 as one
// NZ-point complex line z = a + i b: forward, A_k = (Z_k + conj Z_{NZ-k}) / 2 and
// B_k = (Z_k - conj Z_{NZ-k}) / (2i) for k <= NZ/2; inverse, Z_k = A_k + i B_k
// (k <= NZ/2, the imaginary parts of A_0, A_{NZ/2}, B_0, B_{NZ/2} dropped) and
// Z_{NZ-k} = conj A_k + i conj B_k, then a = Re z, b = Im z. One full-length
// transform per line pair instead of two half-length ones.
// ZT y tiles per CTA, consecutive in y: a warp issues the loads of its next line
// pair before the CTA writes the current tile out, so each warp keeps one pair
// of lines in flight through the store phase.
template <int NZ, int ZT>
__global__ void __launch_bounds__(FFT_THREADS) k_fft_z_r2c(const float *__restrict__ f, float2 *__restrict__ A,
                                                            int nx, int ny, const float2 *__restrict__ tw) {
  static_assert(FFT_TILE == 2 * FFT_WARPS, "two lines per warp");
  constexpr int H = NZ / 2, M = (NZ / 32), SW = xf_sw<NZ>();
  extern __shared__ float2 fft_smem[];
  float2 *T = fft_smem;  // (H + 1) x FFT_TS
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2 *S = fft_smem + (H + 1) * FFT_TS + warp * SW;
  const int nyg = ny / (FFT_TILE * ZT);  // groups of ZT tiles along y
  const int yg = blockIdx.x % nyg;
  const int x = (blockIdx.x / nyg) % nx;
  const int c = blockIdx.x / (nyg * nx);
  const int wa = warp, wb = warp + FFT_WARPS;
  const size_t plane = (size_t)nx * ny;
  float2 v[M];
  auto load = [&](int yt) {
    const float *la = f + (((size_t)c * nx + x) * ny + (size_t)yt * FFT_TILE + wa) * NZ;
    const float *lb = la + (size_t)FFT_WARPS * NZ;
#pragma unroll
    for (int m = 0; m < M; ++m) v[m] = make_float2(__ldg(la + lane + 32 * m), __ldg(lb + lane + 32 * m));
  };
  load(yg * ZT);
#pragma unroll 1
  for (int t = 0; t < ZT; ++t) {
    const int yt = yg * ZT + t;
    xf_fwd<NZ, 1>(v, S, tw, lane);
#pragma unroll
    for (int i = 0; i < M; ++i) S[xf_row<NZ>(xf_index<NZ>(lane, i))] = v[i];
    if (t + 1 < ZT) load(yt + 1);
    __syncwarp();
#pragma unroll
    for (int m = 0; m < (H + 32) / 32; ++m) {
      const int k = lane + 32 * m;
      if (k <= H) {
        const float2 zk = S[xf_row<NZ>(k)], zr = S[xf_row<NZ>(k == 0 ? 0 : NZ - k)];
        T[k * FFT_TS + wa] = make_float2(0.5f * (zk.x + zr.x), 0.5f * (zk.y - zr.y));
        T[k * FFT_TS + wb] = make_float2(0.5f * (zk.y + zr.y), -0.5f * (zk.x - zr.x));
      }
    }
    __syncthreads();
    float2 *out = A + ((size_t)c * (H + 1) * nx + x) * ny + (size_t)yt * FFT_TILE;
    for (int idx = threadIdx.x; idx < (H + 1) * FFT_TILE; idx += FFT_THREADS) {
      const int k = idx / FFT_TILE, j = idx % FFT_TILE;
      out[(size_t)k * plane + j] = T[k * FFT_TS + j];
    }
    if (t + 1 < ZT) __syncthreads();  // T and S are rewritten by the next tile
  }
}

template <int NZ>
__global__ void __launch_bounds__(FFT_THREADS) k_fft_z_c2r(const float2 *__restrict__ A, float *__restrict__ u,
                                                            int nx, int ny, const float2 *__restrict__ tw) {
  static_assert(FFT_TILE == 2 * FFT_WARPS, "two lines per warp");
  constexpr int H = NZ / 2, M = (NZ / 32), SW = xf_sw<NZ>();
  extern __shared__ float2 fft_smem[];
  float2 *T = fft_smem;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2 *S = fft_smem + (H + 1) * FFT_TS + warp * SW;
  const int nyt = ny / FFT_TILE;
  const int yt = blockIdx.x % nyt;
  const int x = (blockIdx.x / nyt) % nx;
  const int c = blockIdx.x / (nyt * nx);
  const float2 *in = A + ((size_t)c * (H + 1) * nx + x) * ny + (size_t)yt * FFT_TILE;
  const size_t plane = (size_t)nx * ny;
  for (int idx = threadIdx.x; idx < (H + 1) * FFT_TILE; idx += FFT_THREADS) {
    const int k = idx / FFT_TILE, j = idx % FFT_TILE;
    cp_async8(T + k * FFT_TS + j, in + (size_t)k * plane + j);
  }
  cp_async_wait_all();
  __syncthreads();
  const int wa = warp, wb = warp + FFT_WARPS;
  float2 v[M];
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int k = lane + 32 * m;
    if (k <= H) {
      float2 a = T[k * FFT_TS + wa], b = T[k * FFT_TS + wb];
      if (k == 0 || k == H) a.y = b.y = 0.f;
      v[m] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      const int kk = NZ - k;
      const float2 a = T[kk * FFT_TS + wa], b = T[kk * FFT_TS + wb];
      v[m] = make_float2(a.x + b.y, b.x - a.y);
    }
  }
  xf_fwd<NZ, -1>(v, S, tw, lane);
  float *oa = u + (((size_t)c * nx + x) * ny + (size_t)yt * FFT_TILE + wa) * NZ;
  float *ob = oa + (size_t)FFT_WARPS * NZ;
  if constexpr (NZ % 3 == 0) {  // register order scatters at stride 3: store in natural order
#pragma unroll
    for (int i = 0; i < M; ++i) S[xf_row<NZ>(xf_index<NZ>(lane, i))] = v[i];
    __syncwarp();
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const float2 z = S[xf_row<NZ>(lane + 32 * m)];
      oa[lane + 32 * m] = z.x;
      ob[lane + 32 * m] = z.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int o = xf_index<NZ>(lane, i);
      oa[o] = v[i].x;
      ob[o] = v[i].y;
    }
  }
}

template <int NZ>
constexpr size_t smem_z() { return sizeof(float2) * ((NZ / 2 + 1) * FFT_TS + FFT_WARPS * xf_sw<NZ>()); }

template <int NY>
constexpr size_t smem_y() { return sizeof(float2) * (xf_rows<NY>() * FFT_TS + FFT_WARPS * xf_sw<NY>()); }

bool pow2_in(int n, int lo, int hi) { return n >= lo && n <= hi && (n & (n - 1)) == 0; }

// y tiles per z_r2c CTA where the grid has an even number of y tiles (the same
// overlap in z_c2r and y_inv, with the next tile's asynchronous copy under the
// current tile's transforms, was slower at 512^3: 0.732 vs 0.724 ms and 0.689 vs
// 0.667 ms)
constexpr int Z_TILES = 2;

template <int NZ>
fs_status z_attr() {
  FS_CUDA(cudaFuncSetAttribute(k_fft_z_r2c<NZ, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_z<NZ>()));
  FS_CUDA(cudaFuncSetAttribute(k_fft_z_r2c<NZ, Z_TILES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem_z<NZ>()));
  FS_CUDA(cudaFuncSetAttribute(k_fft_z_c2r<NZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_z<NZ>()));
  return FS_OK;
}
template <int NY>
fs_status y_attr() {
  FS_CUDA(cudaFuncSetAttribute(k_fft_y_fwd<NY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_y<NY>()));
  FS_CUDA(cudaFuncSetAttribute(k_fft_y_inv<NY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_y<NY>()));
  return FS_OK;
}

template <int NZ>
fs_status z_fwd(fs_ctx *c, const float *f, float2 *A, const float2 *tw) {
  const int nyt = c->ny / FFT_TILE;
  if (nyt % Z_TILES == 0)
    k_fft_z_r2c<NZ, Z_TILES><<<3 * c->nx * (nyt / Z_TILES), FFT_THREADS, smem_z<NZ>(), c->stream>>>(f, A, c->nx,
                                                                                                    c->ny, tw);
  else
    k_fft_z_r2c<NZ, 1><<<3 * c->nx * nyt, FFT_THREADS, smem_z<NZ>(), c->stream>>>(f, A, c->nx, c->ny, tw);
  FS_LAUNCH_CHECK();
  return FS_OK;
}
template <int NZ>
fs_status z_inv(fs_ctx *c, const float2 *A, float *u, const float2 *tw) {
  k_fft_z_c2r<NZ><<<3 * c->nx * (c->ny / FFT_TILE), FFT_THREADS, smem_z<NZ>(), c->stream>>>(A, u, c->nx, c->ny, tw);
  FS_LAUNCH_CHECK();
  return FS_OK;
}
template <int NY>
fs_status y_fwd(fs_ctx *c, const float2 *A, float2 *B, const float2 *tw) {
  k_fft_y_fwd<NY><<<3 * c->nzh * (c->nx / FFT_TILE), FFT_THREADS, smem_y<NY>(), c->stream>>>(A, B, c->nx, tw);
  FS_LAUNCH_CHECK();
  return FS_OK;
}
template <int NY>
fs_status y_inv(fs_ctx *c, const float2 *B, float2 *A, const float2 *tw) {
  k_fft_y_inv<NY><<<3 * c->nzh * (c->nx / FFT_TILE), FFT_THREADS, smem_y<NY>(), c->stream>>>(B, A, c->nx, tw);
  FS_LAUNCH_CHECK();
  return FS_OK;
}
template <int NX>
fs_status x_project(fs_ctx *c, float2 *B, const float2 *tw) {
  const double TwoPI = 2. * FS_PI;
  const float ffx = (float)(TwoPI / (c->nx * c->p.dx)), ffy = (float)(TwoPI / (c->ny * c->p.dx)),
              ffz = (float)(TwoPI / (c->nz * c->p.dx));
  // 1 / (Nx Ny Nz) is a power of two here, so the product equals the reference's quotient
  const float inv_total = (float)(1.0 / ((double)c->nx * (double)c->ny * (double)c->nz));
  const int pairs = c->nzh * c->ny;
  const size_t cstride = (size_t)c->nzh * c->ny * c->nx;
  k_fft_x_project<NX><<<fs_blocks(pairs, XP_PAIRS), XP_THREADS, 0, c->stream>>>(B, c->ny, c->nzh, cstride, ffx, ffy,
                                                                                ffz, inv_total, tw);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

#define FS_FFT_SWITCH_Z(n, fn, ...)                  \
  switch (n) {                                       \
    case 64: FS_TRY(fn<64>(__VA_ARGS__)); break;     \
    case 96: FS_TRY(fn<96>(__VA_ARGS__)); break;     \
    case 128: FS_TRY(fn<128>(__VA_ARGS__)); break;   \
    case 192: FS_TRY(fn<192>(__VA_ARGS__)); break;   \
    case 256: FS_TRY(fn<256>(__VA_ARGS__)); break;   \
    case 384: FS_TRY(fn<384>(__VA_ARGS__)); break;   \
    case 512: FS_TRY(fn<512>(__VA_ARGS__)); break;   \
    default: return FS_ERR_INVALID_ARG;              \
  }
#define FS_FFT_SWITCH(n, fn, ...)                    \
  if (n == 32) {                                     \
    FS_TRY(fn<32>(__VA_ARGS__));                     \
  } else {                                           \
    FS_FFT_SWITCH_Z(n, fn, __VA_ARGS__)              \
  }

}  // namespace

// line lengths of the warp transforms: 2^p in [lo, 512], or 96, 192, 384
static bool fft_len(int n, int lo) { return n >= lo && (pow2_in(n, lo, 512) || n == 96 || n == 192 || n == 384); }

bool fft32_supported(const fs_ctx *c) { return fft_len(c->nx, 32) && fft_len(c->ny, 32) && fft_len(c->nz, 64); }

fs_status fft32_init(fs_ctx *c) {
  c->fft_tw = nullptr;
  if (!fft32_supported(c)) return FS_OK;
  // [0, 1024): exp(-2 pi i j / 1024); then per N in {32, ..., 512}, at 1024 + N - 32,
  // the lane table [k2 * 32 + lane] = exp(-2 pi i lane k2 / N), k2 < N / 32; then per
  // N in {96, 192, 384}, at tw3_off<N>, exp(-2 pi i j / N), j < 2N/3.
  const int ntw = TW3_BASE + TW3_LEN;
  float2 *h = (float2 *)malloc(sizeof(float2) * ntw);
  if (!h) return FS_ERR_OOM;
  const double TwoPI = 2. * FS_PI;
  for (int j = 0; j < TW_FULL; ++j) h[j] = make_float2((float)cos(TwoPI * j / TW_FULL), (float)-sin(TwoPI * j / TW_FULL));
  for (int n = 32; n <= 512; n <<= 1)
    for (int k2 = 0; k2 < n / 32; ++k2)
      for (int l = 0; l < 32; ++l) {
        const long long j = (long long)l * k2;
        h[TW_FULL + n - 32 + k2 * 32 + l] = make_float2((float)cos(TwoPI * j / n), (float)-sin(TwoPI * j / n));
      }
  const int n3[3] = {96, 192, 384}, off3[3] = {tw3_off<96>(), tw3_off<192>(), tw3_off<384>()};
  for (int q = 0; q < 3; ++q)
    for (int j = 0; j < 2 * n3[q] / 3; ++j)
      h[off3[q] + j] = make_float2((float)cos(TwoPI * j / n3[q]), (float)-sin(TwoPI * j / n3[q]));
  cudaError_t e = cudaMalloc(&c->fft_tw, sizeof(float2) * ntw);
  if (e == cudaSuccess) e = cudaMemcpy(c->fft_tw, h, sizeof(float2) * ntw, cudaMemcpyHostToDevice);
  free(h);
  if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? FS_ERR_OOM : FS_ERR_CUDA;
  c->bytes += sizeof(float2) * ntw;
  FS_FFT_SWITCH_Z(c->nz, z_attr);
  FS_FFT_SWITCH(c->ny, y_attr);
  return FS_OK;
}

void fft32_free(fs_ctx *c) {
  cudaFree(c->fft_tw);
  c->fft_tw = nullptr;
}

// u = Stokes solve of f, both FP32 [3][nx][ny][nz] in c->grid_real (in place);
// c->grid_cplx holds the two half spectra A and B.
fs_status fft32_flow_solve(fs_ctx *c) {
  const float2 *tw = (const float2 *)c->fft_tw;
  float *g = (float *)c->grid_real;
  float2 *A = (float2 *)c->grid_cplx;
  float2 *B = A + (size_t)3 * c->nzh * c->nx * c->ny;
  {
    ProfScope ps(c, FS_STAGE_FFT_FWD);
    {
      ProfScope pk(c, FS_STAGE_K_FFT_Z_FWD);
      FS_FFT_SWITCH_Z(c->nz, z_fwd, c, g, A, tw);
    }
    ProfScope pk(c, FS_STAGE_K_FFT_Y_FWD);
    FS_FFT_SWITCH(c->ny, y_fwd, c, A, B, tw);
  }
  {
    ProfScope ps(c, FS_STAGE_PROJECT);
    FS_FFT_SWITCH(c->nx, x_project, c, B, tw);
  }
  {
    ProfScope ps(c, FS_STAGE_FFT_INV);
    {
      ProfScope pk(c, FS_STAGE_K_FFT_Y_INV);
      FS_FFT_SWITCH(c->ny, y_inv, c, B, A, tw);
    }
    ProfScope pk(c, FS_STAGE_K_FFT_Z_INV);
    FS_FFT_SWITCH_Z(c->nz, z_inv, c, A, g, tw);
  }
  return FS_OK;
}
