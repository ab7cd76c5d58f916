// fs_fcm.cu -- Force Coupling Method mobility solve on sm_100a.
//
// Replaces Fcm::mobility_solve (FCMfunctions.cpp:175-464):
//   1. k_fcm_bin_keys + counting sort: beads binned by the 16-point tile that
//      holds the start of their Gaussian stencil (gaussian_setup's index rule,
//      FCMfunctions.cpp:565-589).
//   2. k_spread (FP64) / k_spread_records32 + k_spread32 (FP32 chain): CTAs over
//      16^3 grid tiles gather the monopole + rotlet Gaussians of every bead whose
//      stencil reaches the tile (mono_and_dipole_force_distribution, :596-646);
//      each lane owns grid points and sums in registers (FP32: Kahan-compensated,
//      on packed f32x2 pairs): no atomics, bit-reproducible.
//   3. cuFFT R2C (batched x3), 4. k_project / k_project_planes: the Stokes
//      projection of flow_solve (:648-736), 5. cuFFT C2R (batched x3).
//   6. k_interp: one warp per bead (in spread-bin order for L2 locality)
//      reduces U and Omega over the stencil (particle_velocities :740-770,
//      particle_rotations :774-808) with warp shuffles.
// FP64 mode follows the reference arithmetic; FP32 mode keeps grids, FFTs and
// weights in float, with Kahan-compensated spread sums and FP64 accumulation of
// the interpolation products.
#include "fs_internal.cuh"
#include "fs_f32x2.cuh"

namespace {

struct FcmConsts {
  int N[3];
  int gnx, x0;  // x extent of the whole box and the grid's first plane in it (a slab window; else N[0], 0)
  int ngd, ngdh;
  int nbin[3];
  double dx;
  double anorm, anorm2, anormdip, anormdip2, sigmadipsq;
};

__host__ __device__ inline int wrap_int(int x, int n) {
  int r = x % n;
  return r < 0 ? r + n : r;
}
// x in (-n, 2n): one conditional add or subtract
__device__ __forceinline__ int wrap_near(int x, int n) {
  x += (x < 0) ? n : 0;
  return x >= n ? x - n : x;
}

// ---- 1. binning -------------------------------------------------------------
// key: the tile bin of the wrapped stencil start; sw: the wrapped stencil
// start per axis (gaussian_setup's index rule, FCMfunctions.cpp:565-585), kept
// for the spread and interpolation kernels so they need no integer division.
__global__ void k_fcm_bin_keys(const double *__restrict__ Y, int np, FcmConsts c, int *__restrict__ key,
                               int *__restrict__ sw_out) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= np) return;
  int bi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int xc = (int)(Y[3 * b + d] / c.dx);
    // the stencil start in the whole box, then in this grid (a slab window holds the
    // beads whose x start lies in its own planes; others are clamped, never out of range)
    int sw = wrap_int(xc - c.ngdh + 1, d == 0 ? c.gnx : c.N[d]) - (d == 0 ? c.x0 : 0);
    sw = sw < 0 ? 0 : (sw >= c.N[d] ? c.N[d] - 1 : sw);
    sw_out[3 * b + d] = sw;
    bi[d] = sw / FS_TILE;
  }
  key[b] = (bi[0] * c.nbin[1] + bi[1]) * c.nbin[2] + bi[2];
}

// ---- 2. spread ----------------------------------------------------------------
// One CTA (16 warps) per 16^3 grid tile; the tile is cut into 2x2x8 blocks and
// warp w owns the 8 blocks of column (bx, bz) = (w/2, w%2), one grid point per
// lane. Candidate beads (stencil start in the tile's bin or the one before it,
// per axis) are staged as per-axis weight tables indexed by tile coordinate
// (zero outside the bead's stencil). Each warp builds, by ballots, the set of
// staged beads that reach its column and, per block, those that reach the
// block; every lane then sums those beads' contributions to its point in
// registers, in sorted bead order, and writes the point once. No atomics and no
// shared-memory read-modify-write; bit-reproducible. FP32 mode keeps Kahan
// compensated register sums.
#define FS_SPREAD_THREADS 512

template <typename R>
struct W4 {
  R g, d, r, pad;
};

// CH beads are staged per pass (32 or 64, chosen per grid by fs_autotune)
template <typename R, int CH>
struct SpreadStage {
  W4<R> w[CH][3][FS_TILE];  // weights by tile-local coordinate
  R f[CH][4];                // force
  R th[CH][4];               // half torque (GA_setup, :536-547)
  unsigned mask[CH][3];      // per axis: tile-local coordinates covered
};

template <typename R>
struct KAcc;
template <>
struct KAcc<double> {
  double s;
  __device__ void init() { s = 0.0; }
  __device__ void add(double v) { s += v; }
  __device__ double value() const { return s; }
};
template <>
struct KAcc<float> {
  float s, c;
  __device__ void init() { s = 0.f; c = 0.f; }
  __device__ void add(float v) {
    float y = v - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ float value() const { return s - c; }
};

template <typename R>
__device__ inline R fs_exp(R x);
template <>
__device__ inline double fs_exp<double>(double x) { return exp(x); }
template <>
__device__ inline float fs_exp<float>(float x) { return expf(x); }

template <typename R, int CH>
__global__ void __launch_bounds__(FS_SPREAD_THREADS)
    k_spread(const double *__restrict__ Y, const double *__restrict__ F, const double *__restrict__ T,
             const int *__restrict__ bin_start, const int *__restrict__ sorted, const int *__restrict__ bead_sw,
             FcmConsts c, R *__restrict__ fgrid) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SpreadStage<R, CH> &st = *reinterpret_cast<SpreadStage<R, CH> *>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tile = blockIdx.x;
  const int tz = tile % c.nbin[2], ty = (tile / c.nbin[2]) % c.nbin[1], tx = tile / (c.nbin[2] * c.nbin[1]);
  const int X0[3] = {tx * FS_TILE, ty * FS_TILE, tz * FS_TILE};
  // candidate bins per axis: the tile's own bin and the ones before it that a
  // stencil reaches (fs_cand_bins), each bin once on an axis with fewer bins
  int cb[3][3], ncb[3];
  const int tb[3] = {tx, ty, tz};
  const int K = fs_cand_bins(c.ngd);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    ncb[d] = min(K, c.nbin[d]);
    for (int j = 0; j < ncb[d]; ++j) cb[d][j] = wrap_int(tb[d] - (ncb[d] - 1 - j), c.nbin[d]);
  }
  int rs[27], re[27], nr = 0, total = 0;
  for (int a = 0; a < ncb[0]; ++a)
    for (int b2 = 0; b2 < ncb[1]; ++b2)
      for (int e = 0; e < ncb[2]; ++e) {
        int bin = (cb[0][a] * c.nbin[1] + cb[1][b2]) * c.nbin[2] + cb[2][e];
        rs[nr] = bin_start[bin];
        re[nr] = bin_start[bin + 1];
        total += re[nr] - rs[nr];
        nr++;
      }
  // this lane's point in block (bx, by, bz): x = 2bx + (lane&1), y = 2by + ((lane>>1)&1), z = 8bz + (lane>>2)
  const int bx = warp >> 1, bz = warp & 1;
  const int px = 2 * bx + (lane & 1), pyo = (lane >> 1) & 1, pz = 8 * bz + (lane >> 2);
  const size_t N = (size_t)c.N[0] * c.N[1] * c.N[2];
  const int ngd = c.ngd;
  for (int base = 0; base < total; base += CH) {
    const int nb = min(CH, total - base);
    __syncthreads();  // the previous chunk's tables are no longer read
    // stage: one half-warp per (bead slot, axis), lane l -> tile-local coordinate l
    const int nitems = nb * 3 * FS_TILE;
    for (int it0 = warp * 32; it0 < nitems; it0 += FS_SPREAD_THREADS) {
      const int it = it0 + lane;
      const bool act = it < nitems;
      const int s = act ? it / (3 * FS_TILE) : 0;
      const int a = act ? (it / FS_TILE) % 3 : 0;
      const int l = it % FS_TILE;
      bool valid = false;
      W4<R> wv = {(R)0, (R)0, (R)0, (R)0};
      int bead = 0;
      if (act) {
        int rank = base + s, r = 0;
        while (rank >= re[r] - rs[r]) {
          rank -= re[r] - rs[r];
          ++r;
        }
        bead = sorted[rs[r] + rank];
        const int Nn = c.N[a];
        // tile-local l holds stencil index i = (l + X0 - sw) mod N if i < ngd
        const int i = wrap_near(l + wrap_near(X0[a] - bead_sw[3 * bead + a], Nn), Nn);
        if (i < ngd) {
          valid = true;
          const double Yv = Y[3 * bead + a];
          const int xc = (int)(Yv / c.dx);
          const int xg = xc - c.ngdh + (i + 1);
          const double xx = ((double)xg) * c.dx - Yv;
          if (sizeof(R) == 8) {
            wv.g = (R)(c.anorm * exp(-xx * xx / c.anorm2));
            wv.d = (R)(c.anormdip * exp(-xx * xx / c.anormdip2));
            wv.r = (R)(-xx / c.sigmadipsq);
          } else {
            const R xf = (R)xx;
            wv.g = (R)c.anorm * fs_exp<R>(-xf * xf / (R)c.anorm2);
            wv.d = (R)c.anormdip * fs_exp<R>(-xf * xf / (R)c.anormdip2);
            wv.r = -xf / (R)c.sigmadipsq;
          }
        }
        st.w[s][a][l] = wv;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, valid);
      if (act && l == 0) {
        st.mask[s][a] = (bal >> (lane & 16)) & 0xffffu;
        if (a == 0)
          for (int d = 0; d < 3; ++d) {
            st.f[s][d] = (R)F[3 * bead + d];
            st.th[s][d] = (R)(0.5 * T[3 * bead + d]);
          }
      }
    }
    __syncthreads();
    // beads reaching this warp's column (its x pair and z octet)
    unsigned col[CH / 32];
#pragma unroll
    for (int h = 0; h < CH / 32; ++h) {
      const int s = 32 * h + lane;
      unsigned mx = 0, mz = 0;
      if (s < nb) {
        mx = st.mask[s][0];
        mz = st.mask[s][2];
      }
      col[h] = __ballot_sync(0xffffffffu, ((mx >> (2 * bx)) & 3u) && ((mz >> (8 * bz)) & 0xffu));
    }
    const W4<R> *wxp = &st.w[0][0][px];
    const W4<R> *wzp = &st.w[0][2][pz];
    // two passes of four y pairs; per bead the x and z factors and the rotlet cross
    // terms are formed once per pass, each y row then needs one weight load:
    //   f_a += F_a gx gy gz + (T/2 x grad)_a gdx gdy gdz, regrouped by y
#pragma unroll 1
    for (int half = 0; half < 2; ++half) {
      KAcc<R> acc[4][3];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        acc[q][0].init();
        acc[q][1].init();
        acc[q][2].init();
      }
#pragma unroll
      for (int h = 0; h < CH / 32; ++h) {
        unsigned m = col[h];
        while (m) {
          const int s = 32 * h + __ffs(m) - 1;
          m &= m - 1;
          const unsigned my = (st.mask[s][1] >> (8 * half)) & 0xffu;  // y pairs 4 half .. 4 half + 3
          if (my == 0) continue;
          const W4<R> wx = wxp[s * 3 * FS_TILE], wz = wzp[s * 3 * FS_TILE];
          const R F0 = st.f[s][0], F1 = st.f[s][1], F2 = st.f[s][2];
          const R h0 = st.th[s][0], h1 = st.th[s][1], h2 = st.th[s][2];
          const R gxz = wx.g * wz.g, dxz = wx.d * wz.d;
          const R f0 = F0 * gxz, f1 = F1 * gxz, f2 = F2 * gxz;
          const R h2d = h2 * dxz, h0d = h0 * dxz;
          const R c0 = -h1 * wz.r * dxz, c1 = (-h2 * wx.r + h0 * wz.r) * dxz, c2 = h1 * wx.r * dxz;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            if ((my >> (2 * q)) & 3u) {
              const W4<R> wy = st.w[s][1][2 * (4 * half + q) + pyo];
              acc[q][0].add(f0 * wy.g + (h2d * wy.r + c0) * wy.d);
              acc[q][1].add(f1 * wy.g + c1 * wy.d);
              acc[q][2].add(f2 * wy.g + (c2 - h0d * wy.r) * wy.d);
            }
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int py = 2 * (4 * half + q) + pyo;
        const size_t m0 = ((size_t)(X0[0] + px) * c.N[1] + (X0[1] + py)) * c.N[2] + (X0[2] + pz);
        if (base == 0) {
          fgrid[m0] = acc[q][0].value();
          fgrid[N + m0] = acc[q][1].value();
          fgrid[2 * N + m0] = acc[q][2].value();
        } else {  // more candidates than one chunk: add in chunk order
          fgrid[m0] += acc[q][0].value();
          fgrid[N + m0] += acc[q][1].value();
          fgrid[2 * N + m0] += acc[q][2].value();
        }
      }
    }
  }
  if (total == 0)
    for (int by = 0; by < 8; ++by) {
      const size_t m0 = ((size_t)(X0[0] + px) * c.N[1] + (X0[1] + 2 * by + pyo)) * c.N[2] + (X0[2] + pz);
      fgrid[m0] = (R)0;
      fgrid[N + m0] = (R)0;
      fgrid[2 * N + m0] = (R)0;
    }
}

// ---- 2b. FP32 spread on packed pairs -------------------------------------------
// The FP32 chain's spread. k_spread_records32 writes each bead's record once per
// solve: stencil starts, F, T/2 and the weights (g, d, r, r d) per axis and
// stencil index, with the FP32 arithmetic of k_spread<float> (gaussian_setup,
// FCMfunctions.cpp:565-589: xx = xg dx - Y in double, then the float Gaussians).
// k_spread32 then runs one CTA (8 warps) per 16^3 tile, which stages tables of
// the tile's candidate beads (by tile coordinate, from their records) and covers
// its 16 column blocks in two passes; with the default 4 x 16 x 4 blocks, in
// pass p warp w owns x in [4(w&3), +4), z in [4cz, +4) with cz = (w>>2) + 2p;
// lane l owns x = 4(w&3) + (l&3), the z pair 4cz + 2((l>>2)&1) + {0, 1} and
// y = (l>>3) + 4k, k < 4: eight points held as four packed pairs per component
// (two blocks per warp even out the warps' bead counts; the block shape is a
// template knob). Per staged bead reaching the warp's column the lane forms the
// x-z factors of its pair once, then each covered y row costs three packed
// FMA chains and three packed Kahan updates:
//   y = term + nc, t = s + y, nc = y - (t - s), s = t      (nc = -c of Kahan)
// The sums run over the candidates in sorted bead order and are written once
// per point (s + nc): no atomics, bit-reproducible.
#define FS_SPREAD32_THREADS 256

// Record of the bead in sorted slot q (float4 units): [0] stencil starts (int),
// [1] F0, F1, F2, h0, [2] h1, h2, -, -, then (g, d, r, r d) for axis a and stencil
// index i at 3 + a ngd + i.
__host__ __device__ inline int spread_rec_len(int ngd) { return 3 + 3 * ngd; }

__global__ void k_spread_records32(const double *__restrict__ Y, const double *__restrict__ F,
                                   const double *__restrict__ T, const int *__restrict__ sorted,
                                   const int *__restrict__ bead_sw, int np, FcmConsts c, float4 *__restrict__ rec) {
  const int ngd = c.ngd, RL = spread_rec_len(ngd);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)np * RL) return;
  const int q = (int)(t / RL), e = (int)(t - (long long)q * RL);
  const int bead = sorted[q];
  float4 v;
  if (e == 0) {
    v = make_float4(__int_as_float(bead_sw[3 * bead]), __int_as_float(bead_sw[3 * bead + 1]),
                    __int_as_float(bead_sw[3 * bead + 2]), 0.f);
  } else if (e == 1) {
    v = make_float4((float)F[3 * bead], (float)F[3 * bead + 1], (float)F[3 * bead + 2], (float)(0.5 * T[3 * bead]));
  } else if (e == 2) {
    v = make_float4((float)(0.5 * T[3 * bead + 1]), (float)(0.5 * T[3 * bead + 2]), 0.f, 0.f);
  } else {
    const int a = (e - 3) / ngd, i = (e - 3) - a * ngd;
    const double Yv = Y[3 * bead + a];
    const int xc = (int)(Yv / c.dx);
    const int xg = xc - c.ngdh + (i + 1);
    const double xx = ((double)xg) * c.dx - Yv;
    const float xf = (float)xx;
    const float g = (float)c.anorm * expf(-xf * xf / (float)c.anorm2);
    const float d = (float)c.anormdip * expf(-xf * xf / (float)c.anormdip2);
    const float r = -xf / (float)c.sigmadipsq;
    v = make_float4(g, d, r, r * d);
  }
  rec[t] = v;
}


// the staged chunk: tables by tile coordinate, built straight from the records in
// global memory (spread32_smem bytes of dynamic shared memory)
template <int CH>
struct SpreadStage32 {
  float4 xw[CH][FS_TILE];                    // (g, d, r, -) by tile-local x
  float zg[CH][FS_TILE], zd[CH][FS_TILE], zr[CH][FS_TILE];  // by tile-local z
  float4 yw[CH][FS_TILE];                    // (g, g, d, d) by tile-local y
  float2 yrd[CH][FS_TILE];                   // (r d, r d)
  float4 fh[CH], hh[CH];                     // (F0, F1, F2, h0), (h1, h2, -, -): h = T / 2
  unsigned xzm[CH];                          // x coverage (16 bits) | z coverage (16 bits) << 16
  unsigned rows[CH];                         // y rows k with a covered y in [4k, 4k + 4)
};

template <int CH>
__host__ __device__ constexpr size_t spread32_smem(int) {
  return (sizeof(SpreadStage32<CH>) + 15) / 16 * 16;
}

// CX: the shape of a warp's column block, CX x 16 x (16 / CX) points (x, y, z),
// an autotuner knob (2, 4 or 8); a lane owns one x, one z pair and four y rows
template <int CH, int CX>
__global__ void __launch_bounds__(FS_SPREAD32_THREADS, 3)
    k_spread32(const int *__restrict__ bin_start, const float4 *__restrict__ rec, FcmConsts c,
               float *__restrict__ fgrid) {
  static_assert(CX == 2 || CX == 4 || CX == 8, "column widths");
  constexpr int CZ = FS_TILE / CX, NCX = FS_TILE / CX;  // z width; columns across x
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SpreadStage32<CH> &st = *reinterpret_cast<SpreadStage32<CH> *>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tile = blockIdx.x;
  const int tz = tile % c.nbin[2], ty = (tile / c.nbin[2]) % c.nbin[1], tx = tile / (c.nbin[2] * c.nbin[1]);
  const int X0[3] = {tx * FS_TILE, ty * FS_TILE, tz * FS_TILE};
  // candidate bins, the tile's own bin and the ones before it that a stencil
  // reaches (fs_cand_bins: K per axis), in the order (x, y, z) of k_spread;
  // thread r < K^3 reads combination r: per axis digit p in [0, K) names the bin
  // K - 1 - p before the tile's own (empty when it would repeat a bin on an axis
  // with fewer than K bins)
  __shared__ int cand_rs[27], cand_len[27];
  const int K = fs_cand_bins(c.ngd), nr = K * K * K;
  if (tid < nr) {
    const int tb[3] = {tx, ty, tz};
    const int pick[3] = {tid / (K * K), (tid / K) % K, tid % K};
    int bin = 0;
    bool valid = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int back = K - 1 - pick[d];
      valid = valid && back < c.nbin[d];
      bin = bin * c.nbin[d] + wrap_int(tb[d] - back, c.nbin[d]);
    }
    cand_rs[tid] = valid ? bin_start[bin] : 0;
    cand_len[tid] = valid ? bin_start[bin + 1] - bin_start[bin] : 0;
  }
  __syncthreads();
  int total = 0;
  for (int r = 0; r < nr; ++r) total += cand_len[r];
  const int ngd = c.ngd, RL = spread_rec_len(ngd);
  // staging of candidates [base, base + nb): tables by tile coordinate, eight
  // threads per bead slot (thread j takes x, y and z in {j, j + 8}), each reading
  // its slot's record (candidate base + sl: bin range r, rank q in it) from global
  // memory; not copying the records in first keeps a CTA at 55 KB of shared memory
  // with 64 beads per pass (92.5 KB with the copies), so three CTAs fit on an SM
  auto stage = [&](int base, int nb) {
    __syncthreads();  // the previous tables are no longer read
    const int j = tid & 7;
#pragma unroll 1
    for (int s0 = 0; s0 < CH; s0 += FS_SPREAD32_THREADS / 8) {
      const int sl = s0 + (tid >> 3);
      const bool act = sl < nb;
      bool cov[6] = {false, false, false, false, false, false};
      if (act) {
        int q = base + sl, r = 0;
        while (q >= cand_len[r]) {
          q -= cand_len[r];
          ++r;
        }
        const float4 *rw = rec + (size_t)(cand_rs[r] + q) * RL;
        const float4 hd = __ldg(rw);
        if (j == 0) {
          st.fh[sl] = __ldg(rw + 1);
          st.hh[sl] = __ldg(rw + 2);
        }
        const int swv[3] = {__float_as_int(hd.x), __float_as_int(hd.y), __float_as_int(hd.z)};
        float4 w[6];
#pragma unroll
        for (int it = 0; it < 6; ++it) {
          const int a = it >> 1, l = j + 8 * (it & 1), Nn = c.N[a];
          const int i = wrap_near(l + wrap_near(X0[a] - swv[a], Nn), Nn);
          cov[it] = i < ngd;
          w[it] = cov[it] ? __ldg(rw + 3 + a * ngd + i) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        st.xw[sl][j] = w[0];
        st.xw[sl][j + 8] = w[1];
        st.yw[sl][j] = make_float4(w[2].x, w[2].x, w[2].y, w[2].y);
        st.yrd[sl][j] = make_float2(w[2].w, w[2].w);
        st.yw[sl][j + 8] = make_float4(w[3].x, w[3].x, w[3].y, w[3].y);
        st.yrd[sl][j + 8] = make_float2(w[3].w, w[3].w);
        st.zg[sl][j] = w[4].x;
        st.zd[sl][j] = w[4].y;
        st.zr[sl][j] = w[4].z;
        st.zg[sl][j + 8] = w[5].x;
        st.zd[sl][j + 8] = w[5].y;
        st.zr[sl][j + 8] = w[5].z;
      }
      // coverage masks by ballot: lanes 8q .. 8q+7 of this warp hold slot s0 + 4 warp + q
      unsigned bal[6];
#pragma unroll
      for (int it = 0; it < 6; ++it) bal[it] = __ballot_sync(0xffffffffu, cov[it]);
      if (act && j == 0) {
        const int sh = lane & 24;
        unsigned m3[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) m3[a] = ((bal[2 * a] >> sh) & 0xffu) | (((bal[2 * a + 1] >> sh) & 0xffu) << 8);
        st.xzm[sl] = m3[0] | (m3[2] << 16);
        unsigned rows = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) rows |= ((m3[1] >> (4 * k)) & 0xfu) ? (1u << k) : 0u;
        st.rows[sl] = rows;
      }
    }
    __syncthreads();
  };
  const bool one_chunk = total <= CH;
  if (one_chunk && total > 0) stage(0, total);  // both column passes read these tables
  // two column passes over the tile's 16 column blocks: in pass p warp w owns block
  // w + 8 p, x in [CX cx, +CX) and z in [CZ cz, +CZ) (CX = 4: the lane roles of the
  // header); a lane owns x = CX cx + lane % CX, the z pair (lane / CX) % (CZ / 2)
  // and the four y rows ly + 4 k, ly = lane / 8
  // (8 is a multiple of NCX, so a warp keeps its x columns in both passes)
  const int ly = lane >> 3, cx = warp % NCX;
  const int xl = CX * cx + (lane % CX);
#pragma unroll 1
  for (int pass = 0; pass < 2; ++pass) {
    const int cz = warp / NCX + (8 / NCX) * pass;
    const int zl = CZ * cz + 2 * ((lane / CX) % (CZ / 2));
    f2p s[4][3], nc[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int a = 0; a < 3; ++a) s[k][a] = nc[k][a] = 0ull;
    for (int base = 0; base < total; base += CH) {
      const int nb = min(CH, total - base);
      if (!one_chunk) stage(base, nb);  // block-uniform
      // staged beads reaching this warp's column
      unsigned col[CH / 32];
#pragma unroll
      for (int h = 0; h < CH / 32; ++h) {
        const int sl = 32 * h + lane;
        bool hit = false;
        if (sl < nb) {
          const unsigned m = st.xzm[sl];
          hit = ((m >> (CX * cx)) & ((1u << CX) - 1u)) && ((m >> (16 + CZ * cz)) & ((1u << CZ) - 1u)) && st.rows[sl];
        }
        col[h] = __ballot_sync(0xffffffffu, hit);
      }
#pragma unroll
      for (int h = 0; h < CH / 32; ++h) {
        unsigned m = col[h];
        while (m) {
          const int sl = 32 * h + __ffs(m) - 1;
          m &= m - 1;
          const unsigned rows = st.rows[sl];
          const float4 wx = st.xw[sl][xl];
          const float2 gz = *reinterpret_cast<const float2 *>(&st.zg[sl][zl]);
          const float2 dz = *reinterpret_cast<const float2 *>(&st.zd[sl][zl]);
          const float2 rz = *reinterpret_cast<const float2 *>(&st.zr[sl][zl]);
          const float4 fh = st.fh[sl];  // F0, F1, F2, h0 (h = T / 2, GA_setup :536-547)
          const float4 hh = st.hh[sl];  // h1, h2
          // per z of the pair: f_a = F_a gx gz, the rotlet factors of k_spread (d = gdx gdz)
          const float gxz0 = wx.x * gz.x, gxz1 = wx.x * gz.y;
          const float dxz0 = wx.y * dz.x, dxz1 = wx.y * dz.y;
          const f2p f0 = f2_pack(fh.x * gxz0, fh.x * gxz1);
          const f2p f1 = f2_pack(fh.y * gxz0, fh.y * gxz1);
          const f2p f2v = f2_pack(fh.z * gxz0, fh.z * gxz1);
          const f2p h2d = f2_pack(hh.y * dxz0, hh.y * dxz1);
          const f2p mh0d = f2_pack(-fh.w * dxz0, -fh.w * dxz1);
          const f2p c0 = f2_pack(-hh.x * rz.x * dxz0, -hh.x * rz.y * dxz1);
          const f2p c1 = f2_pack((-hh.y * wx.z + fh.w * rz.x) * dxz0, (-hh.y * wx.z + fh.w * rz.y) * dxz1);
          const f2p c2 = f2_pack(hh.x * wx.z * dxz0, hh.x * wx.z * dxz1);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            if (rows & (1u << k)) {
              const ulonglong2 gd = *reinterpret_cast<const ulonglong2 *>(&st.yw[sl][ly + 4 * k]);
              const f2p rd = *reinterpret_cast<const f2p *>(&st.yrd[sl][ly + 4 * k]);
              f2p y, t;
              // f0 g + h2d (r d) + c0 d
              y = f2_fma(f0, gd.x, f2_fma(h2d, rd, f2_fma(c0, gd.y, nc[k][0])));
              t = f2_add(s[k][0], y);
              nc[k][0] = f2_sub(y, f2_sub(t, s[k][0]));
              s[k][0] = t;
              // f1 g + c1 d
              y = f2_fma(f1, gd.x, f2_fma(c1, gd.y, nc[k][1]));
              t = f2_add(s[k][1], y);
              nc[k][1] = f2_sub(y, f2_sub(t, s[k][1]));
              s[k][1] = t;
              // f2 g + c2 d - h0d (r d)
              y = f2_fma(f2v, gd.x, f2_fma(mh0d, rd, f2_fma(c2, gd.y, nc[k][2])));
              t = f2_add(s[k][2], y);
              nc[k][2] = f2_sub(y, f2_sub(t, s[k][2]));
              s[k][2] = t;
            }
          }
        }
      }
    }
    // one write per point: s - c
    const size_t N = (size_t)c.N[0] * c.N[1] * c.N[2];
    const int gx = X0[0] + xl, gz0 = X0[2] + zl;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const size_t m0 = ((size_t)gx * c.N[1] + (X0[1] + ly + 4 * k)) * c.N[2] + gz0;
#pragma unroll
      for (int a = 0; a < 3; ++a)
        *reinterpret_cast<float2 *>(fgrid + a * N + m0) = f2_unpack(f2_add(s[k][a], nc[k][a]));
    }
  }
}

// ---- 4. Stokes projection -----------------------------------------------------
template <typename R>
struct Cplx;
template <>
struct Cplx<double> { typedef double2 T; };
template <>
struct Cplx<float> { typedef float2 T; };

template <typename R>
__device__ inline void project_mode(R q1, R q2, R q3, R a1, R a2, R a3, R total, R &u1, R &u2, R &u3) {
  const R qq = q2 * q2 + q1 * q1 + (R)1e-18;
  const R norm = (R)1.0 / (qq + q3 * q3);
  const R kdotf = (q1 * a1 + q2 * a2 + q3 * a3) * norm;
  u1 = norm * (a1 - q1 * kdotf) / total;
  u2 = norm * (a2 - q2 * kdotf) / total;
  u3 = norm * (a3 - q3 * kdotf) / total;
}

template <typename R>
__device__ inline R wavenumber(int i, int n, R ff) {
  return (R)((i <= n / 2) ? i : i - n) * ff;
}

// modes with 0 < kz < nz/2 (each stored once in the half spectrum)
template <typename R>
__global__ void k_project(typename Cplx<R>::T *__restrict__ fh, size_t NH, int nx, int ny, int nz, int nzh, R ffx,
                          R ffy, R ffz, R total) {
  typedef typename Cplx<R>::T C;
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= NH) return;
  const int k = (int)(idx % nzh);
  if (k == 0 || 2 * k == nz) return;
  const int j = (int)((idx / nzh) % ny);
  const int i = (int)(idx / ((size_t)nzh * ny));
  const R q1 = wavenumber<R>(i, nx, ffx), q2 = wavenumber<R>(j, ny, ffy), q3 = (R)k * ffz;
  C a = fh[idx], b = fh[NH + idx], d = fh[2 * NH + idx];
  C ua, ub, ud;
  project_mode<R>(q1, q2, q3, a.x, b.x, d.x, total, ua.x, ub.x, ud.x);
  project_mode<R>(q1, q2, q3, a.y, b.y, d.y, total, ua.y, ub.y, ud.y);
  fh[idx] = ua;
  fh[NH + idx] = ub;
  fh[2 * NH + idx] = ud;
}

// kz = 0 and kz = nz/2 planes. The reference's inverse real transform uses
// only the real part of the last axis's DC and Nyquist coefficients after the
// complex transforms of the other axes, which equals inverting the Hermitian
// part of these planes: u_sym(i,j) = (u(i,j) + conj(u(-i,-j))) / 2. Writing
// that exactly Hermitian plane makes the C2R result well defined.
template <typename R>
__global__ void k_project_planes(typename Cplx<R>::T *__restrict__ fh, size_t NH, int nx, int ny, int nz, int nzh,
                                 R ffx, R ffy, R ffz, R total) {
  typedef typename Cplx<R>::T C;
  const int ij = blockIdx.x * blockDim.x + threadIdx.x;
  if (ij >= nx * ny) return;
  const int kp = blockIdx.y == 0 ? 0 : nz / 2;
  if (blockIdx.y == 1 && (nz % 2 != 0 || nz / 2 == 0)) return;
  const int i = ij / ny, j = ij % ny;
  const int ip = (nx - i) % nx, jp = (ny - j) % ny;
  const int ijp = ip * ny + jp;
  if (ijp < ij) return;  // the partner handles the pair
  const size_t m = (size_t)ij * nzh + kp, mp = (size_t)ijp * nzh + kp;
  const R q3 = (R)kp * ffz;
  C u[3], up[3];
  {
    const R q1 = wavenumber<R>(i, nx, ffx), q2 = wavenumber<R>(j, ny, ffy);
    C a = fh[m], b = fh[NH + m], d = fh[2 * NH + m];
    project_mode<R>(q1, q2, q3, a.x, b.x, d.x, total, u[0].x, u[1].x, u[2].x);
    project_mode<R>(q1, q2, q3, a.y, b.y, d.y, total, u[0].y, u[1].y, u[2].y);
  }
  {
    const R q1 = wavenumber<R>(ip, nx, ffx), q2 = wavenumber<R>(jp, ny, ffy);
    C a = fh[mp], b = fh[NH + mp], d = fh[2 * NH + mp];
    project_mode<R>(q1, q2, q3, a.x, b.x, d.x, total, up[0].x, up[1].x, up[2].x);
    project_mode<R>(q1, q2, q3, a.y, b.y, d.y, total, up[0].y, up[1].y, up[2].y);
  }
  const bool zero_mode = (kp == 0 && ij == 0);
#pragma unroll
  for (int cpt = 0; cpt < 3; ++cpt) {
    C s;
    s.x = (R)0.5 * (u[cpt].x + up[cpt].x);
    s.y = (R)0.5 * (u[cpt].y - up[cpt].y);
    if (zero_mode) s.x = s.y = (R)0;
    if (ijp == ij) s.y = (R)0;
    fh[(size_t)cpt * NH + m] = s;
    if (ijp != ij) {
      C sc;
      sc.x = s.x;
      sc.y = -s.y;
      fh[(size_t)cpt * NH + mp] = sc;
    }
  }
}

// ---- 6. interpolation -------------------------------------------------------
template <typename R>
struct InterpWarp {
  R g[3][FS_NGD_MAX], gd[3][FS_NGD_MAX], r[3][FS_NGD_MAX];
  int ind[3][FS_NGD_MAX];
};
template <typename R>
struct __align__(4 * sizeof(R)) XY4 {
  R gg, dd, rx, ry;  // gx gy, gdx gdy, rx, ry of one (i, j) of the x-y stencil
};
// dynamic shared memory per warp: the per-axis tables, then per (i, j) the
// products and the grid offset of (x_i, y_j, 0)
template <typename R>
__host__ __device__ constexpr size_t interp_xy_offset() {
  return (sizeof(InterpWarp<R>) + 4 * sizeof(R) - 1) / (4 * sizeof(R)) * (4 * sizeof(R));
}
// rounded up to 32 bytes, so that every warp's tables and XY4 entries keep their
// alignment also for odd ngd (ngd^2 (sizeof(XY4) + 8) is then an odd multiple of 8)
template <typename R>
__host__ __device__ constexpr size_t interp_warp_bytes(int ngd) {
  return (interp_xy_offset<R>() + (size_t)ngd * ngd * (sizeof(XY4<R>) + sizeof(long long)) + 31) / 32 * 32;
}

// One warp per bead; lanes take the stencil points p = lane + 32 t (z fastest),
// all 32 lanes busy. FP32 mode multiplies in FP32 and accumulates in FP64 per lane.
template <typename R, int WPB>
__global__ void __launch_bounds__(32 * WPB) k_interp(const R *__restrict__ u, const double *__restrict__ Y,
                                                     const int *__restrict__ order, const int *__restrict__ bead_sw,
                                                     int np, FcmConsts c, double *__restrict__ V,
                                                     double *__restrict__ W) {
  extern __shared__ __align__(32) unsigned char interp_smem[];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int wid = blockIdx.x * WPB + wl;
  if (wid >= np) return;
  const int b = order[wid];
  const int ngd = c.ngd, n2 = ngd * ngd, n3 = n2 * ngd;
  unsigned char *base = interp_smem + (size_t)wl * interp_warp_bytes<R>(ngd);
  InterpWarp<R> &s = *reinterpret_cast<InterpWarp<R> *>(base);
  XY4<R> *xy = reinterpret_cast<XY4<R> *>(base + interp_xy_offset<R>());
  long long *off = reinterpret_cast<long long *>(xy + n2);
  for (int a = 0; a < 3; ++a) {  // lane i < ngd <= 20 takes stencil index i of each axis
    const int i = lane;
    if (i >= ngd) continue;
    const double Yv = Y[3 * b + a];
    const int xc = (int)(Yv / c.dx);
    const int xg = xc - c.ngdh + (i + 1);
    const int ix = bead_sw[3 * b + a] + i;  // (stencil start + i) mod N, as gaussian_setup's indx
    s.ind[a][i] = ix >= c.N[a] ? ix - c.N[a] : ix;
    const double xx = ((double)xg) * c.dx - Yv;
    if (sizeof(R) == 8) {
      s.g[a][i] = (R)(c.anorm * exp(-xx * xx / c.anorm2));
      s.gd[a][i] = (R)(c.anormdip * exp(-xx * xx / c.anormdip2));
      s.r[a][i] = (R)(-xx / c.sigmadipsq);
    } else {
      const R xf = (R)xx;
      s.g[a][i] = (R)c.anorm * fs_exp<R>(-xf * xf / (R)c.anorm2);
      s.gd[a][i] = (R)c.anormdip * fs_exp<R>(-xf * xf / (R)c.anormdip2);
      s.r[a][i] = -xf / (R)c.sigmadipsq;
    }
  }
  __syncwarp();
  for (int ij = lane; ij < n2; ij += 32) {
    const int i = ij / ngd, j = ij - i * ngd;
    XY4<R> e;
    e.gg = s.g[0][i] * s.g[1][j];
    e.dd = s.gd[0][i] * s.gd[1][j];
    e.rx = s.r[0][i];
    e.ry = s.r[1][j];
    xy[ij] = e;
    off[ij] = ((long long)s.ind[0][i] * c.N[1] + s.ind[1][j]) * c.N[2];
  }
  __syncwarp();
  const size_t N = (size_t)c.N[0] * c.N[1] * c.N[2];
  const R *ux = u, *uy = u + N, *uz = u + 2 * N;
  double v0 = 0, v1 = 0, v2 = 0, w0 = 0, w1 = 0, w2 = 0;
  // point p = ij * ngd + k; a step of 32 points advances (ij, k) by (32 / ngd, 32 % ngd)
  // (loads one point at a time: four points in flight per lane, at 64 registers,
  // ran 0.97 ms at 512^3 against 0.72 ms for this loop; the gathers are bound by
  // the load units, not by latency; the z tables packed into one float4 per index,
  // three shared loads per point fewer, left it unchanged)
  const int dij = 32 / ngd, dk = 32 - dij * ngd;
  int ij = lane / ngd, k = lane - ij * ngd;
  for (int p = lane; p < n3; p += 32) {
    const XY4<R> e = xy[ij];
    const long long m = off[ij] + s.ind[2][k];
    const R temp = e.gg * s.g[2][k];    // (gx gy) gz, the reference's order
    const R tempd = e.dd * s.gd[2][k];
    const R zz = s.r[2][k];
    const R a0 = ux[m], a1 = uy[m], a2 = uz[m];
    v0 += (double)(a0 * temp);
    v1 += (double)(a1 * temp);
    v2 += (double)(a2 * temp);
    w0 += (double)((a2 * e.ry - a1 * zz) * tempd);
    w1 += (double)((a0 * zz - a2 * e.rx) * tempd);
    w2 += (double)((a1 * e.rx - a0 * e.ry) * tempd);
    k += dk;
    ij += dij;
    if (k >= ngd) {
      k -= ngd;
      ++ij;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v0 += __shfl_xor_sync(0xffffffffu, v0, o);
    v1 += __shfl_xor_sync(0xffffffffu, v1, o);
    v2 += __shfl_xor_sync(0xffffffffu, v2, o);
    w0 += __shfl_xor_sync(0xffffffffu, w0, o);
    w1 += __shfl_xor_sync(0xffffffffu, w1, o);
    w2 += __shfl_xor_sync(0xffffffffu, w2, o);
  }
  if (lane == 0) {
    const double norm = c.dx * c.dx * c.dx;
    V[3 * b + 0] = v0 * norm;
    V[3 * b + 1] = v1 * norm;
    V[3 * b + 2] = v2 * norm;
    W[3 * b + 0] = -0.5 * w0 * norm;
    W[3 * b + 1] = -0.5 * w1 * norm;
    W[3 * b + 2] = -0.5 * w2 * norm;
  }
}


// FP32 interpolation with float4 gathers along z. The stencil's z run of ngd
// points starting at zs lies in nq = ceil(((zs & 3) + ngd) / 4) aligned quads of
// four points (a quad's first index is a multiple of 4; with Nz a multiple of 4 and
// Nz >= ngd + 6 the quads of one run are distinct modulo Nz). A lane takes (ij,
// quad) slots: one 16-byte load per component instead of four 4-byte ones, z weights
// per quad position (zero off the run), the quad's four products summed in FP32
// and the sum added in FP64. The products are k_interp<float>'s.
constexpr int IQ_MAX = (FS_NGD_MAX + 6) / 4;  // quads a z run of ngd points can touch
struct InterpQuad {
  float4 wg[IQ_MAX], wd[IQ_MAX], wr[IQ_MAX];  // g, gd, r of the quad's four points (0 off the run)
  int zq[IQ_MAX];                              // the quad's first z index
};
__host__ __device__ constexpr size_t interp_q_quad_offset() { return (sizeof(InterpWarp<float>) + 15) / 16 * 16; }
__host__ __device__ constexpr size_t interp_q_xy_offset() {
  return (interp_q_quad_offset() + sizeof(InterpQuad) + 15) / 16 * 16;
}
__host__ __device__ constexpr size_t interp_q_warp_bytes(int ngd) {
  return (interp_q_xy_offset() + (size_t)ngd * ngd * (sizeof(XY4<float>) + sizeof(long long)) + 31) / 32 * 32;
}
inline bool interp_q_ok(const fs_ctx *c) { return c->nz % 4 == 0 && c->nz >= c->p.ngd + 6; }

template <int WPB>
__global__ void __launch_bounds__(32 * WPB) k_interp_q(const float *__restrict__ u, const double *__restrict__ Y,
                                                       const int *__restrict__ order, const int *__restrict__ bead_sw,
                                                       int np, FcmConsts c, double *__restrict__ V,
                                                       double *__restrict__ W) {
  extern __shared__ __align__(32) unsigned char interp_smem[];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int wid = blockIdx.x * WPB + wl;
  if (wid >= np) return;
  const int b = order[wid];
  const int ngd = c.ngd, n2 = ngd * ngd, Nz = c.N[2];
  unsigned char *base = interp_smem + (size_t)wl * interp_q_warp_bytes(ngd);
  InterpWarp<float> &s = *reinterpret_cast<InterpWarp<float> *>(base);
  InterpQuad &q = *reinterpret_cast<InterpQuad *>(base + interp_q_quad_offset());
  XY4<float> *xy = reinterpret_cast<XY4<float> *>(base + interp_q_xy_offset());
  long long *off = reinterpret_cast<long long *>(xy + n2);
  for (int a = 0; a < 3; ++a) {  // lane i < ngd takes stencil index i of each axis (as k_interp)
    const int i = lane;
    if (i >= ngd) continue;
    const double Yv = Y[3 * b + a];
    const int xc = (int)(Yv / c.dx);
    const int xg = xc - c.ngdh + (i + 1);
    const int ix = bead_sw[3 * b + a] + i;
    s.ind[a][i] = ix >= c.N[a] ? ix - c.N[a] : ix;
    const double xx = ((double)xg) * c.dx - Yv;
    const float xf = (float)xx;
    s.g[a][i] = (float)c.anorm * fs_exp<float>(-xf * xf / (float)c.anorm2);
    s.gd[a][i] = (float)c.anormdip * fs_exp<float>(-xf * xf / (float)c.anormdip2);
    s.r[a][i] = -xf / (float)c.sigmadipsq;
  }
  __syncwarp();
  const int zs = s.ind[2][0];
  const int nq = ((zs & 3) + ngd + 3) >> 2;
  if (lane < nq) {
    int z0 = (zs & ~3) + 4 * lane;
    if (z0 >= Nz) z0 -= Nz;
    float w[3][4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      int k = z0 + t - zs;
      if (k < 0) k += Nz;
      const bool on = k < ngd;
      const int kk = on ? k : 0;  // the tables are read only inside the run
      w[0][t] = on ? s.g[2][kk] : 0.f;
      w[1][t] = on ? s.gd[2][kk] : 0.f;
      w[2][t] = on ? s.r[2][kk] : 0.f;
    }
    q.wg[lane] = make_float4(w[0][0], w[0][1], w[0][2], w[0][3]);
    q.wd[lane] = make_float4(w[1][0], w[1][1], w[1][2], w[1][3]);
    q.wr[lane] = make_float4(w[2][0], w[2][1], w[2][2], w[2][3]);
    q.zq[lane] = z0;
  }
  for (int ij = lane; ij < n2; ij += 32) {
    const int i = ij / ngd, j = ij - i * ngd;
    XY4<float> e;
    e.gg = s.g[0][i] * s.g[1][j];
    e.dd = s.gd[0][i] * s.gd[1][j];
    e.rx = s.r[0][i];
    e.ry = s.r[1][j];
    xy[ij] = e;
    off[ij] = ((long long)s.ind[0][i] * c.N[1] + s.ind[1][j]) * Nz;
  }
  __syncwarp();
  const size_t N = (size_t)c.N[0] * c.N[1] * Nz;
  const float *ux = u, *uy = u + N, *uz = u + 2 * N;
  double v0 = 0, v1 = 0, v2 = 0, w0 = 0, w1 = 0, w2 = 0;
  // slot sl = ij * nq + qi; a step of 32 slots advances (ij, qi) by (32 / nq, 32 % nq)
  const int nslot = n2 * nq, dij = 32 / nq, dq = 32 - dij * nq;
  int ij = lane / nq, qi = lane - ij * nq;
  for (int sl = lane; sl < nslot; sl += 32) {
    const XY4<float> e = xy[ij];
    const long long m = off[ij] + q.zq[qi];
    const float4 a0 = __ldg(reinterpret_cast<const float4 *>(ux + m));
    const float4 a1 = __ldg(reinterpret_cast<const float4 *>(uy + m));
    const float4 a2 = __ldg(reinterpret_cast<const float4 *>(uz + m));
    const float4 g = q.wg[qi], gd = q.wd[qi], r = q.wr[qi];
    float p0 = 0.f, p1 = 0.f, p2 = 0.f, p3 = 0.f, p4 = 0.f, p5 = 0.f;
    auto acc = [&](float x0, float x1, float x2, float gz, float gdz, float zz) {
      const float temp = e.gg * gz;  // (gx gy) gz, the reference's order
      const float tempd = e.dd * gdz;
      p0 += x0 * temp;
      p1 += x1 * temp;
      p2 += x2 * temp;
      p3 += (x2 * e.ry - x1 * zz) * tempd;
      p4 += (x0 * zz - x2 * e.rx) * tempd;
      p5 += (x1 * e.rx - x0 * e.ry) * tempd;
    };
    acc(a0.x, a1.x, a2.x, g.x, gd.x, r.x);
    acc(a0.y, a1.y, a2.y, g.y, gd.y, r.y);
    acc(a0.z, a1.z, a2.z, g.z, gd.z, r.z);
    acc(a0.w, a1.w, a2.w, g.w, gd.w, r.w);
    v0 += (double)p0;
    v1 += (double)p1;
    v2 += (double)p2;
    w0 += (double)p3;
    w1 += (double)p4;
    w2 += (double)p5;
    qi += dq;
    ij += dij;
    if (qi >= nq) {
      qi -= nq;
      ++ij;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v0 += __shfl_xor_sync(0xffffffffu, v0, o);
    v1 += __shfl_xor_sync(0xffffffffu, v1, o);
    v2 += __shfl_xor_sync(0xffffffffu, v2, o);
    w0 += __shfl_xor_sync(0xffffffffu, w0, o);
    w1 += __shfl_xor_sync(0xffffffffu, w1, o);
    w2 += __shfl_xor_sync(0xffffffffu, w2, o);
  }
  if (lane == 0) {
    const double norm = c.dx * c.dx * c.dx;
    V[3 * b + 0] = v0 * norm;
    V[3 * b + 1] = v1 * norm;
    V[3 * b + 2] = v2 * norm;
    W[3 * b + 0] = -0.5 * w0 * norm;
    W[3 * b + 1] = -0.5 * w1 * norm;
    W[3 * b + 2] = -0.5 * w2 * norm;
  }
}

template <typename A, typename B>
__global__ void k_convert(const A *__restrict__ in, B *__restrict__ out, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (B)in[i];
}

__global__ void k_friction(const double *__restrict__ F, const double *__restrict__ T, double *__restrict__ V,
                           double *__restrict__ W, int n3, double a1, double a2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) {
    V[i] = a1 * F[i];
    W[i] = a2 * T[i];
  }
}

FcmConsts make_consts(const fs_ctx *c) {
  FcmConsts k;
  k.N[0] = c->nx;
  k.N[1] = c->ny;
  k.N[2] = c->nz;
  k.gnx = c->slab_nx > 0 ? c->slab_nx : c->nx;
  k.x0 = c->slab_nx > 0 ? c->slab_x0 : 0;
  k.ngd = c->p.ngd;
  k.ngdh = c->p.ngd / 2;
  for (int d = 0; d < 3; ++d) k.nbin[d] = c->nbin[d];
  k.dx = c->p.dx;
  const double PI = FS_PI;
  k.sigmadipsq = c->p.sigma_dip * c->p.sigma_dip;
  k.anormdip = 1.0 / sqrt(2.0 * PI * k.sigmadipsq);
  k.anormdip2 = 2.0 * k.sigmadipsq;
  const double sigmasq = c->p.sigma * c->p.sigma;
  k.anorm = 1.0 / sqrt(2.0 * PI * sigmasq);
  k.anorm2 = 2.0 * sigmasq;
  return k;
}

fs_status ensure_plans(fs_ctx *c, int prec) {
  if (c->plan_ok[prec]) return FS_OK;
  int n[3] = {c->nx, c->ny, c->nz};
  size_t ws = 0;
  if (cufftCreate(&c->plan_fwd[prec]) != CUFFT_SUCCESS) return FS_ERR_CUFFT;
  if (cufftCreate(&c->plan_inv[prec]) != CUFFT_SUCCESS) return FS_ERR_CUFFT;
  cufftType tf = prec == FS_PREC_FP64 ? CUFFT_D2Z : CUFFT_R2C;
  cufftType ti = prec == FS_PREC_FP64 ? CUFFT_Z2D : CUFFT_C2R;
  if (cufftMakePlanMany(c->plan_fwd[prec], 3, n, NULL, 1, 0, NULL, 1, 0, tf, 3, &ws) != CUFFT_SUCCESS)
    return FS_ERR_CUFFT;
  c->bytes += ws;
  if (cufftMakePlanMany(c->plan_inv[prec], 3, n, NULL, 1, 0, NULL, 1, 0, ti, 3, &ws) != CUFFT_SUCCESS)
    return FS_ERR_CUFFT;
  c->bytes += ws;
  if (cufftSetStream(c->plan_fwd[prec], c->stream) != CUFFT_SUCCESS) return FS_ERR_CUFFT;
  if (cufftSetStream(c->plan_inv[prec], c->stream) != CUFFT_SUCCESS) return FS_ERR_CUFFT;
  c->plan_ok[prec] = true;
  return FS_OK;
}

template <typename R>
fs_status flow_solve_t(fs_ctx *c) {
  const int prec = sizeof(R) == 8 ? FS_PREC_FP64 : FS_PREC_FP32;
  if (prec == FS_PREC_FP32 && c->fft_tw && c->tune_fft32 == 0) return fft32_flow_solve(c);
  FS_TRY(ensure_plans(c, prec));
  cufftResult r;
  {
    ProfScope ps(c, FS_STAGE_FFT_FWD);
    if (prec == FS_PREC_FP64)
      r = cufftExecD2Z(c->plan_fwd[prec], (cufftDoubleReal *)c->grid_real, (cufftDoubleComplex *)c->grid_cplx);
    else
      r = cufftExecR2C(c->plan_fwd[prec], (cufftReal *)c->grid_real, (cufftComplex *)c->grid_cplx);
  }
  if (r != CUFFT_SUCCESS) return FS_ERR_CUFFT;
  const double TwoPI = 2. * FS_PI;
  const R ffx = (R)(TwoPI / (c->nx * c->p.dx)), ffy = (R)(TwoPI / (c->ny * c->p.dx)),
          ffz = (R)(TwoPI / (c->nz * c->p.dx));
  const R total = (R)((double)c->nx * (double)c->ny * (double)c->nz);
  typedef typename Cplx<R>::T C;
  C *fh = (C *)c->grid_cplx;
  {
    ProfScope ps(c, FS_STAGE_PROJECT);
    k_project<R><<<fs_blocks((long long)c->NH, 256), 256, 0, c->stream>>>(fh, c->NH, c->nx, c->ny, c->nz, c->nzh,
                                                                            ffx, ffy, ffz, total);
    FS_LAUNCH_CHECK();
    dim3 gp(fs_blocks((long long)c->nx * c->ny, 256), 2);
    k_project_planes<R><<<gp, 256, 0, c->stream>>>(fh, c->NH, c->nx, c->ny, c->nz, c->nzh, ffx, ffy, ffz, total);
    FS_LAUNCH_CHECK();
  }
  {
    ProfScope ps(c, FS_STAGE_FFT_INV);
    if (prec == FS_PREC_FP64)
      r = cufftExecZ2D(c->plan_inv[prec], (cufftDoubleComplex *)c->grid_cplx, (cufftDoubleReal *)c->grid_real);
    else
      r = cufftExecC2R(c->plan_inv[prec], (cufftComplex *)c->grid_cplx, (cufftReal *)c->grid_real);
  }
  if (r != CUFFT_SUCCESS) return FS_ERR_CUFFT;
  return FS_OK;
}

// binning, sort and the spread of the force grid into c->grid_real (R precision)
template <typename R>
fs_status spread_t(fs_ctx *c, const FcmConsts &k, const double *Y, const double *F, const double *T, int np) {
  if (np > 0) {
    k_fcm_bin_keys<<<fs_blocks(np, 256), 256, 0, c->stream>>>(Y, np, k, c->bins.key, c->bead_sw);
    FS_LAUNCH_CHECK();
  }
  FS_TRY(fs_sort_run(&c->bins, np, c->stream));
  if (sizeof(R) == 4) {
    const float4 *rec = (const float4 *)c->spread_wb;
    if (np > 0) {
      k_spread_records32<<<fs_blocks((long long)np * spread_rec_len(k.ngd), 256), 256, 0, c->stream>>>(
          Y, F, T, c->bins.sorted, c->bead_sw, np, k, c->spread_wb);
      FS_LAUNCH_CHECK();
    }
    ProfScope pk(c, FS_STAGE_K_SPREAD);
    const int ch = c->tune_spread_chunk, cx = c->tune_spread_cols;
#define FS_SPREAD32_LAUNCH(CHV, CXV)                                                                             \
  k_spread32<CHV, CXV><<<c->nbins, FS_SPREAD32_THREADS, spread32_smem<CHV>(k.ngd), c->stream>>>(c->bins.start, rec, \
                                                                                                 k, (float *)c->grid_real)
    if (ch == 32 && cx == 2) FS_SPREAD32_LAUNCH(32, 2);
    else if (ch == 32 && cx == 8) FS_SPREAD32_LAUNCH(32, 8);
    else if (ch == 32) FS_SPREAD32_LAUNCH(32, 4);
    else if (cx == 2) FS_SPREAD32_LAUNCH(64, 2);
    else if (cx == 8) FS_SPREAD32_LAUNCH(64, 8);
    else FS_SPREAD32_LAUNCH(64, 4);
#undef FS_SPREAD32_LAUNCH
  } else if (c->tune_spread_chunk == 32) {
    ProfScope pk(c, FS_STAGE_K_SPREAD);
    k_spread<R, 32><<<c->nbins, FS_SPREAD_THREADS, sizeof(SpreadStage<R, 32>), c->stream>>>(
        Y, F, T, c->bins.start, c->bins.sorted, c->bead_sw, k, (R *)c->grid_real);
  } else {
    ProfScope pk(c, FS_STAGE_K_SPREAD);
    k_spread<R, 64><<<c->nbins, FS_SPREAD_THREADS, sizeof(SpreadStage<R, 64>), c->stream>>>(
        Y, F, T, c->bins.start, c->bins.sorted, c->bead_sw, k, (R *)c->grid_real);
  }
  FS_LAUNCH_CHECK();
  return FS_OK;
}

// interpolation of U, Omega from the velocity grid in c->grid_real (R precision); the
// beads must have been binned (k_fcm_bin_keys + sort) for this Y
template <typename R>
fs_status interp_t(fs_ctx *c, const FcmConsts &k, const double *Y, double *V, double *W, int np) {
  if (np <= 0) return FS_OK;
  ProfScope ps(c, FS_STAGE_INTERP);
  ProfScope pk(c, FS_STAGE_K_INTERP);
  const R *ug = (const R *)c->grid_real;
  if constexpr (sizeof(R) == 4) {
    if (interp_q_ok(c)) {  // float4 gathers along z
      const size_t wq = interp_q_warp_bytes(c->p.ngd);
      const int wpb = (c->tune_interp_wpb == 16 && 16 * wq > FS_SMEM_MAX) ? 8 : c->tune_interp_wpb;
      if (wpb == 4)
        k_interp_q<4><<<fs_blocks(np, 4), 128, 4 * wq, c->stream>>>(ug, Y, c->bins.sorted, c->bead_sw, np, k, V, W);
      else if (wpb == 16)
        k_interp_q<16><<<fs_blocks(np, 16), 512, 16 * wq, c->stream>>>(ug, Y, c->bins.sorted, c->bead_sw, np, k, V, W);
      else
        k_interp_q<8><<<fs_blocks(np, 8), 256, 8 * wq, c->stream>>>(ug, Y, c->bins.sorted, c->bead_sw, np, k, V, W);
      FS_LAUNCH_CHECK();
      return FS_OK;
    }
  }
  const size_t wb = interp_warp_bytes<R>(c->p.ngd);
  const int wpb = (c->tune_interp_wpb == 16 && 16 * wb > FS_SMEM_MAX) ? 8 : c->tune_interp_wpb;
  if (wpb == 4)
    k_interp<R, 4><<<fs_blocks(np, 4), 128, 4 * wb, c->stream>>>(ug, Y, c->bins.sorted, c->bead_sw, np, k, V, W);
  else if (wpb == 16)
    k_interp<R, 16><<<fs_blocks(np, 16), 512, 16 * wb, c->stream>>>(ug, Y, c->bins.sorted, c->bead_sw, np, k, V, W);
  else
    k_interp<R, 8><<<fs_blocks(np, 8), 256, 8 * wb, c->stream>>>(ug, Y, c->bins.sorted, c->bead_sw, np, k, V, W);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

template <typename R>
fs_status mobility_t(fs_ctx *c, const double *Y, const double *F, const double *T, double *V, double *W, int np) {
  FcmConsts k = make_consts(c);
  {
    ProfScope ps(c, FS_STAGE_SPREAD);
    FS_TRY(spread_t<R>(c, k, Y, F, T, np));
  }
  FS_TRY(flow_solve_t<R>(c));
  FS_TRY(interp_t<R>(c, k, Y, V, W, np));
  c->last_grid_prec = sizeof(R) == 8 ? FS_PREC_FP64 : FS_PREC_FP32;
  return FS_OK;
}

}  // namespace

fs_status fcm_init(fs_ctx *c) {
  c->nx = c->p.npts_x;
  c->ny = c->p.npts_y;
  c->nz = c->p.npts_z;
  c->nzh = c->nz / 2 + 1;
  c->N = (size_t)c->nx * c->ny * c->nz;
  c->NH = (size_t)c->nx * c->ny * c->nzh;
  for (int d = 0; d < 3; ++d) c->nbin[d] = (d == 0 ? c->nx : d == 1 ? c->ny : c->nz) / FS_TILE;
  c->nbins = c->nbin[0] * c->nbin[1] * c->nbin[2];
  c->last_grid_prec = -1;
  FS_CUDA(cudaMalloc(&c->grid_real, sizeof(double) * 3 * c->N));
  FS_CUDA(cudaMalloc(&c->grid_cplx, sizeof(double2) * 3 * c->NH));
  c->bytes += sizeof(double) * 3 * c->N + sizeof(double2) * 3 * c->NH;
  FS_TRY(fs_sort_alloc(&c->bins, c->nbins, c->max_beads, &c->bytes));
  FS_CUDA(cudaMalloc(&c->bead_sw, sizeof(int) * 3 * (size_t)(c->max_beads > 0 ? c->max_beads : 1)));
  c->bytes += sizeof(int) * 3 * (size_t)c->max_beads;
  {
    const size_t nb = (size_t)(c->max_beads > 0 ? c->max_beads : 1);
    const size_t nw = nb * spread_rec_len(c->p.ngd);
    FS_CUDA(cudaMalloc(&c->spread_wb, sizeof(float4) * nw));
    c->bytes += sizeof(float4) * nw;
  }
  FS_CUDA(cudaFuncSetAttribute(k_spread32<64, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)spread32_smem<64>(FS_NGD_MAX)));
  FS_CUDA(cudaFuncSetAttribute(k_spread32<64, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)spread32_smem<64>(FS_NGD_MAX)));
  FS_CUDA(cudaFuncSetAttribute(k_spread32<64, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)spread32_smem<64>(FS_NGD_MAX)));
  FS_CUDA(cudaFuncSetAttribute(k_spread32<32, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)spread32_smem<32>(FS_NGD_MAX)));
  FS_CUDA(cudaFuncSetAttribute(k_spread32<32, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)spread32_smem<32>(FS_NGD_MAX)));
  FS_CUDA(cudaFuncSetAttribute(k_spread32<32, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)spread32_smem<32>(FS_NGD_MAX)));
  FS_CUDA(cudaFuncSetAttribute(k_spread<double, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(SpreadStage<double, 64>)));
  FS_CUDA(cudaFuncSetAttribute(k_spread<float, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(SpreadStage<float, 64>)));
  FS_CUDA(cudaFuncSetAttribute(k_spread<double, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(SpreadStage<double, 32>)));
  FS_CUDA(cudaFuncSetAttribute(k_spread<float, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(SpreadStage<float, 32>)));
  {
    // the attribute is per kernel, shared by every context: set for the largest
    // ngd (capped at what a CTA may ask for; larger launches take 8 warps per CTA)
    const size_t wd = interp_warp_bytes<double>(FS_NGD_MAX), wf = interp_warp_bytes<float>(FS_NGD_MAX);
    auto cap = [](size_t b) { return (int)(b < (size_t)FS_SMEM_MAX ? b : (size_t)FS_SMEM_MAX); };
    FS_CUDA(cudaFuncSetAttribute(k_interp<double, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap(4 * wd)));
    FS_CUDA(cudaFuncSetAttribute(k_interp<double, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap(8 * wd)));
    FS_CUDA(cudaFuncSetAttribute(k_interp<double, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap(16 * wd)));
    FS_CUDA(cudaFuncSetAttribute(k_interp<float, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap(4 * wf)));
    FS_CUDA(cudaFuncSetAttribute(k_interp<float, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap(8 * wf)));
    FS_CUDA(cudaFuncSetAttribute(k_interp<float, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap(16 * wf)));
    const size_t wq = interp_q_warp_bytes(FS_NGD_MAX);
    FS_CUDA(cudaFuncSetAttribute(k_interp_q<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap(4 * wq)));
    FS_CUDA(cudaFuncSetAttribute(k_interp_q<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap(8 * wq)));
    FS_CUDA(cudaFuncSetAttribute(k_interp_q<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap(16 * wq)));
  }
  c->tune_spread_chunk = 64;
  c->tune_spread_cols = 2;  // 2 x 16 x 8 blocks: fs_autotune's choice at 384^3 and 512^3
  c->tune_interp_wpb = 8;
  c->tune_fft32 = 0;
  return fft32_init(c);
}

void fcm_free(fs_ctx *c) {
  for (int p = 0; p < 2; ++p)
    if (c->plan_ok[p]) {
      cufftDestroy(c->plan_fwd[p]);
      cufftDestroy(c->plan_inv[p]);
      c->plan_ok[p] = false;
    }
  cudaFree(c->grid_real);
  cudaFree(c->grid_cplx);
  c->grid_real = c->grid_cplx = nullptr;
  fft32_free(c);
  fs_sort_free(&c->bins);
  cudaFree(c->bead_sw);
  c->bead_sw = nullptr;
  cudaFree(c->spread_wb);
  c->spread_wb = nullptr;
}

fs_status fcm_set_stream(fs_ctx *c, cudaStream_t st) {
  const int prec = c->precision;
  if (prec == FS_PREC_FP32 && c->fft_tw && c->tune_fft32 == 0) return FS_OK;  // the warp FFT uses no cuFFT plan
  FS_TRY(ensure_plans(c, prec));
  if (cufftSetStream(c->plan_fwd[prec], st) != CUFFT_SUCCESS) return FS_ERR_CUFFT;
  if (cufftSetStream(c->plan_inv[prec], st) != CUFFT_SUCCESS) return FS_ERR_CUFFT;
  return FS_OK;
}

fs_status fcm_mobility(fs_ctx *c, const double *Y, const double *F, const double *T, double *V, double *W, int np) {
  if (c->precision == FS_PREC_FP32) return mobility_t<float>(c, Y, F, T, V, W, np);
  return mobility_t<double>(c, Y, F, T, V, W, np);
}

fs_status fcm_friction(fs_ctx *c, const double *F, const double *T, double *V, double *W, int np) {
  const double PI = FS_PI, a = c->p.a, mu = c->p.mu;
  const double a1 = 1. / (6 * PI * a * mu);
  const double a2 = 1. / (8 * PI * a * a * a * mu);
  if (np > 0) {
    ProfScope ps(c, FS_STAGE_FRICTION);
    k_friction<<<fs_blocks(3 * np, 256), 256, 0, c->stream>>>(F, T, V, W, 3 * np, a1, a2);
    FS_LAUNCH_CHECK();
  }
  return FS_OK;
}

fs_status fcm_interpolate_only(fs_ctx *c, const double *u, const double *Y, int np, double *V, double *W) {
  FcmConsts k = make_consts(c);
  const size_t n = 3 * c->N;
  if (np > 0) {
    k_fcm_bin_keys<<<fs_blocks(np, 256), 256, 0, c->stream>>>(Y, np, k, c->bins.key, c->bead_sw);
    FS_LAUNCH_CHECK();
  }
  FS_TRY(fs_sort_run(&c->bins, np, c->stream));
  if (c->precision == FS_PREC_FP32) {
    k_convert<double, float><<<fs_blocks((long long)n, 256), 256, 0, c->stream>>>(u, (float *)c->grid_real, n);
    FS_LAUNCH_CHECK();
    FS_TRY(interp_t<float>(c, k, Y, V, W, np));
  } else {
    FS_CUDA(cudaMemcpyAsync(c->grid_real, u, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    FS_TRY(interp_t<double>(c, k, Y, V, W, np));
  }
  c->last_grid_prec = -1;
  return FS_OK;
}

fs_status fcm_spread_only(fs_ctx *c, const double *Y, const double *F, const double *T, int np, double *f) {
  FcmConsts k = make_consts(c);
  const size_t n = 3 * c->N;
  if (c->precision == FS_PREC_FP32) {
    FS_TRY(spread_t<float>(c, k, Y, F, T, np));
    k_convert<float, double><<<fs_blocks((long long)n, 256), 256, 0, c->stream>>>((const float *)c->grid_real, f, n);
    FS_LAUNCH_CHECK();
  } else {
    FS_TRY(spread_t<double>(c, k, Y, F, T, np));
    FS_CUDA(cudaMemcpyAsync(f, c->grid_real, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
  }
  c->last_grid_prec = -1;
  return FS_OK;
}

fs_status fcm_flow_solve_only(fs_ctx *c, const double *f, double *u) {
  const size_t n = 3 * c->N;
  if (c->precision == FS_PREC_FP32) {
    // FP32 chain: f rounded to float, solved, widened back
    k_convert<double, float><<<fs_blocks((long long)n, 256), 256, 0, c->stream>>>(f, (float *)c->grid_real, n);
    FS_LAUNCH_CHECK();
    FS_TRY(flow_solve_t<float>(c));
    k_convert<float, double><<<fs_blocks((long long)n, 256), 256, 0, c->stream>>>((const float *)c->grid_real, u, n);
    FS_LAUNCH_CHECK();
    c->last_grid_prec = FS_PREC_FP32;
    return FS_OK;
  }
  FS_CUDA(cudaMemcpyAsync(c->grid_real, f, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
  FS_TRY(flow_solve_t<double>(c));
  FS_CUDA(cudaMemcpyAsync(u, c->grid_real, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
  c->last_grid_prec = FS_PREC_FP64;
  return FS_OK;
}
