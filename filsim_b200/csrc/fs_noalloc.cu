// fs_noalloc.cu -- the collision barrier for callers that cannot allocate
// device memory.
//
// fs_collision_barrier_noalloc bins the beads into cells and adds the barrier
// forces in one call, like fs_cells_link followed by fs_collision_barrier, but
// without a context: it calls no cudaMalloc, cudaFree or allocating library
// routine. Some callers cannot allocate: a host program that hands this
// library a fixed device-memory budget through its own pool, or a time-step
// loop that must not pay cudaMalloc's device-wide synchronisation between
// kernels. Its working memory is the file-scope array g_noalloc_scratch below,
// which every GPU that loads the library holds until the process exits.
//
// Every call uses the same array and leaves its contents behind; the call
// clears what must start at zero. Two calls that overlap on the GPU (on
// different streams, or from different host threads) race on the array.
#include <cmath>
#include <mutex>
#include "fs_internal.cuh"

#define FS_NOALLOC_SCRATCH_BYTES (4u << 20)  // 4 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[FS_NOALLOC_SCRATCH_BYTES];

namespace {

// scratch layout (ints): cell key, sorted beads and list rank per bead; count,
// start and fill cursor per cell; the minimum squared distance
constexpr int kMaxBeads = FS_NOALLOC_MAX_BEADS;
constexpr int kMaxCells = FS_NOALLOC_MAX_CELLS;
constexpr size_t kOffKey = 0;
constexpr size_t kOffSorted = kOffKey + sizeof(int) * kMaxBeads;
constexpr size_t kOffRank = kOffSorted + sizeof(int) * kMaxBeads;
constexpr size_t kOffCount = kOffRank + sizeof(int) * kMaxBeads;
constexpr size_t kOffStart = kOffCount + sizeof(int) * (kMaxCells + 1);
constexpr size_t kOffCursor = kOffStart + sizeof(int) * (kMaxCells + 1);
constexpr size_t kOffMin = (kOffCursor + sizeof(int) * (kMaxCells + 1) + 255) / 256 * 256;
static_assert(kOffMin + 8 <= FS_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the static array");

struct NaConsts {
  double L[3];
  int M[3];
  double chiRnm2, den, cap, cap2, fs;
  int nt, initial_friction_steps, ncell;
};

__device__ __forceinline__ int na_icell(const int *M, int x, int y, int z) {
  int xx = (x + M[0]) % M[0], yy = (y + M[1]) % M[1], zz = (z + M[2]) % M[2];
  return xx + yy * M[0] + zz * M[0] * M[1];
}

// neighbour slots of LinkedList::bulkmap (CollisionBarrierFilament.cpp:326-338)
__constant__ int c_na_off[13][3] = {{1, 0, 0},  {1, 1, 0},  {0, 1, 0},  {-1, 1, 0}, {1, 0, -1},
                                    {1, 1, -1}, {0, 1, -1}, {-1, 1, -1}, {1, 0, 1}, {1, 1, 1},
                                    {0, 1, 1},  {-1, 1, 1}, {0, 0, 1}};

__global__ void k_na_keys(const double *__restrict__ Xs, int np, NaConsts k, int *__restrict__ key,
                          int *__restrict__ count) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= np) return;
  const int large_number = 100000;
  int ci[3];
  for (int d = 0; d < 3; ++d) {
    const double x = Xs[3 * b + d];
    const int w = __double2int_rz(__dadd_rn(__ddiv_rn(x, k.L[d]), (double)large_number)) - large_number;
    const double xr = __dsub_rn(x, __dmul_rn(k.L[d], (double)w));
    int cc = __double2int_rz(__dmul_rn(__ddiv_rn(xr, k.L[d]), (double)k.M[d]));
    cc = cc >= k.M[d] ? k.M[d] - 1 : cc;
    ci[d] = cc < 0 ? 0 : cc;
  }
  const int c = ci[0] + ci[1] * k.M[0] + ci[2] * k.M[0] * k.M[1];
  key[b] = c;
  atomicAdd(&count[c], 1);
}

// exclusive scan of count[0..n] into start (one CTA)
__global__ void __launch_bounds__(1024) k_na_scan(const int *__restrict__ count, int n, int *__restrict__ start) {
  __shared__ int warp_tot[32];
  __shared__ int carry;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  if (t == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += 1024) {
    const int idx = base + t;
    const int v = idx < n ? count[idx] : 0;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
      int x = warp_tot[lane];
      int ix = x;
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, ix, o);
        if (lane >= o) ix += y;
      }
      warp_tot[lane] = ix - x;
    }
    __syncthreads();
    if (idx < n) start[idx] = carry + warp_tot[w] + incl - v;
    __syncthreads();
    if (t == 1023) carry += warp_tot[31] + incl;
    __syncthreads();
  }
}

__global__ void k_na_scatter(const int *__restrict__ key, int np, const int *__restrict__ start,
                             int *__restrict__ cursor, int *__restrict__ sorted) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < np) {
    const int c = key[b];
    sorted[start[c] + atomicAdd(&cursor[c], 1)] = b;
  }
}

// per cell: ascending bead ids (shell sort) and each bead's list rank. The
// visiting-order key of k_na_barrier holds a list position in 12 bits, so a
// cell of 4096 beads or more sets bit 1 of the flag (the barrier then adds
// nothing and the call returns FS_ERR_CAPACITY).
__global__ void k_na_cells(const int *__restrict__ start, int ncell, int *__restrict__ sorted,
                           int *__restrict__ rank_desc, int *__restrict__ overflow_flag) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int s0 = start[c], n = start[c + 1] - s0;
  if (n >= 4096) atomicOr(overflow_flag, 2);
  int *a = sorted + s0;
  int gap = 1;
  while (gap < n / 3) gap = 3 * gap + 1;
  for (; gap > 0; gap /= 3)
    for (int i = gap; i < n; ++i) {
      int v = a[i], j = i;
      while (j >= gap && a[j - gap] > v) {
        a[j] = a[j - gap];
        j -= gap;
      }
      a[j] = v;
    }
  for (int p = 0; p < n; ++p) rank_desc[a[p]] = n - 1 - p;
}

// one pair as CollisionBarrierFilament.cpp:80-149 computes it
__device__ __noinline__ int na_pair(const NaConsts &k, const double *__restrict__ Yi, const double *__restrict__ Yj,
                                    double *rsq_out, double *f) {
  double d[3];
  for (int a = 0; a < 3; ++a) {
    double x = __dsub_rn(Yi[a], Yj[a]);
    double s = floor(__dadd_rn(__ddiv_rn(x, k.L[a]), 0.5));
    d[a] = __dsub_rn(x, __dmul_rn(k.L[a], s));
  }
  double rijsq = __dadd_rn(__dadd_rn(__dmul_rn(d[0], d[0]), __dmul_rn(d[1], d[1])), __dmul_rn(d[2], d[2]));
  *rsq_out = rijsq;
  if (!(rijsq < k.chiRnm2)) return 0;
  if (rijsq < k.cap2) {
    double rij = __dsqrt_rn(rijsq);
    for (int a = 0; a < 3; ++a) d[a] = __dmul_rn(__ddiv_rn(d[a], rij), k.cap);
    rijsq = k.cap2;
  }
  double prefac = __ddiv_rn(__dsub_rn(k.chiRnm2, rijsq), k.den);
  prefac = __dmul_rn(prefac, prefac);
  prefac = __dmul_rn(prefac, prefac);
  prefac = __dmul_rn(prefac, k.fs);
  for (int a = 0; a < 3; ++a) f[a] = __dmul_rn(prefac, d[a]);
  return 1;
}

// each bead folds its interactions in the reference's visiting order
// (cell of i, list position of i, neighbour slot, list position of j)
__global__ void __launch_bounds__(128) k_na_barrier(const double *__restrict__ Y, double *__restrict__ F, int np,
                                                    NaConsts k, const int *__restrict__ cell_of,
                                                    const int *__restrict__ start, const int *__restrict__ sorted,
                                                    const int *__restrict__ rank_desc, const int *__restrict__ fil_id,
                                                    const int *__restrict__ seg_id,
                                                    unsigned long long *__restrict__ min_bits,
                                                    int *__restrict__ overflow_flag) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= np || (*overflow_flag & 2)) return;  // a cell too full for the key: F is left as it was
  const int cb = cell_of[b], pb = rank_desc[b];
  const int s0 = start[cb], e0 = start[cb + 1], p_asc = e0 - 1 - pb;
  const int Mx = k.M[0], My = k.M[1];
  const int cx = cb % Mx, cy = (cb / Mx) % My, cz = cb / (Mx * My);
  const double Yb[3] = {Y[3 * b], Y[3 * b + 1], Y[3 * b + 2]};
  const bool all_pairs = k.nt < k.initial_friction_steps;
  unsigned long long keys[FS_MAX_EVENTS];
  double fx[FS_MAX_EVENTS], fy[FS_MAX_EVENTS], fz[FS_MAX_EVENTS];
  int nev = 0, overflow = 0;
  double local_min = 100000.0, f[3], rsq;
  for (int role = 0; role < 2; ++role)
    for (int slot = 0; slot < 14; ++slot) {
      int cell, qs, qe;
      if (slot == 0) {
        cell = cb;
        qs = role == 0 ? s0 : p_asc + 1;
        qe = role == 0 ? p_asc : e0;
      } else {
        const int sg = role == 0 ? 1 : -1;
        cell = na_icell(k.M, cx + sg * c_na_off[slot - 1][0], cy + sg * c_na_off[slot - 1][1],
                        cz + sg * c_na_off[slot - 1][2]);
        qs = start[cell];
        qe = start[cell + 1];
      }
      const int ec = start[cell + 1];
      for (int q = qs; q < qe; ++q) {
        const int o = sorted[q];
        const int i = role == 0 ? b : o, j = role == 0 ? o : b;
        if (!all_pairs && fil_id[j] == fil_id[i] && abs(seg_id[j] - seg_id[i]) == 1) continue;
        const double Yo[3] = {Y[3 * o], Y[3 * o + 1], Y[3 * o + 2]};
        const int hit = role == 0 ? na_pair(k, Yb, Yo, &rsq, f) : na_pair(k, Yo, Yb, &rsq, f);
        if (role == 0 && rsq < local_min) local_min = rsq;
        if (!hit) continue;
        if (nev == FS_MAX_EVENTS) {
          overflow = 1;
          continue;
        }
        const int pos_o = ec - 1 - q;
        const unsigned long long c_i = role == 0 ? cb : cell;
        const unsigned long long p_i = role == 0 ? pb : pos_o, p_j = role == 0 ? pos_o : pb;
        keys[nev] = ((c_i * 4096ull + p_i) * 16ull + (unsigned long long)slot) * 4096ull + p_j;
        const double sgn = role == 0 ? 1.0 : -1.0;
        fx[nev] = sgn * f[0];
        fy[nev] = sgn * f[1];
        fz[nev] = sgn * f[2];
        ++nev;
      }
    }
  if (overflow) atomicOr(overflow_flag, 1);
  for (int a = 1; a < nev; ++a) {
    unsigned long long kk = keys[a];
    double x = fx[a], y = fy[a], z = fz[a];
    int j = a - 1;
    while (j >= 0 && keys[j] > kk) {
      keys[j + 1] = keys[j];
      fx[j + 1] = fx[j];
      fy[j + 1] = fy[j];
      fz[j + 1] = fz[j];
      --j;
    }
    keys[j + 1] = kk;
    fx[j + 1] = x;
    fy[j + 1] = y;
    fz[j + 1] = z;
  }
  double ax = 0.0, ay = 0.0, az = 0.0;
  for (int a = 0; a < nev; ++a) {
    ax = __dadd_rn(ax, fx[a]);
    ay = __dadd_rn(ay, fy[a]);
    az = __dadd_rn(az, fz[a]);
  }
  F[3 * b] = __dadd_rn(F[3 * b], ax);
  F[3 * b + 1] = __dadd_rn(F[3 * b + 1], ay);
  F[3 * b + 2] = __dadd_rn(F[3 * b + 2], az);
  atomicMin(min_bits, fs_dbits(local_min));
}

__global__ void k_na_init(unsigned long long *min_bits, int *overflow) {
  *min_bits = fs_dbits(100000.0);
  *overflow = 0;
}

// device address of the scratch array, looked up once per device
std::mutex g_na_mutex;
unsigned char *g_na_ptr[64];

fs_status na_setup(int *dev_out, unsigned char **ptr_out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return FS_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_ptr[dev]) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return FS_ERR_NO_DEVICE;
    if (prop.major != 10) return FS_ERR_NO_DEVICE;
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      fprintf(stderr, "filsim_gpu: cudaGetSymbolAddress(g_noalloc_scratch) failed: %s\n", cudaGetErrorString(e));
      return FS_ERR_CUDA;
    }
    g_na_ptr[dev] = (unsigned char *)p;
  }
  *dev_out = dev;
  *ptr_out = g_na_ptr[dev];
  return FS_OK;
}

}  // namespace

extern "C" fs_status fs_collision_barrier_noalloc(const fs_params *p, const double *Xs, const double *Y,
                                                  double *F_inout, int np, int nt, const int *fil_id,
                                                  const int *seg_id, void *stream, double *min_dist2_h) {
  if (!p || np < 0 || (np > 0 && (!Xs || !Y || !F_inout || !fil_id || !seg_id))) return FS_ERR_INVALID_ARG;
  if (np > kMaxBeads) {
    fprintf(stderr, "filsim_gpu: fs_collision_barrier_noalloc: %d beads exceed the limit of %d\n", np, kMaxBeads);
    return FS_ERR_INVALID_ARG;
  }
  NaConsts k;
  const double Lb[3] = {p->npts_x * p->dx, p->npts_y * p->dx, p->npts_z * p->dx};
  for (int d = 0; d < 3; ++d) {
    // the cell count per axis is checked as a double before the conversion to int
    const double m = Lb[d] / p->cell_width;
    if (!std::isfinite(p->cell_width) || !(p->cell_width > 0) || !std::isfinite(Lb[d]) || !(Lb[d] > 0) ||
        !(m >= 1.0) || m > (double)kMaxCells) {
      fprintf(stderr, "filsim_gpu: fs_collision_barrier_noalloc: box %g / cell width %g gives no valid cell count\n",
              Lb[d], p->cell_width);
      return FS_ERR_INVALID_ARG;
    }
    k.L[d] = Lb[d];
    k.M[d] = (int)m;  // LinkedList::initialise (CollisionBarrierFilament.cpp:277-281)
  }
  const long long ncell = (long long)k.M[0] * k.M[1] * k.M[2];
  if (ncell > kMaxCells) {
    fprintf(stderr, "filsim_gpu: fs_collision_barrier_noalloc: %lld cells exceed the limit of %d\n", ncell, kMaxCells);
    return FS_ERR_INVALID_ARG;
  }
  k.ncell = (int)ncell;
  const double Rnm = 2 * p->a, Rnm2 = Rnm * Rnm;
  k.chiRnm2 = 1.21 * Rnm2;
  k.den = k.chiRnm2 - Rnm2;
  k.cap = p->barrier_distance_cap;
  k.cap2 = k.cap * k.cap;
  k.fs = p->barrier_fs_over_2a;
  k.nt = nt;
  k.initial_friction_steps = p->initial_friction_steps;
  int dev;
  unsigned char *base;
  FS_TRY(na_setup(&dev, &base));
  cudaStream_t st = (cudaStream_t)stream;
  int *key = (int *)(base + kOffKey), *sorted = (int *)(base + kOffSorted), *rank = (int *)(base + kOffRank);
  int *count = (int *)(base + kOffCount), *start = (int *)(base + kOffStart), *cursor = (int *)(base + kOffCursor);
  unsigned long long *min_bits = (unsigned long long *)(base + kOffMin);
  int *overflow = (int *)(base + kOffMin + 8);  // the int after the minimum
  static_assert(kOffMin + 16 <= FS_NOALLOC_SCRATCH_BYTES, "flag slot");
  FS_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (ncell + 1), st));
  FS_CUDA(cudaMemsetAsync(cursor, 0, sizeof(int) * (ncell + 1), st));
  k_na_init<<<1, 1, 0, st>>>(min_bits, overflow);
  FS_LAUNCH_CHECK();
  if (np > 0) {
    k_na_keys<<<fs_blocks(np, 256), 256, 0, st>>>(Xs, np, k, key, count);
    FS_LAUNCH_CHECK();
  }
  k_na_scan<<<1, 1024, 0, st>>>(count, k.ncell + 1, start);
  FS_LAUNCH_CHECK();
  if (np > 0) {
    k_na_scatter<<<fs_blocks(np, 256), 256, 0, st>>>(key, np, start, cursor, sorted);
    FS_LAUNCH_CHECK();
    k_na_cells<<<fs_blocks(k.ncell, 256), 256, 0, st>>>(start, k.ncell, sorted, rank, overflow);
    FS_LAUNCH_CHECK();
    k_na_barrier<<<fs_blocks(np, 128), 128, 0, st>>>(Y, F_inout, np, k, key, start, sorted, rank, fil_id, seg_id,
                                                      min_bits, overflow);
    FS_LAUNCH_CHECK();
  }
  int ovf = 0;
  FS_CUDA(cudaMemcpyAsync(&ovf, overflow, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (min_dist2_h) {
    unsigned long long bits = 0;
    FS_CUDA(cudaMemcpyAsync(&bits, min_bits, sizeof bits, cudaMemcpyDeviceToHost, st));
    FS_CUDA(cudaStreamSynchronize(st));
    memcpy(min_dist2_h, &bits, sizeof bits);
  } else {
    FS_CUDA(cudaStreamSynchronize(st));
  }
  return ovf ? FS_ERR_CAPACITY : FS_OK;
}
