// fs_cells.cu -- cell linked list and collision barrier on sm_100a.
//
// LinkedList::link (CollisionBarrierFilament.cpp:370-433) head-inserts beads
// into cells, so each cell's list runs from the largest bead id down. A
// counting sort by (cell, id) produces the same lists: head[c] is the last
// bead of the cell's segment and list[b] the one before it. k_cell_lists
// writes head/list exactly as the reference holds them.
//
// LinkedList::apply_collision_barrier (:24-271) walks cells in order, and for
// each bead i the rest of its own cell and the 13 half-shell neighbour cells,
// adding the pair force to i and subtracting it from j. k_barrier gives each
// bead one thread that collects every interaction it takes part in (as i and
// as j), sorts them by the reference's visiting order
// (cell of i, list position of i, neighbour slot, list position of j) and
// folds them in that order, so each bead's total is bit-identical to the
// reference's sequential accumulation. Pair arithmetic uses explicit
// round-to-nearest intrinsics (no FMA contraction) to match the reference's
// x86-64 doubles.
#include "fs_internal.cuh"

fs_status fs_exclusive_scan(const int *in, int *out, int n, int *block_sums, cudaStream_t st);

namespace {

struct BarrierConsts {
  double L[3];
  int M[3];
  double chiRnm2, den, cap, cap2, fs;
  int nt, initial_friction_steps;
  int mode, np;  // pair filter (FS_BARRIER_*) and bead count
};

// bulkmap neighbour offsets (CollisionBarrierFilament.cpp:326-338)
__constant__ int c_nb_off[13][3] = {{1, 0, 0},  {1, 1, 0},  {0, 1, 0},  {-1, 1, 0}, {1, 0, -1},
                                    {1, 1, -1}, {0, 1, -1}, {-1, 1, -1}, {1, 0, 1}, {1, 1, 1},
                                    {0, 1, 1},  {-1, 1, 1}, {0, 0, 1}};

__device__ __forceinline__ int icell(const int *M, int x, int y, int z) {
  int xx = (x + M[0]) % M[0], yy = (y + M[1]) % M[1], zz = (z + M[2]) % M[2];
  return xx + yy * M[0] + zz * M[0] * M[1];
}

__global__ void k_bulkmap(int Mx, int My, int Mz, int *__restrict__ map) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  int M[3] = {Mx, My, Mz};
  if (c >= Mx * My * Mz) return;
  int x = c % Mx, y = (c / Mx) % My, z = c / (Mx * My);
  for (int nb = 0; nb < 13; ++nb) map[13 * c + nb] = icell(M, x + c_nb_off[nb][0], y + c_nb_off[nb][1], z + c_nb_off[nb][2]);
}

// cell of an unwrapped position (CollisionBarrierFilament.cpp:387-409)
__global__ void k_cell_keys(const double *__restrict__ Xs, int np, BarrierConsts k, int *__restrict__ key) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= np) return;
  const int large_number = 100000;
  int ci[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double x = Xs[3 * b + d];
    const int w = __double2int_rz(__dadd_rn(__ddiv_rn(x, k.L[d]), (double)large_number)) - large_number;
    const double xr = __dsub_rn(x, __dmul_rn(k.L[d], (double)w));
    int cc = __double2int_rz(__dmul_rn(__ddiv_rn(xr, k.L[d]), (double)k.M[d]));
    cc = cc >= k.M[d] ? k.M[d] - 1 : cc;
    cc = cc < 0 ? 0 : cc;
    ci[d] = cc;
  }
  key[b] = ci[0] + ci[1] * k.M[0] + ci[2] * k.M[0] * k.M[1];
}

__global__ void k_cell_lists(const int *__restrict__ start, const int *__restrict__ sorted, int ncell,
                             int *__restrict__ head, int *__restrict__ list, int *__restrict__ rank_desc,
                             int *__restrict__ flags) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int s = start[c], e = start[c + 1];
  head[c] = (e > s) ? sorted[e - 1] : -1;
  if (e - s >= 4096) atomicOr(&flags[FLAG_CAPACITY], 1);
  for (int p = s; p < e; ++p) {
    int b = sorted[p];
    list[b] = (p > s) ? sorted[p - 1] : -1;
    rank_desc[b] = e - 1 - p;
  }
}

// one pair as the reference computes it (CollisionBarrierFilament.cpp:80-149);
// returns 1 inside the barrier range
__device__ __noinline__ int pair_force(const BarrierConsts &k, const double *__restrict__ Yi,
                                       const double *__restrict__ Yj, double *rsq_out, double *f) {
  double d[3];
#pragma unroll
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
#pragma unroll
    for (int a = 0; a < 3; ++a) d[a] = __dmul_rn(__ddiv_rn(d[a], rij), k.cap);
    rijsq = k.cap2;
  }
  double prefac = __dsub_rn(k.chiRnm2, rijsq);
  prefac = __ddiv_rn(prefac, k.den);
  prefac = __dmul_rn(prefac, prefac);
  prefac = __dmul_rn(prefac, prefac);
  prefac = __dmul_rn(prefac, k.fs);
#pragma unroll
  for (int a = 0; a < 3; ++a) f[a] = __dmul_rn(prefac, d[a]);
  return 1;
}

__device__ __forceinline__ unsigned long long ev_key(int cell, int pos_i, int slot, int pos_j) {
  return ((((unsigned long long)cell * 4096ull + (unsigned long long)pos_i) * 16ull + (unsigned long long)slot) *
          4096ull) + (unsigned long long)pos_j;
}

// pairs the barrier skips: neighbours on one filament (CollisionBarrierFilament.cpp:57),
// and per mode swimmer-network pairs (apply_collision_barrier_not_swimmer, :474-477)
// or pairs with one of the last two beads (apply_collision_barrier_not_test_particles, :754)
__device__ __forceinline__ bool excluded(const BarrierConsts &k, const int *fil_id, const int *seg_id, int i, int j) {
  if (k.mode == FS_BARRIER_NOT_SWIMMER && ((fil_id[i] == 0) != (fil_id[j] == 0))) return true;
  if (k.mode == FS_BARRIER_NOT_TEST_PARTICLES && (i >= k.np - 2 || j >= k.np - 2)) return true;
  return (fil_id[j] == fil_id[i] && abs(seg_id[j] - seg_id[i]) == 1) && !(k.nt < k.initial_friction_steps);
}

// mode 0: add barrier forces to F; mode 1: count i-role pairs; mode 2: write pairs
__global__ void __launch_bounds__(128) k_barrier(const double *__restrict__ Y, double *__restrict__ F, int np,
                                                 BarrierConsts k, const int *__restrict__ cell_of,
                                                 const int *__restrict__ start, const int *__restrict__ sorted,
                                                 const int *__restrict__ rank_desc, const int *__restrict__ map,
                                                 const int *__restrict__ fil_id, const int *__restrict__ seg_id,
                                                 unsigned long long *__restrict__ min_bits, int *__restrict__ flags,
                                                 int mode, int *__restrict__ pair_count,
                                                 const int *__restrict__ pair_off, int *__restrict__ pairs,
                                                 int max_pairs) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= np) return;
  const int cb = cell_of[b];
  const int pb = rank_desc[b];
  const int e0 = start[cb + 1];
  const int p_asc = e0 - 1 - pb;
  const double Yb[3] = {Y[3 * b], Y[3 * b + 1], Y[3 * b + 2]};
  unsigned long long keys[FS_MAX_EVENTS];
  double fx[FS_MAX_EVENTS], fy[FS_MAX_EVENTS], fz[FS_MAX_EVENTS];
  int nev = 0, overflow = 0;
  double local_min = 100000.0;
  int npairs_here = 0;
  int out_base = (mode == 2) ? pair_off[b] : 0;
  double f[3], rsq;
  // cell ranges of both halves loaded up front (independent loads in flight together)
  int rs_i[14], re_i[14];
#pragma unroll
  for (int slot = 0; slot < 14; ++slot) {
    const int cj = slot == 0 ? cb : map[13 * cb + slot - 1];
    rs_i[slot] = start[cj];
    re_i[slot] = start[cj + 1];
  }
  // ---- b as i: the rest of its own cell, then the 13 neighbour cells ----
#pragma unroll 1
  for (int slot = 0; slot < 14; ++slot) {
    const int qs = rs_i[slot];
    const int qe = slot == 0 ? p_asc : re_i[slot];  // own cell: ascending positions below b's
    const int ej = re_i[slot];
    for (int q = qe - 1; q >= qs; --q) {
      const int j = sorted[q];
      if (excluded(k, fil_id, seg_id, b, j)) continue;
      const double Yj[3] = {Y[3 * j], Y[3 * j + 1], Y[3 * j + 2]};
      if (pair_force(k, Yb, Yj, &rsq, f)) {
        if (mode == 0) {
          if (nev < FS_MAX_EVENTS) {
            keys[nev] = ev_key(cb, pb, slot, ej - 1 - q);
            fx[nev] = f[0];
            fy[nev] = f[1];
            fz[nev] = f[2];
            nev++;
          } else {
            overflow = 1;
          }
        } else if (mode == 2) {
          int o = out_base + npairs_here;
          if (o < max_pairs) {
            pairs[2 * o] = b;
            pairs[2 * o + 1] = j;
          }
        }
        npairs_here++;
      }
      if (rsq < local_min) local_min = rsq;
    }
  }
  if (mode == 1) {
    pair_count[b] = npairs_here;
    return;
  }
  if (mode == 2) return;
  // ---- b as j: beads before it in its own cell, and the cells whose slot maps to b's cell ----
  const int Mx = k.M[0], My = k.M[1];
  const int cx = cb % Mx, cy = (cb / Mx) % My, cz = cb / (Mx * My);
  int rs_j[14], re_j[14], ci_j[14];
#pragma unroll
  for (int slot = 0; slot < 14; ++slot) {
    const int ci = slot == 0 ? cb
                             : icell(k.M, cx - c_nb_off[slot - 1][0], cy - c_nb_off[slot - 1][1],
                                     cz - c_nb_off[slot - 1][2]);
    ci_j[slot] = ci;
    rs_j[slot] = start[ci];
    re_j[slot] = start[ci + 1];
  }
#pragma unroll 1
  for (int slot = 0; slot < 14; ++slot) {
    int qs, qe;
    if (slot == 0) {
      qs = p_asc + 1;
      qe = e0;
    } else {
      qs = rs_j[slot];
      qe = re_j[slot];
    }
    const int ci = ci_j[slot], ei = re_j[slot];
    for (int q = qs; q < qe; ++q) {
      const int i = sorted[q];
      if (excluded(k, fil_id, seg_id, i, b)) continue;
      const double Yi[3] = {Y[3 * i], Y[3 * i + 1], Y[3 * i + 2]};
      if (pair_force(k, Yi, Yb, &rsq, f)) {
        if (nev < FS_MAX_EVENTS) {
          keys[nev] = ev_key(ci, ei - 1 - q, slot, pb);
          fx[nev] = -f[0];  // marks subtraction; folded as acc - f
          fy[nev] = -f[1];
          fz[nev] = -f[2];
          nev++;
        } else {
          overflow = 1;
        }
      }
    }
  }
  if (overflow) atomicOr(&flags[FLAG_CAPACITY], 1);
  // insertion sort by visiting order
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
  // fold: adding -f equals subtracting f exactly
  double ax = 0.0, ay = 0.0, az = 0.0;
  for (int a = 0; a < nev; ++a) {
    ax = __dadd_rn(ax, fx[a]);
    ay = __dadd_rn(ay, fy[a]);
    az = __dadd_rn(az, fz[a]);
  }
  F[3 * b] = __dadd_rn(F[3 * b], ax);
  F[3 * b + 1] = __dadd_rn(F[3 * b + 1], ay);
  F[3 * b + 2] = __dadd_rn(F[3 * b + 2], az);
  // the minimum squared distance: one atomic per full warp after a shuffle
  // reduction (per bead, all beads would contend for one address); the last,
  // partial warp of the grid keeps per-thread atomics
  unsigned long long mb = fs_dbits(local_min);
  if (__activemask() == 0xffffffffu) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long other = __shfl_xor_sync(0xffffffffu, mb, o);
      mb = other < mb ? other : mb;
    }
    if ((threadIdx.x & 31) == 0) atomicMin(min_bits, mb);
  } else {
    atomicMin(min_bits, mb);
  }
}

__global__ void k_pair_pos(const int *__restrict__ cell_of, const int *__restrict__ start,
                           const int *__restrict__ rank_desc, const int *__restrict__ count, int np,
                           int *__restrict__ by_pos) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < np) by_pos[start[cell_of[b]] + rank_desc[b]] = count[b];
}

__global__ void k_pair_off(const int *__restrict__ cell_of, const int *__restrict__ start,
                           const int *__restrict__ rank_desc, const int *__restrict__ off_by_pos, int np,
                           int *__restrict__ off) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < np) off[b] = off_by_pos[start[cell_of[b]] + rank_desc[b]];
}

// local minimum starts at 100000 as in apply_collision_barrier (CollisionBarrierFilament.cpp:41)
__global__ void k_set_min_init(unsigned long long *bits) { *bits = fs_dbits(100000.0); }

BarrierConsts make_bconsts(const fs_ctx *c, int nt) {
  BarrierConsts k;
  for (int d = 0; d < 3; ++d) {
    k.L[d] = c->L[d];
    k.M[d] = c->M[d];
  }
  const double Rnm = 2 * c->p.a;
  const double Rnm2 = Rnm * Rnm;
  k.chiRnm2 = 1.21 * Rnm2;
  k.den = k.chiRnm2 - Rnm2;
  k.cap = c->p.barrier_distance_cap;
  k.cap2 = k.cap * k.cap;
  k.fs = c->p.barrier_fs_over_2a;
  k.nt = nt;
  k.initial_friction_steps = c->p.initial_friction_steps;
  k.mode = FS_BARRIER_ALL;
  k.np = 0;
  return k;
}

}  // namespace

fs_status cells_init(fs_ctx *c) {
  const double Rref = c->p.cell_width;
  for (int d = 0; d < 3; ++d) {
    c->M[d] = (int)(c->L[d] / Rref);
    if (c->M[d] < 1) return FS_ERR_INVALID_ARG;
  }
  c->ncell = c->M[0] * c->M[1] * c->M[2];
  FS_TRY(fs_sort_alloc(&c->cells, c->ncell, c->max_beads, &c->bytes));
  const int nb = c->max_beads > 0 ? c->max_beads : 1;
  FS_CUDA(cudaMalloc(&c->head, sizeof(int) * c->ncell));
  FS_CUDA(cudaMalloc(&c->list, sizeof(int) * nb));
  FS_CUDA(cudaMalloc(&c->map, sizeof(int) * 13 * (size_t)c->ncell));
  FS_CUDA(cudaMalloc(&c->cell_rank, sizeof(int) * nb));
  FS_CUDA(cudaMalloc(&c->pair_count, sizeof(int) * (size_t)(nb + 1)));
  FS_CUDA(cudaMalloc(&c->pair_off, sizeof(int) * (size_t)(nb + 1)));
  FS_CUDA(cudaMalloc(&c->min_dist2_bits, sizeof(unsigned long long)));
  FS_CUDA(cudaMalloc(&c->pair_scan_tmp, sizeof(int) * (size_t)((nb + 1) / 4096 + 2)));
  c->bytes += sizeof(int) * ((size_t)14 * c->ncell + 4 * (size_t)nb);
  k_bulkmap<<<fs_blocks(c->ncell, 256), 256, 0, c->stream>>>(c->M[0], c->M[1], c->M[2], c->map);
  FS_LAUNCH_CHECK();
  c->cells_np = -1;
  return FS_OK;
}

void cells_free(fs_ctx *c) {
  fs_sort_free(&c->cells);
  cudaFree(c->head);
  cudaFree(c->list);
  cudaFree(c->map);
  cudaFree(c->cell_rank);
  cudaFree(c->pair_count);
  cudaFree(c->pair_off);
  cudaFree(c->min_dist2_bits);
  cudaFree(c->pair_scan_tmp);
}

fs_status cells_link(fs_ctx *c, const double *Xs, int np) {
  ProfScope ps(c, FS_STAGE_LINK);
  BarrierConsts k = make_bconsts(c, 0);
  if (np > 0) {
    k_cell_keys<<<fs_blocks(np, 256), 256, 0, c->stream>>>(Xs, np, k, c->cells.key);
    FS_LAUNCH_CHECK();
  }
  FS_TRY(fs_sort_run(&c->cells, np, c->stream));
  k_cell_lists<<<fs_blocks(c->ncell, 256), 256, 0, c->stream>>>(c->cells.start, c->cells.sorted, c->ncell, c->head,
                                                                c->list, c->cell_rank, c->flags);
  FS_LAUNCH_CHECK();
  c->cells_np = np;
  return FS_OK;
}

fs_status cells_barrier(fs_ctx *c, const double *Y, double *F, int np, int nt, const int *fil_id,
                        const int *seg_id, int *pairs_d, int max_pairs, int *npairs_h, int mode) {
  if (c->cells_np != np) return FS_ERR_STATE;
  ProfScope ps(c, FS_STAGE_BARRIER);
  BarrierConsts k = make_bconsts(c, nt);
  k.mode = mode;
  k.np = np;
  k_set_min_init<<<1, 1, 0, c->stream>>>(c->min_dist2_bits);
  FS_LAUNCH_CHECK();
  c->min_dist2_valid = true;
  if (np == 0) return FS_OK;
  const int T = 128;
  if (npairs_h) {
    k_barrier<<<fs_blocks(np, T), T, 0, c->stream>>>(Y, F, np, k, c->cells.key, c->cells.start, c->cells.sorted,
                                                     c->cell_rank, c->map, fil_id, seg_id, c->min_dist2_bits,
                                                     c->flags, 1, c->pair_count, nullptr, nullptr, 0);
    FS_LAUNCH_CHECK();
    // offsets in the reference's visiting order of the i beads
    k_pair_pos<<<fs_blocks(np, 256), 256, 0, c->stream>>>(c->cells.key, c->cells.start, c->cell_rank, c->pair_count,
                                                           np, c->pair_off);
    FS_LAUNCH_CHECK();
    FS_CUDA(cudaMemsetAsync(c->pair_off + np, 0, sizeof(int), c->stream));
    FS_TRY(fs_exclusive_scan(c->pair_off, c->pair_count, np + 1, c->pair_scan_tmp, c->stream));
    FS_CUDA(cudaMemcpyAsync(npairs_h, c->pair_count + np, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    k_pair_off<<<fs_blocks(np, 256), 256, 0, c->stream>>>(c->cells.key, c->cells.start, c->cell_rank, c->pair_count,
                                                           np, c->pair_off);
    FS_LAUNCH_CHECK();
    k_barrier<<<fs_blocks(np, T), T, 0, c->stream>>>(Y, F, np, k, c->cells.key, c->cells.start, c->cells.sorted,
                                                     c->cell_rank, c->map, fil_id, seg_id, c->min_dist2_bits,
                                                     c->flags, 2, nullptr, c->pair_off, pairs_d, max_pairs);
    FS_LAUNCH_CHECK();
    FS_CUDA(cudaStreamSynchronize(c->stream));
    return FS_OK;
  }
  k_barrier<<<fs_blocks(np, T), T, 0, c->stream>>>(Y, F, np, k, c->cells.key, c->cells.start, c->cells.sorted,
                                                   c->cell_rank, c->map, fil_id, seg_id, c->min_dist2_bits, c->flags,
                                                   0, nullptr, nullptr, nullptr, 0);
  FS_LAUNCH_CHECK();
  return FS_OK;
}
