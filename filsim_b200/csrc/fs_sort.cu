// fs_sort.cu -- deterministic counting sort of items by integer key.
//
// count (atomics) -> exclusive scan -> scatter -> per-key sort by item id.
// The scatter's slot order depends on atomic timing; the final per-key sort
// by id makes the output a pure function of the keys: items ascend by
// (key, id). This is the order the collision linked list of
// LinkedList::link (CollisionBarrierFilament.cpp:370-433) encodes in reverse.
#include "fs_internal.cuh"

#define SCAN_THREADS 1024
#define SCAN_ITEMS 4
#define SCAN_SPAN (SCAN_THREADS * SCAN_ITEMS)

__global__ void k_sort_count(const int *__restrict__ key, int n, int *__restrict__ count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(&count[key[i]], 1);
}

// exclusive scan of in[0..n) into out, block totals into bsum
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_block(const int *in, int *out, int n, int *bsum) {
  __shared__ int warp_tot[32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const long long base = (long long)blockIdx.x * SCAN_SPAN + (long long)t * SCAN_ITEMS;
  int v[SCAN_ITEMS];
  int s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    long long idx = base + i;
    v[i] = idx < n ? in[idx] : 0;
    s += v[i];
  }
  int incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[w] = incl;
  __syncthreads();
  if (w == 0) {
    int x = lane < (SCAN_THREADS / 32) ? warp_tot[lane] : 0;
    int ix = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, ix, o);
      if (lane >= o) ix += y;
    }
    warp_tot[lane] = ix - x;
  }
  __syncthreads();
  int run = incl - s + warp_tot[w];
  if (t == SCAN_THREADS - 1 && bsum) bsum[blockIdx.x] = run + s;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    long long idx = base + i;
    if (idx < n) out[idx] = run;
    run += v[i];
  }
}

__global__ void k_scan_add(int *__restrict__ out, int n, const int *__restrict__ bsum) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < n) out[idx] += bsum[idx / SCAN_SPAN];
}

__global__ void k_sort_scatter(const int *__restrict__ key, int n, const int *__restrict__ start,
                               int *__restrict__ cursor, int *__restrict__ sorted) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    int k = key[i];
    int slot = atomicAdd(&cursor[k], 1);
    sorted[start[k] + slot] = i;
  }
}

// per-key shell sort by item id (segments are small for physical inputs;
// shell sort keeps large ones bounded)
__global__ void k_sort_segments(const int *__restrict__ start, int nkeys, int *__restrict__ sorted) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nkeys) return;
  int s0 = start[k], n = start[k + 1] - s0;
  if (n < 2) return;
  int *a = sorted + s0;
  int gap = 1;
  while (gap < n / 3) gap = 3 * gap + 1;
  for (; gap > 0; gap /= 3) {
    for (int i = gap; i < n; ++i) {
      int v = a[i];
      int j = i;
      while (j >= gap && a[j - gap] > v) {
        a[j] = a[j - gap];
        j -= gap;
      }
      a[j] = v;
    }
  }
}

fs_status fs_sort_alloc(fs_sort *s, int nkeys, int max_items, size_t *bytes) {
  s->nkeys = nkeys;
  int nblk = (nkeys + 1 + SCAN_SPAN - 1) / SCAN_SPAN;
  if (nblk > SCAN_SPAN) return FS_ERR_INVALID_ARG;
  FS_CUDA(cudaMalloc(&s->key, sizeof(int) * (size_t)(max_items > 0 ? max_items : 1)));
  FS_CUDA(cudaMalloc(&s->count, sizeof(int) * (size_t)(nkeys + 1)));
  FS_CUDA(cudaMalloc(&s->start, sizeof(int) * (size_t)(nkeys + 1)));
  FS_CUDA(cudaMalloc(&s->cursor, sizeof(int) * (size_t)(nkeys + 1)));
  FS_CUDA(cudaMalloc(&s->sorted, sizeof(int) * (size_t)(max_items > 0 ? max_items : 1)));
  FS_CUDA(cudaMalloc(&s->block_sums, sizeof(int) * (size_t)(nblk + 1)));
  *bytes += sizeof(int) * ((size_t)2 * (max_items > 0 ? max_items : 1) + 3 * (size_t)(nkeys + 1) + nblk + 1);
  return FS_OK;
}

void fs_sort_free(fs_sort *s) {
  cudaFree(s->key);
  cudaFree(s->count);
  cudaFree(s->start);
  cudaFree(s->cursor);
  cudaFree(s->sorted);
  cudaFree(s->block_sums);
  s->key = s->count = s->start = s->cursor = s->sorted = s->block_sums = nullptr;
}

fs_status fs_sort_run(fs_sort *s, int n, cudaStream_t st) {
  const int nk1 = s->nkeys + 1;
  FS_CUDA(cudaMemsetAsync(s->count, 0, sizeof(int) * nk1, st));
  FS_CUDA(cudaMemsetAsync(s->cursor, 0, sizeof(int) * nk1, st));
  if (n > 0) {
    k_sort_count<<<fs_blocks(n, 256), 256, 0, st>>>(s->key, n, s->count);
    FS_LAUNCH_CHECK();
  }
  int nblk = (nk1 + SCAN_SPAN - 1) / SCAN_SPAN;
  k_scan_block<<<nblk, SCAN_THREADS, 0, st>>>(s->count, s->start, nk1, s->block_sums);
  FS_LAUNCH_CHECK();
  if (nblk > 1) {
    k_scan_block<<<1, SCAN_THREADS, 0, st>>>(s->block_sums, s->block_sums, nblk, nullptr);
    FS_LAUNCH_CHECK();
    k_scan_add<<<fs_blocks(nk1, 256), 256, 0, st>>>(s->start, nk1, s->block_sums);
    FS_LAUNCH_CHECK();
  }
  if (n > 0) {
    k_sort_scatter<<<fs_blocks(n, 256), 256, 0, st>>>(s->key, n, s->start, s->cursor, s->sorted);
    FS_LAUNCH_CHECK();
    k_sort_segments<<<fs_blocks(s->nkeys, 256), 256, 0, st>>>(s->start, s->nkeys, s->sorted);
    FS_LAUNCH_CHECK();
  }
  return FS_OK;
}

// exclusive scan of n ints (n <= SCAN_SPAN^2); block_sums needs n/SCAN_SPAN+1 ints
fs_status fs_exclusive_scan(const int *in, int *out, int n, int *block_sums, cudaStream_t st) {
  if (n <= 0) return FS_OK;
  int nblk = (n + SCAN_SPAN - 1) / SCAN_SPAN;
  if (nblk > SCAN_SPAN) return FS_ERR_INVALID_ARG;
  k_scan_block<<<nblk, SCAN_THREADS, 0, st>>>(in, out, n, block_sums);
  FS_LAUNCH_CHECK();
  if (nblk > 1) {
    k_scan_block<<<1, SCAN_THREADS, 0, st>>>(block_sums, block_sums, nblk, nullptr);
    FS_LAUNCH_CHECK();
    k_scan_add<<<fs_blocks(n, 256), 256, 0, st>>>(out, n, block_sums);
    FS_LAUNCH_CHECK();
  }
  return FS_OK;
}
