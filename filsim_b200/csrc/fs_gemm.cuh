// fs_gemm.cuh -- BF16 GEMM on the sm_100a tensor cores (tcgen05.mma, FP32
// accumulators in tensor memory) with fused epilogues, for the warm-start MLP.
//
//   D[m][n] = sum_k A[m][k] B[n][k]      A: M x K, B: N x K, both K contiguous (bf16)
//
// One CTA (4 warps) computes a 128 x BN tile. K advances in 64-element blocks
// through a three-stage shared-memory ring filled by TMA (cp.async.bulk.tensor,
// 128-byte swizzle: row r, 16-byte chunk j at r*128 + (j ^ (r & 7))*16, the
// canonical K-major layout the MMA descriptors name). Thread 0 is the producer:
// per block it waits until the stage's previous MMAs have drained ("empty"
// barrier), announces the stage's bytes on its "full" barrier and issues the two
// tile loads, which complete that barrier. Thread 32 issues the MMAs: it waits on
// "full", issues four K=16 MMAs and commits them to "empty"; after the last block
// it commits to "done". Then each warp reads its 32 accumulator lanes with
// tcgen05.ld and applies the epilogue. Every wait is bounded: on timeout the
// kernel records an error, skips the epilogue, frees its tensor memory and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

typedef __nv_bfloat16 fs_bf16;

enum {
  GEMM_EPI_F32 = 0,    // outF = acc (+ bias)
  GEMM_EPI_SILU = 1,   // z = acc + bias -> aux = z, outH = silu(z), outT = silu(z)^T
  GEMM_EPI_DSILU = 2,  // dz = acc * silu'(aux) -> outH = dz, outT = dz^T
};

struct GemmArgs {
  const fs_bf16 *A;
  const fs_bf16 *B;
  int lda, ldb;
  int M, N, K;
  const float *bias;  // [N] or null
  float *outF;        // [M x N], ldo
  fs_bf16 *outH;      // [M x N], ldh
  fs_bf16 *outT;      // [N x M], ldt
  float *aux;         // [M x N], ldx: pre-activation (stored by SILU, read by DSILU)
  int ldo, ldh, ldt, ldx;
  int *err;           // set to 1 on a timed-out wait
};

namespace fsg {

constexpr int BM = 128, BK = 64, STAGES = 3, THREADS = 128;
constexpr int GEMM_GROUP_M = 32;  // rows of tiles per group of the tile order

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// the stage's bytes announced on its full barrier (this thread's arrival included)
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar), "r"(bytes) : "memory");
}
// one 2-D tile (x = innermost coordinate in elements, y = row) into shared memory,
// completing on mbar; no multicast
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::
          "r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(a), "r"(count) : "memory");
}
// Bounded wait for the completion of the phase with the given parity (about a
// second of polling at most).
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity) {
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.b32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > 2000000000ll) return false;
  }
}

__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(slot), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 bytes apart
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128, N = bn
__host__ __device__ constexpr uint32_t idesc_bf16(int bn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\ntcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar)
               : "memory");
}
// 16 consecutive FP32 accumulator columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float silu_sig(float z) { return 1.0f / (1.0f + expf(-z)); }

template <int BN>
constexpr int smem_bytes() { return STAGES * (BM * 128 + BN * 128) + 1024; }

template <int BN, int EPI>
__global__ void __launch_bounds__(THREADS)
    k_gemm_bf16(GemmArgs g, const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB) {
  constexpr uint32_t A_BYTES = BM * 128, B_BYTES = BN * 128, STAGE_BYTES = A_BYTES + B_BYTES;
  constexpr uint32_t IDESC = idesc_bf16(BN);
  extern __shared__ uint8_t gemm_smem_raw[];
  __shared__ uint64_t full[STAGES], empty[STAGES], done;
  __shared__ uint32_t tmem_slot;
  __shared__ int s_fail, s_issued;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t base = (smem_u32(gemm_smem_raw) + 1023u) & ~1023u;
  // tiles in groups of GEMM_GROUP_M rows of tiles, walked column by column inside a
  // group: the CTAs resident at one time share a few A panels and a band of B
  // panels, which stay in L2 (block x fastest would sweep every A panel per column)
  const int ntm = gridDim.x, ntn = gridDim.y;
  const int lin = blockIdx.x + blockIdx.y * ntm;
  const int per_group = GEMM_GROUP_M * ntn, grp = lin / per_group;
  const int first_m = grp * GEMM_GROUP_M, gsize = min(ntm - first_m, GEMM_GROUP_M);
  const int in_grp = lin - grp * per_group;
  const int m0 = (first_m + in_grp % gsize) * BM, n0 = (in_grp / gsize) * BN;
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    mbar_init(smem_u32(&done), 1);
    s_fail = 0;
    s_issued = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    fence_proxy_async();
  }
  if (warp == 0) tmem_alloc(smem_u32(&tmem_slot), BN);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const int nk = g.K / BK;
  if (tid == 0) {  // producer
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      if (kb >= STAGES && !mbar_wait(smem_u32(&empty[s]), ((kb / STAGES) - 1) & 1)) {
        s_fail = 1;
        break;
      }
      const uint32_t sA = base + s * STAGE_BYTES, sB = sA + A_BYTES;
      mbar_expect_tx(smem_u32(&full[s]), STAGE_BYTES);
      tma_load_2d(sA, &tmA, kb * BK, m0, smem_u32(&full[s]));
      tma_load_2d(sB, &tmB, kb * BK, n0, smem_u32(&full[s]));
      s_issued = kb + 1;
    }
  } else if (tid == 32) {  // MMA issuer
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      if (!mbar_wait(smem_u32(&full[s]), (kb / STAGES) & 1)) {
        s_fail = 1;
        break;
      }
      tc_fence_after();
      const uint32_t sA = base + s * STAGE_BYTES, sB = sA + A_BYTES;
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk)
        mma_bf16(tmem, sw128_desc(sA + kk * 32), sw128_desc(sB + kk * 32), IDESC, (kb | kk) != 0);
      mma_commit(smem_u32(&empty[s]));
    }
    mma_commit(smem_u32(&done));  // arrives once every MMA issued above has completed
  }
  __syncwarp();
  bool ok = mbar_wait(smem_u32(&done), 0);
  __syncthreads();
  ok = ok && !s_fail;
  if (!ok && tid == 0)  // before leaving, the tile loads still in flight land (bounded)
    for (int kb = max(0, s_issued - STAGES); kb < s_issued; ++kb)
      mbar_wait(smem_u32(&full[kb % STAGES]), (kb / STAGES) & 1);
  tc_fence_after();
  if (ok) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
      const int col = n0 + c0;
      if (EPI == GEMM_EPI_F32) {
        if (g.bias)
#pragma unroll
          for (int i = 0; i < 16; ++i) v[i] += g.bias[col + i];
        float4 *o = reinterpret_cast<float4 *>(g.outF + (size_t)row * g.ldo + col);
#pragma unroll
        for (int i = 0; i < 4; ++i) o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
      } else {
        float h[16];
        if (EPI == GEMM_EPI_SILU) {
          float *zx = g.aux + (size_t)row * g.ldx + col;
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const float z = v[i] + g.bias[col + i];
            zx[i] = z;
            h[i] = z * silu_sig(z);
          }
        } else {
          const float *zx = g.aux + (size_t)row * g.ldx + col;
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const float z = zx[i], s = silu_sig(z);
            h[i] = v[i] * s * (1.0f + z * (1.0f - s));
          }
        }
        if (g.outH) {
          __nv_bfloat162 *o = reinterpret_cast<__nv_bfloat162 *>(g.outH + (size_t)row * g.ldh + col);
#pragma unroll
          for (int i = 0; i < 8; ++i) o[i] = __floats2bfloat162_rn(h[2 * i], h[2 * i + 1]);
        }
        if (g.outT)
#pragma unroll
          for (int i = 0; i < 16; ++i) g.outT[(size_t)(col + i) * g.ldt + row] = __float2bfloat16_rn(h[i]);
      }
    }
  } else if (tid == 0) {
    atomicExch(g.err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, BN);
  }
}

}  // namespace fsg
