// fs_f32x2.cuh -- packed FP32 pair arithmetic of sm_100 (add/sub/mul/fma .f32x2).
//
// One instruction applies the operation to both halves of a 64-bit register
// pair, round to nearest even, denormals kept: the same result per half as the
// scalar .f32 instruction, in half the issue slots. Used where a kernel is
// issue-bound on FP32 work over naturally paired values (two grid points of
// one z pair in the spread).
#pragma once
#include <stdint.h>

typedef unsigned long long f2p;  // (lo, hi) floats in one 64-bit register

__device__ __forceinline__ f2p f2_pack(float lo, float hi) {
  f2p r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float2 f2_unpack(f2p v) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
__device__ __forceinline__ f2p f2_add(f2p a, f2p b) {
  f2p d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2p f2_sub(f2p a, f2p b) {
  f2p d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2p f2_mul(f2p a, f2p b) {
  f2p d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
// a * b + c, one rounding per half
__device__ __forceinline__ f2p f2_fma(f2p a, f2p b, f2p c) {
  f2p d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
