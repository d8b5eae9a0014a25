// Helpers of the kernels that issue tcgen05.mma kind::tf32 from shared
// memory operands in the canonical no-swizzle K-major layout: 8-row x
// 16-byte core matrices, row groups kTcSbo = 128 bytes apart, K-direction
// core matrices lbo bytes apart; 3xTF32 operand splits; bounded completion
// waits on an mbarrier.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace bie {
namespace dev {
namespace {

constexpr uint32_t kTcSbo = 128;
constexpr uint32_t kTcWaitLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// x rounded to TF32 (10 mantissa bits, ties away from zero) by integer
// operations: add half of the dropped range, clear the low 13 bits.
__device__ __forceinline__ float tf32_rn(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// Shared-memory matrix descriptor: no swizzle, K-major, sm_100 version bits.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFFu);
  d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((kTcSbo >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46;
  return d;
}

// kind::tf32 instruction descriptor: FP32 accumulator (bits 4-5 = 1), TF32 A
// and B (bits 7-9, 10-12 = 2), both K-major, N >> 3 at bit 17, M >> 4 at 24.
constexpr uint32_t idesc_tf32(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(n >> 3) << 17) |
         (uint32_t(m >> 4) << 24);
}

// Float offset of element (row r, column k), k % 4 == 0, in a K-major
// operand whose K-direction core matrices are lbo bytes apart.
__device__ __forceinline__ int op_off(int r, int k, uint32_t lbo) {
  return (k >> 2) * int(lbo >> 2) + (r >> 3) * 32 + (r & 7) * 4;
}

// Four consecutive columns of one row, split into high and low parts
// (hi = x rounded to TF32, lo = x - hi, exact, then rounded to TF32).
__device__ __forceinline__ void store_split(float* hi, float* lo, int off, float a, float b,
                                            float c, float d) {
  const float ha = tf32_rn(a), hb = tf32_rn(b), hc = tf32_rn(c), hd = tf32_rn(d);
  *reinterpret_cast<float4*>(hi + off) = make_float4(ha, hb, hc, hd);
  *reinterpret_cast<float4*>(lo + off) =
      make_float4(tf32_rn(a - ha), tf32_rn(b - hb), tf32_rn(c - hc), tf32_rn(d - hd));
}

// Bounded wait for phase `parity` of the barrier (thread 0 polls, the others
// wait at the CTA barrier); returns whether it completed.
__device__ __forceinline__ bool wait_phase(uint64_t* bar, uint32_t parity) {
  uint32_t done = threadIdx.x == 0 ? 0u : 1u;
  for (uint32_t it = 0; it < kTcWaitLimit && !done; ++it)
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
  return __syncthreads_or(int(!done)) == 0;
}

}  // namespace
}  // namespace dev
}  // namespace bie
