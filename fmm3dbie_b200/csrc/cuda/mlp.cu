// Learned warm start for the Helmholtz combined-field solver.
//
// A per-node MLP maps (incidence direction d, wavenumber k, node position x,
// node normal n) to the demodulated density tau = sigma * exp(-i k d.x) of the
// plane-wave problem (zid I + K) sigma = -exp(i k d.x).  tau varies slowly
// over the surface, so the network only has to learn a smooth function; the
// guess handed to GMRES is tau_hat * exp(i k d.x).
//
// Network: 10 -> 256 -> 256 -> 256 -> 256 -> 2, tanh on the four hidden
// layers, bf16 weights, fp32 accumulation, fp32 master weights and Adam
// moments.  Rows (samples) are independent, so every layer is a GEMM over a
// row batch:
//   Z0 = X W0^T + b0            K = 10   (CUDA cores)
//   Z_l = H_{l-1} W_l^T + b_l   K = 256  (tensor cores), l = 1..3
//   Y  = H3 W4^T + b4           N = 2    (one warp per row)
// with H_l = tanh(Z_l) stored in bf16.  Backward:
//   dZ_{l-1} = (dZ_l W_l) * (1 - H_{l-1}^2)   (tensor cores, fused tanh')
//   dW_l     = dZ_l^T H_{l-1}                 (tensor cores, split over rows)
// The bf16 tensor-core tiles use mma.sync m16n8k16 with ldmatrix (plain or
// transposed, so each of the three GEMM shapes reads W and the activations
// in their stored layout), cp.async double buffering, 128x128x32 CTA tiles.
//
// Parameter layout (fp32, flat): weights W0[256][10], W1..W3[256][256],
// W4[2][256] back to back (their bf16 copy uses the same offsets), then the
// biases b0..b3[256], b4[2].  Gradients use the same layout.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "../../../include/fmm3dbie_b200.h"
#include "device.cuh"
#include "plan.h"

namespace bie {
namespace mlp {

using bf16 = __nv_bfloat16;

constexpr int kIn = 10, kW = 256, kOut = 2;
constexpr int64_t kOffW0 = 0, kOffW1 = 2560, kOffW2 = kOffW1 + 65536, kOffW3 = kOffW2 + 65536,
                  kOffW4 = kOffW3 + 65536, kNW = kOffW4 + 512;
constexpr int64_t kOffB0 = kNW, kOffB1 = kOffB0 + 256, kOffB2 = kOffB1 + 256,
                  kOffB3 = kOffB2 + 256, kOffB4 = kOffB3 + 256, kNParams = kOffB4 + 2;
constexpr int64_t kOffW[4] = {kOffW0, kOffW1, kOffW2, kOffW3};
constexpr int64_t kOffB[4] = {kOffB0, kOffB1, kOffB2, kOffB3};
static_assert(kNParams == 200706, "parameter count");
static_assert((kOffW1 * 2) % 16 == 0 && (kOffW2 * 2) % 16 == 0 && (kOffW3 * 2) % 16 == 0,
              "bf16 weight blocks start on 16-byte boundaries (cp.async)");

constexpr int kRowTile = 128;     // rows are padded to a multiple of this
constexpr int kWgradChunk = 1024; // rows per split of the weight-gradient GEMM
constexpr int kOutPartial = 2 * kW + 3;   // W4 grad, b4 grad, loss
constexpr int kL0Partial = kW * kIn + kW; // W0 grad, b0 grad

__device__ __forceinline__ float bf2f(bf16 v) { return __bfloat162float(v); }
__device__ __forceinline__ bf16 f2bf(float v) { return __float2bfloat16_rn(v); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(smem)), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void ldsm_x4(uint32_t* r, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t* r, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// ---- tensor-core GEMM: C[M x N] = A[M x K] B[K x N] on 128x128 tiles --------
enum Epilogue { kEpiFwd = 0, kEpiBwd = 1, kEpiWgrad = 2 };
constexpr int kBM = 128, kBN = 128, kBK = 32, kPad = 8;
constexpr int kLdK = kBK + kPad;   // tile stored [row][k]
constexpr int kLdMN = kBM + kPad;  // tile stored [k][row]
constexpr int kTileElems = kBM * kLdK;
static_assert(kBK * kLdMN <= kTileElems, "tile buffer holds both layouts");

struct GemmArgs {
  const bf16* A = nullptr;
  const bf16* B = nullptr;
  int64_t lda = 0, ldb = 0;
  int64_t kchunk = 0;  // reduction length per blockIdx.z
  int64_t ktotal = 0;
  void* out = nullptr;
  int64_t ldo = 0, out_zstride = 0;
  const float* bias = nullptr;   // kEpiFwd
  const bf16* hprev = nullptr;   // kEpiBwd: tanh outputs of the layer below (ld = ldo)
};

// AT: A(m, k) is stored at A[k*lda + m] (else A[m*lda + k]).
// BKN: B(k, n) is stored at B[k*ldb + n] (else B[n*ldb + k]).
// Every dimension is a multiple of the tile (checked by the host).
template <bool AT, bool BKN, int EPI>
__global__ void __launch_bounds__(256) mlp_gemm_kernel(GemmArgs g) {
  __shared__ __align__(128) bf16 sA[2][kTileElems];
  __shared__ __align__(128) bf16 sB[2][kTileElems];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;  // warp tile 32 x 64
  const int64_t m0 = int64_t(blockIdx.x) * kBM, n0 = int64_t(blockIdx.y) * kBN;
  const int64_t kbeg = int64_t(blockIdx.z) * g.kchunk;
  const int64_t kend = kbeg + g.kchunk < g.ktotal ? kbeg + g.kchunk : g.ktotal;
  const int nk = kend > kbeg ? int((kend - kbeg) / kBK) : 0;

  auto load = [&](int stage, int64_t kt) {
#pragma unroll
    for (int c = tid; c < 512; c += 256) {
      if (!AT) {
        const int r = c >> 2, c8 = c & 3;
        cp_async16(&sA[stage][r * kLdK + c8 * 8], g.A + (m0 + r) * g.lda + kt + c8 * 8);
      } else {
        const int r = c >> 4, c8 = c & 15;
        cp_async16(&sA[stage][r * kLdMN + c8 * 8], g.A + (kt + r) * g.lda + m0 + c8 * 8);
      }
      if (!BKN) {
        const int r = c >> 2, c8 = c & 3;
        cp_async16(&sB[stage][r * kLdK + c8 * 8], g.B + (n0 + r) * g.ldb + kt + c8 * 8);
      } else {
        const int r = c >> 4, c8 = c & 15;
        cp_async16(&sB[stage][r * kLdMN + c8 * 8], g.B + (kt + r) * g.ldb + n0 + c8 * 8);
      }
    }
  };

  float acc[2][8][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;

  if (nk > 0) load(0, kbeg);
  cp_async_commit();
  for (int it = 0; it < nk; ++it) {
    const int s = it & 1;
    if (it + 1 < nk) load(s ^ 1, kbeg + int64_t(it + 1) * kBK);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const bf16* a = sA[s];
    const bf16* b = sB[s];
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 16) {
      uint32_t af[2][4], bfr[8][2];
      const int q = lane >> 3;
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) {
        if (!AT) {
          const int r = wm * 32 + mi * 16 + (lane & 7) + 8 * (q & 1);
          ldsm_x4(af[mi], a + r * kLdK + kk + 8 * (q >> 1));
        } else {
          const int k = kk + (lane & 7) + 8 * (q >> 1);
          ldsm_x4_t(af[mi], a + k * kLdMN + wm * 32 + mi * 16 + 8 * (q & 1));
        }
      }
#pragma unroll
      for (int nj = 0; nj < 8; nj += 2) {
        uint32_t r4[4];
        if (!BKN) {
          const int n = wn * 64 + nj * 8 + (lane & 7) + 8 * (q >> 1);
          ldsm_x4(r4, b + n * kLdK + kk + 8 * (q & 1));
        } else {
          const int k = kk + (lane & 7) + 8 * (q & 1);
          ldsm_x4_t(r4, b + k * kLdMN + wn * 64 + nj * 8 + 8 * (q >> 1));
        }
        bfr[nj][0] = r4[0];
        bfr[nj][1] = r4[1];
        bfr[nj + 1][0] = r4[2];
        bfr[nj + 1][1] = r4[3];
      }
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int nj = 0; nj < 8; ++nj) mma_bf16(acc[mi][nj], af[mi], bfr[nj]);
    }
    __syncthreads();
  }

  const int gq = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int nj = 0; nj < 8; ++nj) {
      const int64_t c = n0 + wn * 64 + nj * 8 + 2 * tq;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int64_t r = m0 + wm * 32 + mi * 16 + gq + 8 * h;
        float v0 = acc[mi][nj][2 * h], v1 = acc[mi][nj][2 * h + 1];
        if (EPI == kEpiFwd) {
          v0 = tanhf(v0 + g.bias[c]);
          v1 = tanhf(v1 + g.bias[c + 1]);
          *reinterpret_cast<__nv_bfloat162*>(static_cast<bf16*>(g.out) + r * g.ldo + c) =
              __floats2bfloat162_rn(v0, v1);
        } else if (EPI == kEpiBwd) {
          const __nv_bfloat162 hp =
              *reinterpret_cast<const __nv_bfloat162*>(g.hprev + r * g.ldo + c);
          const float h0 = __low2float(hp), h1 = __high2float(hp);
          *reinterpret_cast<__nv_bfloat162*>(static_cast<bf16*>(g.out) + r * g.ldo + c) =
              __floats2bfloat162_rn(v0 * (1.f - h0 * h0), v1 * (1.f - h1 * h1));
        } else {
          float* o = static_cast<float*>(g.out) + int64_t(blockIdx.z) * g.out_zstride;
          *reinterpret_cast<float2*>(o + r * g.ldo + c) = make_float2(v0, v1);
        }
      }
    }
}

// ---- hidden-layer forward on the 5th-generation tensor cores (tcgen05) ---------
// H_l[m0:m0+128, n0:n0+128] = tanh(H_{l-1}[m0:m0+128, :] W_l[n0:n0+128, :]^T + b_l)
// One CTA of 128 threads per 128 x 128 output tile.  Both operands are
// K-major (rows of 256 bf16) and are staged with cp.async in the canonical
// no-swizzle K-major layout of the UMMA shared-memory descriptor: 8-row x
// 16-byte core matrices, core matrix (row group g, K chunk c) at byte
// c * 2048 + g * 128, so the K-direction core-matrix stride (LBO) is 2048 B
// and the row-group stride (SBO) is 128 B.  One thread issues the 16
// tcgen05.mma (M = 128, N = 128, K = 16, kind::f16 with bf16 inputs and an
// fp32 accumulator in 128 TMEM columns) and commits them to an mbarrier;
// every warp then reads its 32 TMEM lanes (rows) with tcgen05.ld and writes
// the bias + tanh epilogue.  The wait on the mbarrier is bounded: on timeout
// the kernel records the tile in *err, still frees its TMEM and returns.
constexpr int kTcM = 128, kTcN = 128, kTcK = 256;
constexpr int kTcThreads = 128;
constexpr uint32_t kTcTileBytes = kTcM * kTcK * 2;         // 64 KB per operand
constexpr uint32_t kTcSmemBytes = 2 * kTcTileBytes + 1024;   // + alignment slack
constexpr uint32_t kTcLbo = 2048, kTcSbo = 128;
constexpr uint32_t kTcWaitLimit = 1u << 24;

__device__ __forceinline__ uint64_t umma_desc_kmajor(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFFu);          // start address
  d |= uint64_t((kTcLbo >> 4) & 0x3FFFu) << 16;   // leading (K-direction) byte offset
  d |= uint64_t((kTcSbo >> 4) & 0x3FFFu) << 32;   // stride (row-group) byte offset
  d |= uint64_t(1) << 46;                          // descriptor version for sm_100
  return d;                                        // base offset 0, no swizzle
}

// kind::f16 instruction descriptor: fp32 accumulator, bf16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

__global__ void __launch_bounds__(kTcThreads, 1)
    mlp_fwd_tc_kernel(const bf16* __restrict__ A, const bf16* __restrict__ Wt,
                      const float* __restrict__ bias, bf16* __restrict__ out,
                      int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t m0 = int64_t(blockIdx.x) * kTcM;
  const int n0 = blockIdx.y * kTcN;
  unsigned char* sA = tc_smem + ((1024 - (smem_u32(tc_smem) & 1023)) & 1023);
  unsigned char* sB = sA + kTcTileBytes;
  // TMEM accumulator (warp 0) and the completion barrier (thread 0)
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base)),
                 "r"(uint32_t(kTcN)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::);
  }
  // operands -> shared memory: 16-byte chunk (row r, K chunk c)
  for (int q = tid; q < kTcM * (kTcK / 8); q += kTcThreads) {
    const int r = q >> 5, c = q & 31;
    const uint32_t off = uint32_t(c) * kTcLbo + uint32_t(r >> 3) * kTcSbo + uint32_t(r & 7) * 16;
    cp_async16(sA + off, A + (m0 + r) * kTcK + c * 8);
    cp_async16(sB + off, Wt + int64_t(n0 + r) * kTcK + c * 8);
  }
  cp_async_commit();
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  // make the shared-memory writes visible to the tensor core (async proxy)
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  if (tid == 0) {
    const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
    constexpr uint32_t idesc = umma_idesc_bf16(kTcM, kTcN);
#pragma unroll 1
    for (int s = 0; s < kTcK / 16; ++s) {
      const uint64_t da = umma_desc_kmajor(a0 + uint32_t(2 * s) * kTcLbo);
      const uint64_t db = umma_desc_kmajor(b0 + uint32_t(2 * s) * kTcLbo);
      const uint32_t acc = s > 0 ? 1u : 0u;
      asm volatile(
          "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
          "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
          "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(&bar))
                 : "memory");
  }
  // bounded wait for the MMAs (phase 0 of the barrier)
  uint32_t done = 0;
  for (uint32_t it = 0; it < kTcWaitLimit && !done; ++it) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(smem_u32(&bar)), "r"(0u)
        : "memory");
  }
  done = __all_sync(0xffffffffu, done);  // tcgen05.ld below is warp-collective
  if (!done && lane == 0) atomicExch(err, 1 + int(blockIdx.x));
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (done) {
    // warp w owns TMEM lanes (rows) 32w .. 32w+31; 16 columns per load
    const int64_t row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < kTcN; c0 += 16) {
      uint32_t v[16];
      const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
            "=r"(v[14]), "=r"(v[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      __align__(16) bf16 o[16];
#pragma unroll
      for (int j = 0; j < 16; ++j)
        o[j] = f2bf(tanhf(__uint_as_float(v[j]) + bias[n0 + c0 + j]));
      uint4* dst = reinterpret_cast<uint4*>(out + row * kW + n0 + c0);
      dst[0] = reinterpret_cast<const uint4*>(o)[0];
      dst[1] = reinterpret_cast<const uint4*>(o)[1];
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(uint32_t(kTcN)));
}

// ---- first layer (K = 10) ----------------------------------------------------
// H0[r][n] = tanh(b0[n] + sum_c W0[n][c] X[r][c]); rows r >= m read X = 0.
__global__ void __launch_bounds__(256) mlp_in_kernel(const float* __restrict__ X, int64_t m,
                                                     const bf16* __restrict__ W0,
                                                     const float* __restrict__ b0,
                                                     bf16* __restrict__ H0) {
  __shared__ float xs[32][kIn];
  const int n = threadIdx.x;
  const int64_t r0 = int64_t(blockIdx.x) * 32;
  for (int i = n; i < 32 * kIn; i += 256) {
    const int64_t r = r0 + i / kIn;
    xs[i / kIn][i % kIn] = r < m ? X[r * kIn + i % kIn] : 0.f;
  }
  float w[kIn];
#pragma unroll
  for (int c = 0; c < kIn; ++c) w[c] = bf2f(W0[n * kIn + c]);
  const float b = b0[n];
  __syncthreads();
  for (int r = 0; r < 32; ++r) {
    float z = b;
#pragma unroll
    for (int c = 0; c < kIn; ++c) z = fmaf(w[c], xs[r][c], z);
    H0[(r0 + r) * kW + n] = f2bf(tanhf(z));
  }
}

// ---- output layer (N = 2), loss and its gradient ----------------------------
// One warp per row, each lane holding 8 of the 256 hidden values.  TRAIN:
// loss = mean_r |Y_r - T_r|^2 over the m valid rows, dZ3 = dL/dZ3 (bf16),
// per-block partial sums of dW4, db4 and the loss.
template <bool TRAIN>
__global__ void __launch_bounds__(256) mlp_out_kernel(const bf16* __restrict__ H3, int64_t m,
                                                      int64_t mp, const bf16* __restrict__ W4,
                                                      const float* __restrict__ b4,
                                                      const float* __restrict__ T,
                                                      float* __restrict__ Y,
                                                      bf16* __restrict__ dZ3,
                                                      float* __restrict__ partial, float inv_m) {
  __shared__ float red[8][kOutPartial];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float w0[8], w1[8], g0[8], g1[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    w0[j] = bf2f(W4[lane * 8 + j]);
    w1[j] = bf2f(W4[kW + lane * 8 + j]);
    g0[j] = g1[j] = 0.f;
  }
  float gb0 = 0.f, gb1 = 0.f, loss = 0.f;
  const float c0 = b4[0], c1 = b4[1];
  for (int64_t r = int64_t(blockIdx.x) * 8 + warp; r < mp; r += int64_t(gridDim.x) * 8) {
    const uint4 raw = *reinterpret_cast<const uint4*>(H3 + r * kW + lane * 8);
    const bf16* hv = reinterpret_cast<const bf16*>(&raw);
    float h[8], y0 = 0.f, y1 = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      h[j] = bf2f(hv[j]);
      y0 = fmaf(h[j], w0[j], y0);
      y1 = fmaf(h[j], w1[j], y1);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      y0 += __shfl_xor_sync(0xffffffffu, y0, o);
      y1 += __shfl_xor_sync(0xffffffffu, y1, o);
    }
    y0 += c0;
    y1 += c1;
    if (Y && lane == 0 && r < m) {
      Y[2 * r] = y0;
      Y[2 * r + 1] = y1;
    }
    if (!TRAIN) continue;
    float d0 = 0.f, d1 = 0.f;
    if (r < m) {
      d0 = y0 - T[2 * r];
      d1 = y1 - T[2 * r + 1];
      loss += d0 * d0 + d1 * d1;
      d0 *= 2.f * inv_m;
      d1 *= 2.f * inv_m;
    }
    gb0 += d0;
    gb1 += d1;
    __align__(16) bf16 dz[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      g0[j] = fmaf(d0, h[j], g0[j]);
      g1[j] = fmaf(d1, h[j], g1[j]);
      dz[j] = f2bf((d0 * w0[j] + d1 * w1[j]) * (1.f - h[j] * h[j]));
    }
    *reinterpret_cast<uint4*>(dZ3 + r * kW + lane * 8) = *reinterpret_cast<const uint4*>(dz);
  }
  if (!TRAIN) return;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    red[warp][lane * 8 + j] = g0[j];
    red[warp][kW + lane * 8 + j] = g1[j];
  }
  if (lane == 0) {
    red[warp][2 * kW] = gb0;
    red[warp][2 * kW + 1] = gb1;
    red[warp][2 * kW + 2] = loss * inv_m;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kOutPartial; i += 256) {
    float s = 0.f;
#pragma unroll
    for (int w = 0; w < 8; ++w) s += red[w][i];
    partial[int64_t(blockIdx.x) * kOutPartial + i] = s;
  }
}

// ---- bias and first-layer gradients ----------------------------------------
// partial[(y*gridDim.x + x)*256 + n] = sum over this block's rows of dZ_y[r][n]
__global__ void __launch_bounds__(256) mlp_colsum_kernel(const bf16* dz1, const bf16* dz2,
                                                         const bf16* dz3, int64_t mp,
                                                         int64_t rows_per_blk, float* partial) {
  const bf16* d = blockIdx.y == 0 ? dz1 : (blockIdx.y == 1 ? dz2 : dz3);
  const int n = threadIdx.x;
  const int64_t r0 = int64_t(blockIdx.x) * rows_per_blk;
  const int64_t r1 = r0 + rows_per_blk < mp ? r0 + rows_per_blk : mp;
  float s = 0.f;
  for (int64_t r = r0; r < r1; ++r) s += bf2f(d[r * kW + n]);
  partial[(int64_t(blockIdx.y) * gridDim.x + blockIdx.x) * kW + n] = s;
}

// partial[blk][n*10 + c] = sum_r dZ0[r][n] X[r][c];  partial[blk][2560 + n] = sum_r dZ0[r][n]
__global__ void __launch_bounds__(256) mlp_l0grad_kernel(const bf16* __restrict__ dz0,
                                                         const float* __restrict__ X, int64_t m,
                                                         int64_t rows_per_blk,
                                                         float* __restrict__ partial) {
  __shared__ float xs[32][kIn];
  const int n = threadIdx.x;
  float acc[kIn + 1];
#pragma unroll
  for (int c = 0; c <= kIn; ++c) acc[c] = 0.f;
  const int64_t r0 = int64_t(blockIdx.x) * rows_per_blk;
  const int64_t r1 = r0 + rows_per_blk < m ? r0 + rows_per_blk : m;
  for (int64_t rb = r0; rb < r1; rb += 32) {
    __syncthreads();
    for (int i = n; i < 32 * kIn; i += 256) {
      const int64_t r = rb + i / kIn;
      xs[i / kIn][i % kIn] = r < r1 ? X[r * kIn + i % kIn] : 0.f;
    }
    __syncthreads();
    const int nr = r1 - rb < 32 ? int(r1 - rb) : 32;
    for (int j = 0; j < nr; ++j) {
      const float z = bf2f(dz0[(rb + j) * kW + n]);
#pragma unroll
      for (int c = 0; c < kIn; ++c) acc[c] = fmaf(z, xs[j][c], acc[c]);
      acc[kIn] += z;
    }
  }
  float* p = partial + int64_t(blockIdx.x) * kL0Partial;
#pragma unroll
  for (int c = 0; c < kIn; ++c) p[n * kIn + c] = acc[c];
  p[kW * kIn + n] = acc[kIn];
}

// ---- deterministic reduction of per-block partial sums ------------------------
struct Seg {
  const float* src = nullptr;
  int64_t stride = 0;
  int nblk = 0, len = 0;
  float* dst = nullptr;
};
constexpr int kMaxSegs = 12;
struct Segs {
  Seg s[kMaxSegs];
};

__global__ void __launch_bounds__(256) mlp_reduce_kernel(Segs segs) {
  const Seg sg = segs.s[blockIdx.y];
  for (int i = blockIdx.x * 256 + threadIdx.x; i < sg.len; i += gridDim.x * 256) {
    float acc = 0.f;
    for (int b = 0; b < sg.nblk; ++b) acc += sg.src[int64_t(b) * sg.stride + i];
    sg.dst[i] = acc;
  }
}

// ---- Adam (decoupled bias correction) and the bf16 weight copy ----------------
__global__ void __launch_bounds__(256) mlp_adam_kernel(float* __restrict__ P,
                                                       const float* __restrict__ G,
                                                       float* __restrict__ Mo,
                                                       float* __restrict__ V,
                                                       bf16* __restrict__ Wb, float lr, float b1,
                                                       float b2, float eps, float bc1, float bc2) {
  const int64_t i = int64_t(blockIdx.x) * 256 + threadIdx.x;
  if (i >= kNParams) return;
  const float g = G[i];
  const float mo = b1 * Mo[i] + (1.f - b1) * g;
  const float v = b2 * V[i] + (1.f - b2) * g * g;
  Mo[i] = mo;
  V[i] = v;
  const float p = P[i] - lr * (mo / bc1) / (sqrtf(v / bc2) + eps);
  P[i] = p;
  if (i < kNW) Wb[i] = f2bf(p);
}

__global__ void mlp_cast_kernel(const float* __restrict__ P, bf16* __restrict__ Wb) {
  const int64_t i = int64_t(blockIdx.x) * 256 + threadIdx.x;
  if (i < kNW) Wb[i] = f2bf(P[i]);
}

// ---- features, training samples, (de)modulation --------------------------------
// Feature row: d (3), (k - kc) / ks, x / xs (3), n (3).  sv: one srcvals
// column (x, dx/du, dx/dv, n); dk: (dx, dy, dz, k).
__device__ __forceinline__ void features(const double* sv, const double* dk, double xs,
                                         double kc, double ks, float* f) {
  f[0] = float(dk[0]);
  f[1] = float(dk[1]);
  f[2] = float(dk[2]);
  f[3] = float((dk[3] - kc) / ks);
  f[4] = float(sv[0] / xs);
  f[5] = float(sv[1] / xs);
  f[6] = float(sv[2] / xs);
  f[7] = float(sv[9]);
  f[8] = float(sv[10]);
  f[9] = float(sv[11]);
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Row r draws sample s = hash(seed, r) mod (nsolves*npts) (solve s / npts,
// node s % npts); tau[(j*npts + i)] is complex fp32.
__global__ void mlp_gather_kernel(const double* __restrict__ srcvals, int64_t npts,
                                  const double* __restrict__ dirk, int64_t nsolves,
                                  const float* __restrict__ tau, double xs, double kc, double ks,
                                  uint64_t seed, int64_t m, float* __restrict__ X,
                                  float* __restrict__ T) {
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= m) return;
  const uint64_t total = uint64_t(nsolves) * uint64_t(npts);
  const uint64_t s = __umul64hi(splitmix64(seed ^ (uint64_t(r) * 0xD1B54A32D192ED03ull)), total);
  const int64_t j = int64_t(s / uint64_t(npts)), i = int64_t(s % uint64_t(npts));
  float f[kIn];
  features(srcvals + 12 * i, dirk + 4 * j, xs, kc, ks, f);
#pragma unroll
  for (int c = 0; c < kIn; ++c) X[r * kIn + c] = f[c];
  T[2 * r] = tau[2 * (j * npts + i)];
  T[2 * r + 1] = tau[2 * (j * npts + i) + 1];
}

// Rows r in [r0, r0 + mc) of the point-major (node i, solve q) list, r = i*nd + q.
__global__ void mlp_predict_features_kernel(const double* __restrict__ srcvals,
                                            const double* __restrict__ dirk, int64_t nd,
                                            double xs, double kc, double ks, int64_t r0,
                                            int64_t mc, float* __restrict__ X) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= mc) return;
  const int64_t r = r0 + t, i = r / nd, q = r % nd;
  float f[kIn];
  features(srcvals + 12 * i, dirk + 4 * q, xs, kc, ks, f);
#pragma unroll
  for (int c = 0; c < kIn; ++c) X[t * kIn + c] = f[c];
}

// x0[r] = (Y0 + i Y1) exp(i k_q d_q . x_i), complex128 interleaved.
__global__ void mlp_remod_kernel(const double* __restrict__ srcvals,
                                 const double* __restrict__ dirk, int64_t nd, int64_t r0,
                                 int64_t mc, const float* __restrict__ Y,
                                 double* __restrict__ x0) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= mc) return;
  const int64_t r = r0 + t, i = r / nd, q = r % nd;
  const double* sv = srcvals + 12 * i;
  const double* dk = dirk + 4 * q;
  const double ph = dk[3] * (dk[0] * sv[0] + dk[1] * sv[1] + dk[2] * sv[2]);
  double s, c;
  sincos(ph, &s, &c);
  const double yr = Y[2 * t], yi = Y[2 * t + 1];
  x0[2 * r] = yr * c - yi * s;
  x0[2 * r + 1] = yr * s + yi * c;
}

// tau[(q*npts + i)] = sigma[(i*nd + q)] exp(-i k_q d_q . x_i), complex fp32.
__global__ void mlp_demod_kernel(const double* __restrict__ srcvals, int64_t npts,
                                 const double* __restrict__ dirk, int64_t nd,
                                 const double* __restrict__ sigma, float* __restrict__ tau) {
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= npts * nd) return;
  const int64_t i = r / nd, q = r % nd;
  const double* sv = srcvals + 12 * i;
  const double* dk = dirk + 4 * q;
  const double ph = dk[3] * (dk[0] * sv[0] + dk[1] * sv[1] + dk[2] * sv[2]);
  double s, c;
  sincos(ph, &s, &c);
  const double sr = sigma[2 * r], si = sigma[2 * r + 1];
  tau[2 * (q * npts + i)] = float(sr * c + si * s);
  tau[2 * (q * npts + i) + 1] = float(si * c - sr * s);
}

// ---- host side -----------------------------------------------------------------
#define MLP_CUDA(call)                                                           \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess) {                                                     \
      ::bie::set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
      return e_ == cudaErrorMemoryAllocation ? ::bie::kErrNoMem : ::bie::kErrCuda; \
    }                                                                            \
  } while (0)

struct Net {
  int device = 0, num_sms = 148;
  int64_t max_rows = 0, mp_max = 0, nsplit_max = 0, nblk_out = 0, nblk_cs = 0, nblk_l0 = 0;
  int64_t step = 0;
  DBuf<float> P, G, Mo, V, Xs, Ys, wg_part, l0_part, cs_part, out_part, loss;
  DBuf<bf16> Wb, H, dZ;
  DBuf<int> tc_err;   // set by the tcgen05 kernel if its completion wait times out
  int engine = 0;     // hidden-layer forward GEMM: 0 mma.sync, 1 tcgen05

  int init(int64_t rows) {
    MLP_CUDA(cudaGetDevice(&device));
    MLP_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
    max_rows = rows;
    mp_max = (rows + kRowTile - 1) / kRowTile * kRowTile;
    nsplit_max = (mp_max + kWgradChunk - 1) / kWgradChunk;
    nblk_out = std::min<int64_t>(2 * num_sms, mp_max / 8);
    nblk_cs = std::min<int64_t>(num_sms, mp_max / 64);
    nblk_l0 = std::min<int64_t>(num_sms, mp_max / 64);
    MLP_CUDA(P.alloc(kNParams));
    MLP_CUDA(G.alloc(kNParams));
    MLP_CUDA(Mo.alloc(kNParams));
    MLP_CUDA(V.alloc(kNParams));
    MLP_CUDA(Wb.alloc(kNW));
    MLP_CUDA(Xs.alloc(size_t(mp_max) * kIn));
    MLP_CUDA(Ys.alloc(size_t(mp_max) * kOut));
    MLP_CUDA(H.alloc(size_t(4) * mp_max * kW));
    MLP_CUDA(dZ.alloc(size_t(4) * mp_max * kW));
    MLP_CUDA(wg_part.alloc(size_t(3) * nsplit_max * kW * kW));
    MLP_CUDA(l0_part.alloc(size_t(nblk_l0) * kL0Partial));
    MLP_CUDA(cs_part.alloc(size_t(3) * nblk_cs * kW));
    MLP_CUDA(out_part.alloc(size_t(nblk_out) * kOutPartial));
    MLP_CUDA(loss.alloc(1));
    MLP_CUDA(tc_err.alloc(1));
    MLP_CUDA(cudaMemset(tc_err.p, 0, sizeof(int)));
    MLP_CUDA(cudaFuncSetAttribute(mlp_fwd_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(kTcSmemBytes)));
    MLP_CUDA(cudaMemset(P.p, 0, kNParams * sizeof(float)));
    MLP_CUDA(cudaMemset(Mo.p, 0, kNParams * sizeof(float)));
    MLP_CUDA(cudaMemset(V.p, 0, kNParams * sizeof(float)));
    MLP_CUDA(cudaMemset(Wb.p, 0, kNW * sizeof(bf16)));
    MLP_CUDA(cudaMemset(H.p, 0, size_t(4) * mp_max * kW * sizeof(bf16)));
    return kOk;
  }
  bf16* Hl(int l) const { return H.p + size_t(l) * mp_max * kW; }
  bf16* dZl(int l) const { return dZ.p + size_t(l) * mp_max * kW; }

  int check_rows(int64_t m) const {
    if (m < 1 || m > max_rows) {
      set_last_error("mlp: row count " + std::to_string(m) + " outside [1, " +
                     std::to_string(max_rows) + "]");
      return kErrArg;
    }
    return kOk;
  }

  // Forward over m rows (padded to mp).  TRAIN also writes dZ3 and the output
  // partial sums for targets T; Y (optional) receives the m outputs.
  int forward(const float* X, int64_t m, const float* T, float* Y, bool train, cudaStream_t st) {
    const int64_t mp = (m + kRowTile - 1) / kRowTile * kRowTile;
    mlp_in_kernel<<<unsigned(mp / 32), 256, 0, st>>>(X, m, Wb.p + kOffW0, P.p + kOffB0, Hl(0));
    for (int l = 1; l <= 3; ++l) {
      if (engine == 1) {
        mlp_fwd_tc_kernel<<<dim3(unsigned(mp / kTcM), kW / kTcN, 1), kTcThreads, kTcSmemBytes, st>>>(
            Hl(l - 1), Wb.p + kOffW[l], P.p + kOffB[l], Hl(l), tc_err.p);
        continue;
      }
      GemmArgs g;
      g.A = Hl(l - 1);
      g.lda = kW;
      g.B = Wb.p + kOffW[l];
      g.ldb = kW;
      g.kchunk = g.ktotal = kW;
      g.out = Hl(l);
      g.ldo = kW;
      g.bias = P.p + kOffB[l];
      mlp_gemm_kernel<false, false, kEpiFwd><<<dim3(unsigned(mp / kBM), kW / kBN, 1), 256, 0, st>>>(g);
    }
    const unsigned nb = unsigned(std::min<int64_t>(nblk_out, mp / 8));
    if (train)
      mlp_out_kernel<true><<<nb, 256, 0, st>>>(Hl(3), m, mp, Wb.p + kOffW4, P.p + kOffB4, T, Y,
                                               dZl(3), out_part.p, 1.f / float(m));
    else
      mlp_out_kernel<false><<<nb, 256, 0, st>>>(Hl(3), m, mp, Wb.p + kOffW4, P.p + kOffB4,
                                                nullptr, Y, nullptr, nullptr, 1.f);
    dev::note_launches(5);
    MLP_CUDA(cudaGetLastError());
    return kOk;
  }

  // Gradient of the mean squared error into G, the loss into loss_out.
  int grad(const float* X, const float* T, int64_t m, float* loss_out, cudaStream_t st) {
    int ier = forward(X, m, T, nullptr, true, st);
    if (ier) return ier;
    const int64_t mp = (m + kRowTile - 1) / kRowTile * kRowTile;
    const unsigned nb_out = unsigned(std::min<int64_t>(nblk_out, mp / 8));
    // dZ_{l-1} = (dZ_l W_l) * (1 - H_{l-1}^2)
    for (int l = 3; l >= 1; --l) {
      GemmArgs g;
      g.A = dZl(l);
      g.lda = kW;
      g.B = Wb.p + kOffW[l];
      g.ldb = kW;
      g.kchunk = g.ktotal = kW;
      g.out = dZl(l - 1);
      g.ldo = kW;
      g.hprev = Hl(l - 1);
      mlp_gemm_kernel<false, true, kEpiBwd><<<dim3(unsigned(mp / kBM), kW / kBN, 1), 256, 0, st>>>(g);
    }
    // dW_l = dZ_l^T H_{l-1}, split over row chunks
    const int64_t nsplit = (mp + kWgradChunk - 1) / kWgradChunk;
    for (int l = 1; l <= 3; ++l) {
      GemmArgs g;
      g.A = dZl(l);
      g.lda = kW;
      g.B = Hl(l - 1);
      g.ldb = kW;
      g.kchunk = kWgradChunk;
      g.ktotal = mp;
      g.out = wg_part.p + size_t(l - 1) * nsplit_max * kW * kW;
      g.ldo = kW;
      g.out_zstride = int64_t(kW) * kW;
      mlp_gemm_kernel<true, true, kEpiWgrad>
          <<<dim3(kW / kBM, kW / kBN, unsigned(nsplit)), 256, 0, st>>>(g);
    }
    const int64_t ncs = std::min<int64_t>(nblk_cs, mp / 64);
    const int64_t rows_cs = (mp + ncs - 1) / ncs;
    mlp_colsum_kernel<<<dim3(unsigned(ncs), 3), 256, 0, st>>>(dZl(1), dZl(2), dZl(3), mp, rows_cs,
                                                             cs_part.p);
    const int64_t nl0 = std::min<int64_t>(nblk_l0, mp / 64);
    const int64_t rows_l0 = (m + nl0 - 1) / nl0;
    mlp_l0grad_kernel<<<unsigned(nl0), 256, 0, st>>>(dZl(0), X, m, rows_l0, l0_part.p);
    Segs sg;
    int ns = 0;
    sg.s[ns++] = Seg{l0_part.p, kL0Partial, int(nl0), kW * kIn, G.p + kOffW0};
    sg.s[ns++] = Seg{l0_part.p + kW * kIn, kL0Partial, int(nl0), kW, G.p + kOffB0};
    for (int l = 1; l <= 3; ++l) {
      sg.s[ns++] = Seg{wg_part.p + size_t(l - 1) * nsplit_max * kW * kW, int64_t(kW) * kW,
                       int(nsplit), kW * kW, G.p + kOffW[l]};
      sg.s[ns++] = Seg{cs_part.p + size_t(l - 1) * ncs * kW, kW, int(ncs), kW, G.p + kOffB[l]};
    }
    sg.s[ns++] = Seg{out_part.p, kOutPartial, int(nb_out), 2 * kW, G.p + kOffW4};
    sg.s[ns++] = Seg{out_part.p + 2 * kW, kOutPartial, int(nb_out), 2, G.p + kOffB4};
    sg.s[ns++] = Seg{out_part.p + 2 * kW + 2, kOutPartial, int(nb_out), 1,
                     loss_out ? loss_out : loss.p};
    mlp_reduce_kernel<<<dim3(64, unsigned(ns)), 256, 0, st>>>(sg);
    dev::note_launches(3 + 3 + 1 + 1 + 1);
    MLP_CUDA(cudaGetLastError());
    return kOk;
  }

  int adam(double lr, cudaStream_t st) {
    ++step;
    const double b1 = 0.9, b2 = 0.999;
    const float bc1 = float(1.0 - std::pow(b1, double(step)));
    const float bc2 = float(1.0 - std::pow(b2, double(step)));
    mlp_adam_kernel<<<unsigned((kNParams + 255) / 256), 256, 0, st>>>(
        P.p, G.p, Mo.p, V.p, Wb.p, float(lr), float(b1), float(b2), 1e-8f, bc1, bc2);
    dev::note_launches(1);
    MLP_CUDA(cudaGetLastError());
    return kOk;
  }
};

}  // namespace mlp
}  // namespace bie

using bie::mlp::Net;

namespace {

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

int bad(const char* msg) {
  bie::set_last_error(msg);
  return BIE_ERR_ARG;
}

}  // namespace

extern "C" int bie_mlp_create(int64_t max_rows, void** mlp) {
  if (!mlp) return bad("mlp: null handle pointer");
  *mlp = nullptr;
  if (max_rows < 1 || max_rows > (int64_t(1) << 24)) return bad("mlp: max_rows outside [1, 2^24]");
  Net* n = new Net();
  const int ier = n->init(max_rows);
  if (ier) {
    delete n;
    return ier;
  }
  *mlp = n;
  return BIE_OK;
}

extern "C" int bie_mlp_destroy(void* mlp) {
  delete static_cast<Net*>(mlp);
  return BIE_OK;
}

extern "C" int bie_mlp_info(void* mlp, int64_t* info) {
  if (!mlp || !info) return bad("mlp: null argument");
  const Net* n = static_cast<const Net*>(mlp);
  info[0] = bie::mlp::kNParams;
  info[1] = n->max_rows;
  info[2] = bie::mlp::kIn;
  info[3] = bie::mlp::kW;
  info[4] = 4;
  info[5] = bie::mlp::kOut;
  info[6] = n->step;
  info[7] = bie::mlp::kNW;
  info[8] = n->engine;
  int flag = 0;
  if (cudaMemcpy(&flag, n->tc_err.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return BIE_ERR_CUDA;
  info[9] = flag;
  return BIE_OK;
}

extern "C" int bie_mlp_set_engine(void* mlp, int64_t engine) {
  if (!mlp || (engine != 0 && engine != 1)) return bad("mlp: engine must be 0 (mma.sync) or 1 (tcgen05)");
  static_cast<Net*>(mlp)->engine = int(engine);
  return BIE_OK;
}

extern "C" int bie_mlp_set_params(void* mlp, const float* params_dev, void* stream) {
  if (!mlp || !params_dev) return bad("mlp: null argument");
  Net* n = static_cast<Net*>(mlp);
  const cudaStream_t st = as_stream(stream);
  using namespace bie::mlp;
  MLP_CUDA(cudaMemcpyAsync(n->P.p, params_dev, kNParams * sizeof(float), cudaMemcpyDeviceToDevice, st));
  MLP_CUDA(cudaMemsetAsync(n->Mo.p, 0, kNParams * sizeof(float), st));
  MLP_CUDA(cudaMemsetAsync(n->V.p, 0, kNParams * sizeof(float), st));
  mlp_cast_kernel<<<unsigned((kNW + 255) / 256), 256, 0, st>>>(n->P.p, n->Wb.p);
  bie::dev::note_launches(1);
  MLP_CUDA(cudaGetLastError());
  n->step = 0;
  return BIE_OK;
}

extern "C" int bie_mlp_get_params(void* mlp, float* params_dev, void* stream) {
  if (!mlp || !params_dev) return bad("mlp: null argument");
  Net* n = static_cast<Net*>(mlp);
  using namespace bie::mlp;
  MLP_CUDA(cudaMemcpyAsync(params_dev, n->P.p, kNParams * sizeof(float), cudaMemcpyDeviceToDevice,
                           as_stream(stream)));
  return BIE_OK;
}

extern "C" int bie_mlp_forward(void* mlp, const float* x_dev, int64_t m, float* y_dev,
                               void* stream) {
  if (!mlp || !x_dev || !y_dev) return bad("mlp: null argument");
  Net* n = static_cast<Net*>(mlp);
  if (int ier = n->check_rows(m)) return ier;
  return n->forward(x_dev, m, nullptr, y_dev, false, as_stream(stream));
}

extern "C" int bie_mlp_grad(void* mlp, const float* x_dev, const float* t_dev, int64_t m,
                            float* grad_dev, float* loss_dev, void* stream) {
  if (!mlp || !x_dev || !t_dev) return bad("mlp: null argument");
  Net* n = static_cast<Net*>(mlp);
  if (int ier = n->check_rows(m)) return ier;
  const cudaStream_t st = as_stream(stream);
  if (int ier = n->grad(x_dev, t_dev, m, loss_dev, st)) return ier;
  using namespace bie::mlp;
  if (grad_dev)
    MLP_CUDA(cudaMemcpyAsync(grad_dev, n->G.p, kNParams * sizeof(float), cudaMemcpyDeviceToDevice, st));
  return BIE_OK;
}

extern "C" int bie_mlp_train_step(void* mlp, const float* x_dev, const float* t_dev, int64_t m,
                                  double lr, float* loss_dev, void* stream) {
  if (!mlp || !x_dev || !t_dev) return bad("mlp: null argument");
  if (!(lr > 0.0)) return bad("mlp: learning rate must be positive");
  Net* n = static_cast<Net*>(mlp);
  if (int ier = n->check_rows(m)) return ier;
  const cudaStream_t st = as_stream(stream);
  if (int ier = n->grad(x_dev, t_dev, m, loss_dev, st)) return ier;
  return n->adam(lr, st);
}

extern "C" int bie_mlp_gather(const double* srcvals_dev, int64_t npts, const double* dirk_dev,
                              int64_t nsolves, const float* tau_dev, const double* norm,
                              uint64_t seed, int64_t m, float* x_dev, float* t_dev,
                              void* stream) {
  if (!srcvals_dev || !dirk_dev || !tau_dev || !norm || !x_dev || !t_dev)
    return bad("mlp_gather: null argument");
  if (npts < 1 || nsolves < 1 || m < 1) return bad("mlp_gather: sizes must be positive");
  if (!(norm[0] > 0.0) || !(norm[2] > 0.0)) return bad("mlp_gather: scales must be positive");
  using namespace bie::mlp;
  mlp_gather_kernel<<<unsigned((m + 255) / 256), 256, 0, as_stream(stream)>>>(
      srcvals_dev, npts, dirk_dev, nsolves, tau_dev, norm[0], norm[1], norm[2], seed, m, x_dev,
      t_dev);
  bie::dev::note_launches(1);
  MLP_CUDA(cudaGetLastError());
  return BIE_OK;
}

extern "C" int bie_mlp_demodulate(const double* srcvals_dev, int64_t npts, const double* dirk_dev,
                                  int64_t nd, const double* sigma_dev, float* tau_dev,
                                  void* stream) {
  if (!srcvals_dev || !dirk_dev || !sigma_dev || !tau_dev) return bad("mlp_demodulate: null argument");
  if (npts < 1 || nd < 1) return bad("mlp_demodulate: sizes must be positive");
  using namespace bie::mlp;
  const int64_t n = npts * nd;
  mlp_demod_kernel<<<unsigned((n + 255) / 256), 256, 0, as_stream(stream)>>>(
      srcvals_dev, npts, dirk_dev, nd, sigma_dev, tau_dev);
  bie::dev::note_launches(1);
  MLP_CUDA(cudaGetLastError());
  return BIE_OK;
}

extern "C" int bie_mlp_predict_density(void* mlp, const double* srcvals_dev, int64_t npts,
                                       const double* dirk_dev, int64_t nd, const double* norm,
                                       double* x0_dev, void* stream) {
  if (!mlp || !srcvals_dev || !dirk_dev || !norm || !x0_dev)
    return bad("mlp_predict_density: null argument");
  if (npts < 1 || nd < 1) return bad("mlp_predict_density: sizes must be positive");
  if (!(norm[0] > 0.0) || !(norm[2] > 0.0)) return bad("mlp_predict_density: scales must be positive");
  Net* n = static_cast<Net*>(mlp);
  const cudaStream_t st = as_stream(stream);
  using namespace bie::mlp;
  const int64_t total = npts * nd;
  for (int64_t r0 = 0; r0 < total; r0 += n->max_rows) {
    const int64_t mc = std::min(n->max_rows, total - r0);
    const unsigned nb = unsigned((mc + 255) / 256);
    mlp_predict_features_kernel<<<nb, 256, 0, st>>>(srcvals_dev, dirk_dev, nd, norm[0], norm[1],
                                                    norm[2], r0, mc, n->Xs.p);
    bie::dev::note_launches(1);
    MLP_CUDA(cudaGetLastError());
    if (int ier = n->forward(n->Xs.p, mc, nullptr, n->Ys.p, false, st)) return ier;
    mlp_remod_kernel<<<nb, 256, 0, st>>>(srcvals_dev, dirk_dev, nd, r0, mc, n->Ys.p, x0_dev);
    bie::dev::note_launches(1);
    MLP_CUDA(cudaGetLastError());
  }
  return BIE_OK;
}
