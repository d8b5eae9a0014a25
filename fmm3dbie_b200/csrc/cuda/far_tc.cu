// Multi-density far field of the FP32 path on the 5th-generation tensor cores.
//
// For nd densities the far field is, per target t and density m,
//   y(t, m) = sum_s K(t, s) sigma(s, m),
// a product of the kernel matrix with the density matrix.  Each CTA takes
// 128 targets, one source chunk and N densities.  Per tile of 32 sources its
// 512 threads evaluate the 128 x 32 kernel values with the same FP32 pair
// function and block centring as the CUDA-core kernels (so the
// error-matched W_eff32 fold still cancels their near-pair values) and lay
// the complex product out as one real GEMM of M = 128 rows (targets),
// K = 64 (kernel real parts, then imaginary parts) and 2N columns (the
// densities' real parts, then their imaginary parts):
//   A = [Kr | Ki],  B = [[sr, si], [-si, sr]],  Y = A B = [Re y | Im y].
// Both operands are split into high and low parts (x = hi + lo, hi rounded
// to TF32, lo rounded to TF32 as well) and one thread issues tcgen05.mma
// kind::tf32 for hi*hi + hi*lo + lo*hi (the 3xTF32 scheme, about FP32
// accuracy) into an FP32 accumulator of 2N columns in tensor memory, which
// is read with tcgen05.ld after every tile and added into compensated
// (Kahan) FP32 sums in registers;
// the partial sums of the chunk are written in the CUDA-core kernels'
// layout.  While the tensor core works on a tile, the threads load the next
// tile's sources and densities into registers.  (Double-buffering the kernel
// values and the accumulator, so that a tile's kernel values are computed
// while the previous tile's MMAs run, measured slower: the kernel-value
// stage, not the tensor core, sets the pace.)  Operands sit in shared
// memory in the canonical no-swizzle K-major layout (8-row x 16-byte core
// matrices, row groups 128 B apart, K-direction core matrices (rows / 8) x
// 128 B apart).  Completion waits are bounded; on timeout the kernel records
// the CTA in *err, waits once more (bounded) for its tensor-core work, frees
// its tensor memory and writes nothing.
#include <cuda_runtime.h>

#include <cstdint>

#include "device.cuh"
#include "pair.cuh"
#include "tc_common.cuh"

namespace bie {
namespace dev {
namespace {

constexpr int kTcT = 128;                     // targets per CTA = accumulator rows
constexpr int kTcRows = kTcT;
constexpr int kTcS = 32;                      // sources per tile
constexpr int kTcK = 2 * kTcS;                // reduction length of a tile
constexpr int kTcThreads = 512;
constexpr uint32_t kTcLboA = (kTcRows / 8) * 128;
static_assert(kFarTileSources % kTcS == 0, "chunks are whole tiles");

// Compensated (Kahan) FP32 sum s + v: the running error sits in c, so the
// sum stays accurate to about FP32 rounding over the whole chunk without
// FP32-to-FP64 conversions (which would load the XU pipe).
__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
  const float y = v - c;
  const float t = s + y;
  c = (t - s) - y;
  s = t;
}

// (acc, cmp)[n] += accumulator row 32 (w % 4) + lane, columns c0 .. c0 + NH - 1
// (a warp may read only the tensor-memory lanes of its quarter, w % 4).
template <int NH>
__device__ __forceinline__ void flush(uint32_t tmem, int c0, float* acc, float* cmp) {
  const int quarter = (threadIdx.x >> 5) & 3;
  const uint32_t lanes = uint32_t(quarter * 32) << 16;
  if constexpr (NH == 8) {
    uint32_t v[8];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7])
        : "r"(tmem + lanes + uint32_t(c0)));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 8; ++j) kahan_add(acc[j], cmp[j], __uint_as_float(v[j]));
  } else {
#pragma unroll
    for (int cc = 0; cc < NH; cc += 16) {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
          "%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
            "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(tmem + lanes + uint32_t(c0 + cc)));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 16; ++j) kahan_add(acc[cc + j], cmp[cc + j], __uint_as_float(v[j]));
    }
  }
}

// Operands of one source tile held in registers while the previous tile's
// MMAs run: the source (thread < 32) and this thread's density tasks.
template <int N>
struct TileRegs {
  static constexpr int kTasks = (N * (kTcS / 4) + kTcThreads - 1) / kTcThreads;
  double sx, sy, sz, nx, ny, nz;
  float4 abv;
  float2 sig[kTasks][4];
};

template <int N>
__device__ __forceinline__ void tile_load(const Geometry& g, const float* __restrict__ ab,
                                          const float* __restrict__ sig, int nd, int m0,
                                          int64_t sb, int ns, TileRegs<N>& r) {
  const int tid = threadIdx.x;
  if (tid < kTcS) {
    if (tid < ns) {
      const int64_t s = sb + tid;
      r.sx = g.sx[s], r.sy = g.sy[s], r.sz = g.sz[s];
      r.nx = g.snx[s], r.ny = g.sny[s], r.nz = g.snz[s];
      r.abv = *reinterpret_cast<const float4*>(ab + 4 * s);
    }
  }
#pragma unroll
  for (int k = 0; k < TileRegs<N>::kTasks; ++k) {
    const int q = tid + k * kTcThreads;
    const int n = q % N, sq = 4 * (q / N), m = m0 + n;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      r.sig[k][u] = make_float2(0.f, 0.f);
      if (q < N * (kTcS / 4) && sq + u < ns && m < nd)
        r.sig[k][u] = *reinterpret_cast<const float2*>(sig + (size_t(sb + sq + u) * nd + m) * 2);
    }
  }
}

template <int N, bool CK>
__global__ void __launch_bounds__(kTcThreads, 1)
    far_tc_kernel(Geometry g, KParams kp, const float* __restrict__ ab,
                  const float* __restrict__ sig, int nd, double* __restrict__ partial,
                  int64_t chunk_len, int* __restrict__ err) {
  constexpr int NB = 2 * N;  // GEMM columns: real parts, then imaginary parts
  constexpr int NH = NB / 4;  // accumulator columns per thread (four warps per TMEM lane quarter)
  constexpr uint32_t kLboB = (NB / 8) * 128;
  constexpr uint32_t kCols = NB < 32 ? 32 : NB;  // tensor-memory allocation (power of 2 >= 32)
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  __shared__ float4 sg0[kTcS];
  __shared__ float2 sg1[kTcS];
  __shared__ float4 sab[kTcS];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned char* base = tc_smem + ((1024 - (smem_u32(tc_smem) & 1023)) & 1023);
  float* sAh = reinterpret_cast<float*>(base);
  float* sAl = sAh + kTcRows * kTcK;
  float* sBh = sAl + kTcRows * kTcK;
  float* sBl = sBh + NB * kTcK;

  const int64_t ntarg = g.ntarg, nptso = g.nptso;
  const int64_t tbase = int64_t(blockIdx.x) * kTcT;
  const int m0 = int(blockIdx.z) * N;
  // centre of the 512-target block, as the CUDA-core kernels and the fold use
  const int64_t tcen = (tbase / kFarBlockTargets32) * kFarBlockTargets32;
  const int64_t tcc = tcen < ntarg ? tcen : ntarg - 1;
  const double cx = g.tx[tcc], cy = g.ty[tcc], cz = g.tz[tcc];
  // kernel values: target t against sources 4 (4 j + sgrp) .. + 3, j = 0, 1
  const int t = tid & (kTcT - 1), sgrp = tid >> 7;
  const int64_t it = tbase + t;
  const int64_t ic = it < ntarg ? it : ntarg - 1;
  const float tx = float(g.tx[ic] - cx), ty = float(g.ty[ic] - cy), tz = float(g.tz[ic] - cz);
  const float thr2 = float(kp.thresh * kp.thresh);
  const float k = float(kp.kr), kim = float(kp.ki);
  // accumulator: row (target) 32 (warp % 4) + lane, columns c0 .. c0 + NH - 1
  const int row = 32 * (warp & 3) + lane, c0 = (warp >> 2) * NH;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base)),
                 "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  // operand descriptors of the three products hi*hi, hi*lo, lo*hi
  const uint64_t desc_a[3] = {smem_desc(smem_u32(sAh), kTcLboA), smem_desc(smem_u32(sAh), kTcLboA),
                              smem_desc(smem_u32(sAl), kTcLboA)};
  const uint64_t desc_b[3] = {smem_desc(smem_u32(sBh), kLboB), smem_desc(smem_u32(sBl), kLboB),
                              smem_desc(smem_u32(sBh), kLboB)};

  float acc[NH], cmp[NH];
#pragma unroll
  for (int n = 0; n < NH; ++n) acc[n] = cmp[n] = 0.f;
  const int64_t s0 = int64_t(blockIdx.y) * chunk_len;
  const int64_t s1 = s0 + chunk_len < nptso ? s0 + chunk_len : nptso;
  const int ntiles = s1 > s0 ? int((s1 - s0 + kTcS - 1) / kTcS) : 0;
  auto tile_ns = [&](int i) {
    const int64_t sb = s0 + int64_t(i) * kTcS;
    return int(s1 - sb < kTcS ? s1 - sb : kTcS);
  };
  TileRegs<N> pre;
  if (ntiles > 0) tile_load<N>(g, ab, sig, nd, m0, s0, tile_ns(0), pre);
  bool ok = true;
  int issued = -1;  // last tile whose MMAs were committed
  for (int i = 0; i < ntiles; ++i) {
    const int ns = tile_ns(i);
    if (i > 0) {
      // tile i-1's MMAs read the operand buffers and wrote the accumulator
      ok = wait_phase(&bar, uint32_t(i - 1) & 1u);
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      flush<NH>(tmem, c0, acc, cmp);
    }
    // the prefetched tile -> shared memory
    if (tid < kTcS) {
      if (tid < ns) {
        sg0[tid] = make_float4(float(pre.sx - cx), float(pre.sy - cy), float(pre.sz - cz),
                               float(pre.nx));
        sg1[tid] = make_float2(float(pre.ny), float(pre.nz));
        sab[tid] = pre.abv;
      } else {
        sg0[tid] = make_float4(0.f, 0.f, 0.f, 0.f);
        sg1[tid] = make_float2(0.f, 0.f);
        sab[tid] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    // densities: column n (real part of density m0 + n) = [sr; -si], column
    // N + n (imaginary part) = [si; sr], over sources s (rows s, 32 + s)
#pragma unroll
    for (int kq = 0; kq < TileRegs<N>::kTasks; ++kq) {
      const int q = tid + kq * kTcThreads;
      if (q < N * (kTcS / 4)) {
        const int n = q % N, sq = 4 * (q / N);
        const float2* v = pre.sig[kq];
        store_split(sBh, sBl, op_off(n, sq, kLboB), v[0].x, v[1].x, v[2].x, v[3].x);
        store_split(sBh, sBl, op_off(n, kTcS + sq, kLboB), -v[0].y, -v[1].y, -v[2].y, -v[3].y);
        store_split(sBh, sBl, op_off(N + n, sq, kLboB), v[0].y, v[1].y, v[2].y, v[3].y);
        store_split(sBh, sBl, op_off(N + n, kTcS + sq, kLboB), v[0].x, v[1].x, v[2].x, v[3].x);
      }
    }
    __syncthreads();
    // kernel values of the tile: [Kr | Ki] for this thread's target
#pragma unroll 1
    for (int j = 0; j < kTcS / 16; ++j) {
      const int sq = 4 * (4 * j + sgrp);
      float kr[4], ki[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        kr[u] = 0.f;
        ki[u] = 0.f;
        pair_helm(tx, ty, tz, sg0[sq + u], sg1[sq + u], sab[sq + u], k, kim, thr2, CK, kr[u],
                  ki[u]);
      }
      store_split(sAh, sAl, op_off(t, sq, kTcLboA), kr[0], kr[1], kr[2], kr[3]);
      store_split(sAh, sAl, op_off(t, kTcS + sq, kTcLboA), ki[0], ki[1], ki[2], ki[3]);
    }
    // make the operands visible to the tensor core, then one thread issues
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      constexpr uint32_t idesc = idesc_tf32(kTcRows, NB);
      uint32_t accf = 0u;
#pragma unroll
      for (int p = 0; p < 3; ++p)
#pragma unroll
        for (int st = 0; st < kTcK / 8; ++st) {
          // K step st: two K-direction core matrices further
          const uint64_t da = desc_a[p] + uint64_t(st * ((2 * kTcLboA) >> 4));
          const uint64_t db = desc_b[p] + uint64_t(st * ((2 * kLboB) >> 4));
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::
                  "r"(tmem),
              "l"(da), "l"(db), "r"(idesc), "r"(accf), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
          accf = 1u;
        }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              smem_u32(&bar))
          : "memory");
    }
    issued = i;
    // the next tile's operands load while the tensor core works
    if (i + 1 < ntiles) tile_load<N>(g, ab, sig, nd, m0, s0 + int64_t(i + 1) * kTcS, tile_ns(i + 1), pre);
  }
  if (ok && ntiles > 0) {
    ok = wait_phase(&bar, uint32_t(ntiles - 1) & 1u);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) flush<NH>(tmem, c0, acc, cmp);
  }
  if (!ok) {
    if (tid == 0 && err) atomicExch(err, 1 + int(blockIdx.x));
    // let the last committed MMAs finish before the tensor memory is freed
    for (uint32_t r = 0; r < 4 && issued >= 0; ++r)
      if (wait_phase(&bar, uint32_t(issued) & 1u)) break;
  } else {
    // row: target tbase + row; column c0 + n: real (< N) or imaginary part of
    // density m0 + (c0 + n) % N
    const int64_t to = tbase + row;
    const int comp = c0 >= N ? 1 : 0, d0 = m0 + (c0 % N);
    if (to < ntarg)
#pragma unroll
      for (int n = 0; n < NH; ++n)
        if (d0 + n < nd)
          partial[((size_t(blockIdx.y) * ntarg + to) * nd + d0 + n) * 2 + comp] =
              double(acc[n]) - double(cmp[n]);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

template <int N>
size_t tc_smem_bytes() {
  return sizeof(float) * (2 * kTcRows * kTcK + 2 * (2 * N) * kTcK) + 1024;
}

template <int N, bool CK>
cudaError_t far_tc_go(const Geometry& g, const KParams& kp, const MatvecArgs& a, cudaStream_t st,
                      int* occ) {
  auto kern = far_tc_kernel<N, CK>;
  const size_t smem = tc_smem_bytes<N>();
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(smem));
  if (e != cudaSuccess) return e;
  if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, kTcThreads, smem);
  const int64_t tblocks = (g.ntarg + kTcT - 1) / kTcT;
  const int groups = (a.nd + N - 1) / N;
  int64_t chunk = (g.nptso + a.nchunks - 1) / a.nchunks;
  chunk = ((chunk + kFarTileSources - 1) / kFarTileSources) * kFarTileSources;
  const dim3 grid(unsigned(tblocks), unsigned(a.nchunks), unsigned(groups));
  kern<<<grid, kTcThreads, smem, st>>>(g, kp, static_cast<const float*>(a.ab),
                                       static_cast<const float*>(a.strengths), a.nd, a.partial,
                                       chunk, a.tc_err);
  return cudaGetLastError();
}

template <int N>
cudaError_t far_tc_n(const Geometry& g, const KParams& kp, const MatvecArgs& a, cudaStream_t st,
                     int* occ) {
  return kp.ki != 0.0 ? far_tc_go<N, true>(g, kp, a, st, occ)
                      : far_tc_go<N, false>(g, kp, a, st, occ);
}

}  // namespace

int far_tc_targets() { return kTcT; }

int far_tc_group(int variant, int nd, int precision, int kind) {
  if (variant < 3 || variant > 4 || precision != 1 || kind != 1 || nd < 4) return 0;
  if (variant == 4) return nd > 32 ? 64 : 0;
  return nd <= 16 ? 16 : 32;
}

cudaError_t far_tc(int variant, const Geometry& g, const KParams& kp, const MatvecArgs& a,
                   cudaStream_t st, int* occ) {
  switch (far_tc_group(variant, a.nd, a.precision, kp.kind)) {
    case 16:
      return far_tc_n<16>(g, kp, a, st, occ);
    case 32:
      return far_tc_n<32>(g, kp, a, st, occ);
    case 64:
      return far_tc_n<64>(g, kp, a, st, occ);
    default:
      if (occ) *occ = 0;
      return cudaErrorInvalidValue;
  }
}

}  // namespace dev
}  // namespace bie
