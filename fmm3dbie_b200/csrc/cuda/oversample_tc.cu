// Oversampling of several complex densities on the 5th-generation tensor
// cores (oversample_fun_guru, src/surface_routs/surf_routs.f90:511-591, for
// nd densities at once).
//
// Per patch the oversampled densities are one product
//   sigma_over (nf x nd) = I (nf x np) sigma_patch (np x nd),
// I the patch class's interpolation matrix (basis values at the far nodes
// times the inverse Vandermonde at the patch nodes).  Written as a real GEMM
// D = A B with A = I (M = 128 rows: the far nodes, zero-padded), K = np
// padded to a multiple of 8, and B holding the densities' real parts and
// then their imaginary parts as 2 nd columns, so D = [Re | Im] of
// sigma_over.  Both operands are split into TF32 high and low parts and one
// thread issues tcgen05.mma kind::tf32 for hi*hi + hi*lo + lo*hi into an FP32
// accumulator in tensor memory (3xTF32, about FP32 accuracy; the outputs are
// FP32 oversampled densities, as the CUDA-core kernel writes them for the
// FP32 far field).  One CTA (4 warps, one per tensor-memory lane quarter)
// per patch; operands in the canonical no-swizzle K-major layout; the
// completion wait is bounded, and on timeout the kernel records it in *err,
// waits once more (bounded) for its MMAs, frees its tensor memory and
// writes nothing.
//
// The contraction is small (np = 15..45, nf <= 128) and memory-bound: the
// densities are read once and the oversampled densities written once, as in
// the CUDA-core kernel, so the tensor cores cannot shorten it; it is kept as
// an engine of its own (bie_set_oversample_engine) with its accuracy and its
// time measured beside the CUDA-core kernel.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdlib>

#include "device.cuh"
#include "tc_common.cuh"

namespace bie {
namespace dev {
namespace {

constexpr int kOsThreads = 128;  // warp w reads tensor-memory lanes 32 w .. 32 w + 31
constexpr int kOsRows = 128;     // M: far nodes of one patch, zero-padded
constexpr uint32_t kOsLboA = (kOsRows / 8) * 128;

__global__ void __launch_bounds__(kOsThreads)
    oversample_tc_kernel(Geometry g, const double* __restrict__ sigma, float* __restrict__ sover,
                         int nd, int kpad, uint32_t ncols, const int32_t* __restrict__ sdest,
                         int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char os_smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nb = 2 * nd;  // GEMM columns: real parts, then imaginary parts
  const uint32_t lbo_b = uint32_t(nb / 8) * 128;
  unsigned char* base = os_smem + ((1024 - (smem_u32(os_smem) & 1023)) & 1023);
  float* sAh = reinterpret_cast<float*>(base);
  float* sAl = sAh + kOsRows * kpad;
  float* sBh = sAl + kOsRows * kpad;
  float* sBl = sBh + nb * kpad;
  const int p = blockIdx.x;
  const int ps = g.pstart[p], np = g.pstart[p + 1] - ps;
  const int os = g.ostart[p], nf = g.ostart[p + 1] - os;
  const double* M = g.imat + g.cmoff[g.pclass[p]];  // nf x np, row-major

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::);
  }
  // A: row r = far node, columns k .. k + 3 = patch nodes
  for (int idx = tid; idx < kOsRows * (kpad / 4); idx += kOsThreads) {
    const int r = idx % kOsRows, kq = 4 * (idx / kOsRows);
    float v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      v[u] = (r < nf && kq + u < np) ? float(M[size_t(r) * np + kq + u]) : 0.f;
    store_split(sAh, sAl, op_off(r, kq, kOsLboA), v[0], v[1], v[2], v[3]);
  }
  // B: row n = density column (real part of density n for n < nd, imaginary
  // part of density n - nd otherwise), columns k .. k + 3 = patch nodes
  for (int idx = tid; idx < nb * (kpad / 4); idx += kOsThreads) {
    const int n = idx % nb, kq = 4 * (idx / nb);
    const int comp = n >= nd ? 1 : 0, m = n - comp * nd;
    float v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      v[u] = kq + u < np ? float(sigma[2 * ((size_t(ps) + kq + u) * nd + m) + comp]) : 0.f;
    store_split(sBh, sBl, op_off(n, kq, lbo_b), v[0], v[1], v[2], v[3]);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  if (tid == 0) {
    const uint64_t desc_a[3] = {smem_desc(smem_u32(sAh), kOsLboA),
                                smem_desc(smem_u32(sAh), kOsLboA),
                                smem_desc(smem_u32(sAl), kOsLboA)};
    const uint64_t desc_b[3] = {smem_desc(smem_u32(sBh), lbo_b), smem_desc(smem_u32(sBl), lbo_b),
                                smem_desc(smem_u32(sBh), lbo_b)};
    const uint32_t idesc = idesc_tf32(kOsRows, nb);
    uint32_t accf = 0u;
    for (int q = 0; q < 3; ++q)
      for (int st = 0; st < kpad / 8; ++st) {
        // K step st: two K-direction core matrices further
        const uint64_t da = desc_a[q] + uint64_t(st * ((2 * kOsLboA) >> 4));
        const uint64_t db = desc_b[q] + uint64_t(st * ((2 * lbo_b) >> 4));
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
  bool ok = wait_phase(&bar, 0u);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    // row = far node 32 warp + lane; its nb columns, 16 at a time
    const int row = 32 * warp + lane;
    const uint32_t lanes = uint32_t(32 * warp) << 16;
    const int64_t o = row < nf ? int64_t(sdest ? sdest[os + row] : os + row) : -1;
    for (int c = 0; c < nb; c += 16) {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
          "%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
            "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(tmem + lanes + uint32_t(c)));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (o >= 0)
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = c + j, comp = col >= nd ? 1 : 0, m = col - comp * nd;
          sover[2 * (size_t(o) * nd + m) + comp] = __uint_as_float(v[j]);
        }
    }
  } else {
    if (tid == 0 && err) atomicExch(err, 1 + p);
    for (int r = 0; r < 4; ++r)
      if (wait_phase(&bar, 0u)) break;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

std::atomic<int> g_os_engine{-1};

}  // namespace

int oversample_engine() {
  int e = g_os_engine.load();
  if (e < 0) {
    const char* s = std::getenv("BIE_OVERSAMPLE_ENGINE");
    e = (s && s[0] == '1') ? 1 : 0;
    g_os_engine.store(e);
  }
  return e;
}

void set_oversample_engine(int engine) { g_os_engine.store(engine ? 1 : 0); }

bool oversample_tc_fits(const Geometry& g, const KParams& kp, int precision, int nd) {
  return kp.kind == 1 && precision == 1 && nd % 8 == 0 && nd >= 8 && nd <= 128 &&
         g.max_nf <= kOsRows && g.max_np <= 64 && g.npatches > 0;
}

cudaError_t launch_oversample_tc(const Geometry& g, const KParams& kp, const MatvecArgs& a,
                                 cudaStream_t st) {
  if (!oversample_tc_fits(g, kp, a.precision, a.nd)) return cudaErrorNotSupported;
  const int nd = a.nd, nb = 2 * nd;
  const int kpad = ((g.max_np + 7) / 8) * 8;
  uint32_t ncols = 32;
  while (ncols < uint32_t(nb)) ncols <<= 1;
  // shared memory: the split operands, and at least enough that the CTAs an
  // SM can hold together never ask for more than its 512 tensor-memory
  // columns
  const size_t need = sizeof(float) * (2 * size_t(kOsRows) * kpad + 2 * size_t(nb) * kpad) + 1024;
  const size_t floor_smem = (size_t(227) * 1024 * ncols + 511) / 512 + 1024;
  const size_t smem = need > floor_smem ? need : floor_smem;
  if (smem > size_t(227) * 1024) return cudaErrorNotSupported;
  cudaError_t e = cudaFuncSetAttribute(oversample_tc_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  oversample_tc_kernel<<<unsigned(g.npatches), kOsThreads, smem, st>>>(
      g, a.sigma, static_cast<float*>(a.strengths), nd, kpad, ncols, a.sdest, a.tc_err);
  note_launches(1);
  return cudaGetLastError();
}

}  // namespace dev
}  // namespace bie
