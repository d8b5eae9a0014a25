// Matvec and GMRES kernels for the combined-field layer potentials (sm_100a).
//
// Stages of one matvec (lap_comb_dir_eval_addsub, lap_comb_dir.f90:806-1178;
// helm_comb_dir_eval_addsub, helm_comb_dir.f:856-1210):
//   (a) strengths : per patch, sigma_over = imat * sigma_patch
//                   (oversample_fun_guru, surf_routs.f90:511-591), scaled to
//                   charge alpha*w/(4pi) and dipole beta*w/(4pi) strengths;
//   (b) far       : direct sum over all oversampled sources for every
//                   target, skipping r^2 < thresh^2 (stands in for
//                   lfmm3d / hfmm3d, including their self-interaction rule);
//   (c) combine   : pot_i = sum of far partials + sum_k W_eff(k) . sigma,
//                   W_eff = wnear - smooth near part (folded once per plan,
//                   replacing the per-call l3ddirectcdp/h3ddirectcdp subtraction).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <type_traits>
#include <cmath>

#include "device.cuh"

#include "pair.cuh"
#include "trig_table.cuh"

namespace bie {
namespace dev {

namespace {

std::atomic<int64_t> g_launches{0};
inline void count(int64_t n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

constexpr double kOver4Pi = 0.07957747154594767;

// ---------------------------------------------------------------------------
// (a) strengths
// ---------------------------------------------------------------------------
template <typename R, int CPLX>
__device__ __forceinline__ void strengths_body(const Geometry& g, const KParams& kp,
                                               const double* __restrict__ sigma,
                                               R* __restrict__ str, int nd, int p, double* sh,
                                               const int32_t* __restrict__ sdest = nullptr) {
  const int ps = g.pstart[p], np = g.pstart[p + 1] - ps;
  const int os = g.ostart[p], nf = g.ostart[p + 1] - os;
  const double* M = g.imat + g.cmoff[g.pclass[p]];
  const int vals = np * nd * (CPLX ? 2 : 1);
  for (int q = threadIdx.x; q < vals; q += blockDim.x) sh[q] = sigma[size_t(ps) * nd * (CPLX ? 2 : 1) + q];
  __syncthreads();
  for (int q = threadIdx.x; q < nf * nd; q += blockDim.x) {
    const int l = q / nd, m = q - l * nd;
    const double* row = M + size_t(l) * np;
    double sr = 0, si = 0;
    if (CPLX) {
      for (int j = 0; j < np; ++j) {
        const double mv = row[j];
        sr = fma(mv, sh[2 * (j * nd + m)], sr);
        si = fma(mv, sh[2 * (j * nd + m) + 1], si);
      }
    } else {
      for (int j = 0; j < np; ++j) sr = fma(row[j], sh[j * nd + m], sr);
    }
    const double f = g.sw[os + l] * kOver4Pi;
    // sdest: the hierarchical far field keeps its sources in tree order
    const size_t o = size_t(sdest ? sdest[os + l] : os + l) * nd + m;
    if (CPLX) {
      // c = alpha * sigma_over * f, d = beta * sigma_over * f
      str[4 * o + 0] = R((kp.ar * sr - kp.ai * si) * f);
      str[4 * o + 1] = R((kp.ar * si + kp.ai * sr) * f);
      str[4 * o + 2] = R((kp.br * sr - kp.bi * si) * f);
      str[4 * o + 3] = R((kp.br * si + kp.bi * sr) * f);
    } else {
      str[2 * o + 0] = R(kp.ar * sr * f);
      str[2 * o + 1] = R(kp.br * sr * f);
    }
  }
}

template <typename R, int CPLX>
__global__ void strengths_kernel(Geometry g, KParams kp, const double* __restrict__ sigma,
                                 R* __restrict__ str, int nd, const int32_t* __restrict__ sdest) {
  extern __shared__ double sh[];
  strengths_body<R, CPLX>(g, kp, sigma, str, nd, blockIdx.x, sh, sdest);
}

// ---------------------------------------------------------------------------
// (b) far field: tiled direct N-body
// ---------------------------------------------------------------------------
// One block's work of the far field: target block bx (NT*TPT targets),
// source chunk by (chunk_len sources), density bz.  Shared tiles and the
// FP64 trig table come from the calling kernel.
template <int KIND, typename R, int NT, int TPT, int TILE, bool CK>
__device__ __forceinline__ void far_block(const Geometry& g, const KParams& kp,
                                          const R* __restrict__ str, double* __restrict__ partial,
                                          int64_t chunk_len, int nd, int64_t bx, int64_t by, int bz,
                                          const double2* tab, typename Vec<R>::T4* sg0,
                                          typename Vec<R>::T2* sg1, R* sst) {
  using R2 = typename Vec<R>::T2;
  using R4 = typename Vec<R>::T4;
  constexpr int SW = (KIND == 1) ? 4 : 2;  // strength reals per source
  const int64_t ntarg = g.ntarg, nptso = g.nptso;
  const int64_t tbase = int64_t(bx) * NT * TPT;
  const int m = bz;  // density index
  // FP32: coordinates are shifted by the block's first target so that nearby
  // pairs keep their relative accuracy in single precision.  FP64 keeps the
  // absolute coordinates: t - s of two nearby points is then exact, which the
  // double-layer numerator n.(t - s) = O(r^2) of a close pair needs (a shift
  // would leave t - s with rounding of the shifted magnitudes, up to 5e-10 of
  // n.(t - s) on a curved surface).
  const int64_t tc = tbase < ntarg ? tbase : ntarg - 1;
  constexpr bool kShift = sizeof(R) == 4;
  const double cx = kShift ? g.tx[tc] : 0.0, cy = kShift ? g.ty[tc] : 0.0,
               cz = kShift ? g.tz[tc] : 0.0;
  R tx[TPT], ty[TPT], tz[TPT];
  double accr[TPT], acci[TPT];
#pragma unroll
  for (int t = 0; t < TPT; ++t) {
    const int64_t it = tbase + threadIdx.x + int64_t(t) * NT;
    const int64_t ic = it < ntarg ? it : ntarg - 1;
    tx[t] = R(g.tx[ic] - cx);
    ty[t] = R(g.ty[ic] - cy);
    tz[t] = R(g.tz[ic] - cz);
    accr[t] = 0.0;
    acci[t] = 0.0;
  }
  const R thr2 = R(kp.thresh * kp.thresh);
  const R k = R(kp.kr), kim = R(kp.ki);
  // bounding box of this block's targets: the box of the kFarBlockTargets32
  // block that contains them (the block itself in FP32; FP64 blocks of 256 or
  // fewer targets lie inside one, which only makes the test conservative)
  double tbx[6] = {0, 0, 0, 0, 0, 0};
  const bool boxes = (sizeof(R) == 4 ? NT * TPT == kFarBlockTargets32
                                     : kFarBlockTargets32 % (NT * TPT) == 0) &&
                     g.sbox && g.tbox && TILE == kFarTileSources;
  if (boxes)
#pragma unroll
    for (int c = 0; c < 6; ++c) tbx[c] = g.tbox[6 * (tbase / kFarBlockTargets32) + c];
  const int64_t s0 = int64_t(by) * chunk_len;
  const int64_t s1 = min(s0 + chunk_len, nptso);
  for (int64_t sb = s0; sb < s1; sb += TILE) {
    const int ns = int((s1 - sb) < TILE ? (s1 - sb) : TILE);
    __syncthreads();
    for (int q = threadIdx.x; q < TILE; q += NT) {
      if (q < ns) {
        const int64_t s = sb + q;
        sg0[q] = R4{R(g.sx[s] - cx), R(g.sy[s] - cy), R(g.sz[s] - cz), R(g.snx[s])};
        sg1[q] = R2{R(g.sny[s]), R(g.snz[s])};
#pragma unroll
        for (int c = 0; c < SW; ++c) sst[q * SW + c] = str[(size_t(s) * nd + m) * SW + c];
      } else {
        sg0[q] = R4{R(0), R(0), R(0), R(0)};
        sg1[q] = R2{R(0), R(0)};
#pragma unroll
        for (int c = 0; c < SW; ++c) sst[q * SW + c] = R(0);
      }
    }
    __syncthreads();
    R pr[TPT], pi[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) pr[t] = pi[t] = R(0);
    // A full tile whose bounding box stays farther than the margin from the
    // block's targets cannot hold an excluded pair, so it skips the test.
    // A partial tile keeps it: its zero padding sits at the block centre,
    // which is the block's first target.
    bool check = true;
    if (boxes && ns == TILE) {
      const double* sbx = g.sbox + 6 * (sb / kFarTileSources);
      double gap2 = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double gap = fmax(fmax(sbx[c] - tbx[c + 3], tbx[c] - sbx[c + 3]), 0.0);
        gap2 += gap * gap;
      }
      check = gap2 <= g.box_margin2;
    }
    if (check) {
#pragma unroll 4
      for (int j = 0; j < TILE; ++j) {
        const R4 a = sg0[j];
        const R2 b = sg1[j];
        if constexpr (KIND == 1) {
          const R4 s = reinterpret_cast<const R4*>(sst)[j];
#pragma unroll
          for (int t = 0; t < TPT; ++t)
            pair_helm(tx[t], ty[t], tz[t], a, b, s, k, kim, thr2, CK, pr[t], pi[t], tab);
        } else {
          const R2 s = reinterpret_cast<const R2*>(sst)[j];
#pragma unroll
          for (int t = 0; t < TPT; ++t) pair_lap<R>(tx[t], ty[t], tz[t], a, b, s, thr2, pr[t]);
        }
      }
    } else {
#pragma unroll 4
      for (int j = 0; j < TILE; ++j) {
        const R4 a = sg0[j];
        const R2 b = sg1[j];
        if constexpr (KIND == 1) {
          const R4 s = reinterpret_cast<const R4*>(sst)[j];
#pragma unroll
          for (int t = 0; t < TPT; ++t)
            pair_helm<false>(tx[t], ty[t], tz[t], a, b, s, k, kim, thr2, CK, pr[t], pi[t], tab);
        } else {
          const R2 s = reinterpret_cast<const R2*>(sst)[j];
#pragma unroll
          for (int t = 0; t < TPT; ++t) pair_lap<R, false>(tx[t], ty[t], tz[t], a, b, s, thr2, pr[t]);
        }
      }
    }
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
      accr[t] += double(pr[t]);
      acci[t] += double(pi[t]);
    }
  }
#pragma unroll
  for (int t = 0; t < TPT; ++t) {
    const int64_t it = tbase + threadIdx.x + int64_t(t) * NT;
    if (it >= ntarg) continue;
    const size_t o = (size_t(by) * ntarg + it) * nd + m;
    if (KIND == 1) {
      partial[2 * o] = accr[t];
      partial[2 * o + 1] = acci[t];
    } else {
      partial[o] = accr[t];
    }
  }
}


// FP32 far field with two targets per packed instruction (pair_helm_x2,
// pair_lap_x2): the work, the coordinate shift, the tile boxes and the
// threshold test of far_block<float>, with the source tile in shared memory
// holding every value twice (kFarX2Words float4 per source, source-major, so
// the threads of a warp read one source as a broadcast).
template <int KIND>
constexpr int kFarX2Words = KIND == 1 ? 6 : 4;
constexpr int kFarUnroll = 4;  // sources per loop body (1: +5 %, 2: +1 %, 8: +4 % time)

template <int KIND, int NT, int TPT, int TILE, bool CK>
__device__ __forceinline__ void far_block_x2(const Geometry& g, const KParams& kp,
                                             const float* __restrict__ str,
                                             double* __restrict__ partial, int64_t chunk_len,
                                             int nd, int64_t bx, int64_t by, int bz,
                                             float4* tile) {
  static_assert(TPT % 2 == 0, "targets are taken in pairs");
  constexpr int SW = (KIND == 1) ? 4 : 2;  // strength reals per source
  constexpr int W = kFarX2Words<KIND>;
  constexpr int TP = TPT / 2;  // target pairs per thread
  const int64_t ntarg = g.ntarg, nptso = g.nptso;
  const int64_t tbase = int64_t(bx) * NT * TPT;
  const int m = bz;
  const int64_t tc = tbase < ntarg ? tbase : ntarg - 1;
  const double cx = g.tx[tc], cy = g.ty[tc], cz = g.tz[tc];
  float2 tx[TP], ty[TP], tz[TP];
  double accr[TPT], acci[TPT];
#pragma unroll
  for (int t = 0; t < TPT; ++t) {
    const int64_t it = tbase + threadIdx.x + int64_t(t) * NT;
    const int64_t ic = it < ntarg ? it : ntarg - 1;
    const float x = float(g.tx[ic] - cx), y = float(g.ty[ic] - cy), z = float(g.tz[ic] - cz);
    if (t % 2 == 0) {
      tx[t / 2].x = x;
      ty[t / 2].x = y;
      tz[t / 2].x = z;
    } else {
      tx[t / 2].y = x;
      ty[t / 2].y = y;
      tz[t / 2].y = z;
    }
    accr[t] = 0.0;
    acci[t] = 0.0;
  }
  const float thr2 = float(kp.thresh * kp.thresh);
  const float2 k2 = make_float2(float(kp.kr), float(kp.kr)),
               kim2 = make_float2(float(kp.ki), float(kp.ki));
  double tbx[6] = {0, 0, 0, 0, 0, 0};
  const bool boxes = NT * TPT == kFarBlockTargets32 && g.sbox && g.tbox && TILE == kFarTileSources;
  if (boxes)
#pragma unroll
    for (int c = 0; c < 6; ++c) tbx[c] = g.tbox[6 * (tbase / kFarBlockTargets32) + c];
  const int64_t s0 = int64_t(by) * chunk_len;
  const int64_t s1 = min(s0 + chunk_len, nptso);
  for (int64_t sb = s0; sb < s1; sb += TILE) {
    const int ns = int((s1 - sb) < TILE ? (s1 - sb) : TILE);
    __syncthreads();
    for (int q = threadIdx.x; q < TILE; q += NT) {
      float4* T = tile + q * W;
      if (q < ns) {
        const int64_t s = sb + q;
        const float x = -float(g.sx[s] - cx), y = -float(g.sy[s] - cy), z = -float(g.sz[s] - cz);
        const float nx = float(g.snx[s]), ny = float(g.sny[s]), nz = float(g.snz[s]);
        T[0] = make_float4(x, x, y, y);
        T[1] = make_float4(z, z, nx, nx);
        T[2] = make_float4(ny, ny, nz, nz);
        const float* st = str + (size_t(s) * nd + m) * SW;
        if constexpr (KIND == 1) {
          const float4 v = *reinterpret_cast<const float4*>(st);
          T[3] = make_float4(v.x, v.x, v.y, v.y);
          T[4] = make_float4(v.z, v.z, v.w, v.w);
          T[5] = make_float4(-v.z, -v.z, 0.f, 0.f);
        } else {
          T[3] = make_float4(st[0], st[0], st[1], st[1]);
        }
      } else {
#pragma unroll
        for (int w = 0; w < W; ++w) T[w] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    __syncthreads();
    float2 pa[TP], pb[TP], pi[TP];
#pragma unroll
    for (int t = 0; t < TP; ++t) pa[t] = pb[t] = pi[t] = make_float2(0.f, 0.f);
    bool check = true;
    if (boxes && ns == TILE) {
      const double* sbx = g.sbox + 6 * (sb / kFarTileSources);
      double gap2 = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double gap = fmax(fmax(sbx[c] - tbx[c + 3], tbx[c] - sbx[c + 3]), 0.0);
        gap2 += gap * gap;
      }
      check = gap2 <= g.box_margin2;
    }
    auto sweep = [&](auto chk) {
      constexpr bool C = decltype(chk)::value;
#pragma unroll(kFarUnroll)
      for (int j = 0; j < TILE; ++j) {
        const float4* T = tile + j * W;
        const float4 q0 = T[0], q1 = T[1], q2 = T[2], q3 = T[3];
        const float2 msx = make_float2(q0.x, q0.y), msy = make_float2(q0.z, q0.w),
                     msz = make_float2(q1.x, q1.y), nx = make_float2(q1.z, q1.w),
                     ny = make_float2(q2.x, q2.y), nz = make_float2(q2.z, q2.w);
        if constexpr (KIND == 1) {
          const float4 q4 = T[4];
          const float2 q5 = *reinterpret_cast<const float2*>(T + 5);
          const float2 cr = make_float2(q3.x, q3.y), ci = make_float2(q3.z, q3.w),
                       dr = make_float2(q4.x, q4.y), di = make_float2(q4.z, q4.w);
#pragma unroll
          for (int t = 0; t < TP; ++t)
            pair_helm_x2<C>(tx[t], ty[t], tz[t], msx, msy, msz, nx, ny, nz, cr, ci, dr, di, q5, k2,
                            kim2, thr2, CK, pa[t], pb[t], pi[t]);
        } else {
          const float2 c = make_float2(q3.x, q3.y), d = make_float2(q3.z, q3.w);
#pragma unroll
          for (int t = 0; t < TP; ++t)
            pair_lap_x2<C>(tx[t], ty[t], tz[t], msx, msy, msz, nx, ny, nz, c, d, thr2, pa[t]);
        }
      }
    };
    if (check)
      sweep(std::true_type{});
    else
      sweep(std::false_type{});
#pragma unroll
    for (int t = 0; t < TP; ++t) {
      accr[2 * t] += double(pa[t].x) - double(pb[t].x);
      accr[2 * t + 1] += double(pa[t].y) - double(pb[t].y);
      acci[2 * t] += double(pi[t].x);
      acci[2 * t + 1] += double(pi[t].y);
    }
  }
#pragma unroll
  for (int t = 0; t < TPT; ++t) {
    const int64_t it = tbase + threadIdx.x + int64_t(t) * NT;
    if (it >= ntarg) continue;
    const size_t o = (size_t(by) * ntarg + it) * nd + m;
    if (KIND == 1) {
      partial[2 * o] = accr[t];
      partial[2 * o + 1] = acci[t];
    } else {
      partial[o] = accr[t];
    }
  }
}


// Blocks per SM the 128-thread shapes are compiled for.  FP32: a register
// budget of 96 (5 blocks, 20 warps per SM) measured 2 % faster on the
// 35,840-node Helmholtz matvec than the unconstrained 123 registers (4
// blocks), with no spills; 80 and 64 registers measured no faster.  FP64: 128
// registers (4 blocks) measured 2 % faster than the unconstrained 146 (3
// blocks).
template <typename R, int NT>
constexpr int kFarMinBlocks = NT == 128 ? (sizeof(R) == 4 ? 5 : 4) : 1;

template <int KIND, typename R, int NT, int TPT, int TILE, bool CK>
__global__ void __launch_bounds__(NT, (kFarMinBlocks<R, NT>)) far_kernel(Geometry g, KParams kp, const R* __restrict__ str,
                                                 double* __restrict__ partial, int64_t chunk_len,
                                                 int nd) {
  constexpr int SW = (KIND == 1) ? 4 : 2;
  if constexpr (sizeof(R) == 4) {
    __shared__ float4 tile[TILE * kFarX2Words<KIND>];
    far_block_x2<KIND, NT, TPT, TILE, CK>(g, kp, str, partial, chunk_len, nd, blockIdx.x,
                                          blockIdx.y, blockIdx.z, tile);
  } else {
    __shared__ typename Vec<R>::T4 sg0[TILE];
    __shared__ typename Vec<R>::T2 sg1[TILE];
    __shared__ R sst[TILE * SW];
    __shared__ double2 stab[KIND == 1 ? kFarTrigN : 1];
    const double2* tab = nullptr;
    if constexpr (KIND == 1) {
      fill_far_trig_table(stab);  // published by the first __syncthreads of the tile loop
      tab = stab;
    }
    far_block<KIND, R, NT, TPT, TILE, CK>(g, kp, str, partial, chunk_len, nd, blockIdx.x,
                                          blockIdx.y, blockIdx.z, tab, sg0, sg1, sst);
  }
}

// ---------------------------------------------------------------------------
// (b') far field for several densities at once.
//
// Charge and dipole strengths of a layer potential are both proportional to
// the same oversampled density, so each pair's kernel value
//   K(t,s) = a_s G(t,s) + b_s dG/dn_s(t,s),  a_s = alpha w_s/(4pi), b_s = beta w_s/(4pi)
// is computed once (the single-density pair function with unit density) and
// applied to MD densities with one complex multiply-add each.  Coordinates
// are centred on the first target of the enclosing 512-target block, as in
// the single-density FP32 kernel, so the FP32 error-matched fold applies.
// ab: per source (a, b) (complex: 4 reals, real: 2); sig: sigma_over[s][nd].
// ---------------------------------------------------------------------------
constexpr int kMdCentre = 512;

// FP32 Helmholtz blocks of up to 8 densities stage each density as
// (re, im, im, re) for the packed complex multiply-add (4 densities: 4 %
// faster than the scalar form on the 35,840-node matvec); with 16 densities
// that layout and its registers measured 20 % slower, so those stay scalar.
template <int KIND, typename R, int MD>
constexpr bool kMdPacked = sizeof(R) == 4 && KIND == 1 && MD <= 8;
template <int KIND, typename R, int MD>
constexpr int kMdSigWords = kMdPacked<KIND, R, MD> ? 4 : (KIND == 1 ? 2 : 1);


// One block's work of the multi-density far field: target block bx, source
// chunk by, density group bz (MD densities).  Shared tiles and the FP64 trig
// table come from the calling kernel.
template <int KIND, typename R, int NT, int TPT, int MD, int TILE, bool CK>
__device__ __forceinline__ void far_md_block(const Geometry& g, const KParams& kp,
                                             const R* __restrict__ ab, const R* __restrict__ sig,
                                             int nd, double* __restrict__ partial,
                                             int64_t chunk_len, int64_t bx, int64_t by, int bz,
                                             const double2* tab, typename Vec<R>::T4* sg0,
                                             typename Vec<R>::T2* sg1, R* sab, R* ssig) {
  using R2 = typename Vec<R>::T2;
  using R4 = typename Vec<R>::T4;
  constexpr int C = (KIND == 1) ? 2 : 1;  // reals per complex value
  static_assert(MD % 2 == 0, "densities are read from shared memory two at a time");
  const int64_t ntarg = g.ntarg, nptso = g.nptso;
  const int64_t tbase = int64_t(bx) * NT * TPT;
  const int m0 = bz * MD;
  const int64_t tcen = (tbase / kMdCentre) * kMdCentre;
  const int64_t tc = tcen < ntarg ? tcen : ntarg - 1;
  // shifted coordinates in FP32 only (see far_block)
  constexpr bool kShift = sizeof(R) == 4;
  const double cx = kShift ? g.tx[tc] : 0.0, cy = kShift ? g.ty[tc] : 0.0,
               cz = kShift ? g.tz[tc] : 0.0;
  R tx[TPT], ty[TPT], tz[TPT];
  double acc[TPT][MD][C];
#pragma unroll
  for (int t = 0; t < TPT; ++t) {
    const int64_t it = tbase + threadIdx.x + int64_t(t) * NT;
    const int64_t ic = it < ntarg ? it : ntarg - 1;
    tx[t] = R(g.tx[ic] - cx);
    ty[t] = R(g.ty[ic] - cy);
    tz[t] = R(g.tz[ic] - cz);
#pragma unroll
    for (int m = 0; m < MD; ++m)
#pragma unroll
      for (int c = 0; c < C; ++c) acc[t][m][c] = 0.0;
  }
  const R thr2 = R(kp.thresh * kp.thresh);
  const R k = R(kp.kr), kim = R(kp.ki);
  const int64_t s0 = int64_t(by) * chunk_len;
  const int64_t s1 = min(s0 + chunk_len, nptso);
  for (int64_t sb = s0; sb < s1; sb += TILE) {
    const int ns = int((s1 - sb) < TILE ? (s1 - sb) : TILE);
    __syncthreads();
    for (int q = threadIdx.x; q < TILE; q += NT) {
      const bool ok = q < ns;
      const int64_t s = sb + q;
      sg0[q] = ok ? R4{R(g.sx[s] - cx), R(g.sy[s] - cy), R(g.sz[s] - cz), R(g.snx[s])}
                  : R4{R(0), R(0), R(0), R(0)};
      sg1[q] = ok ? R2{R(g.sny[s]), R(g.snz[s])} : R2{R(0), R(0)};
#pragma unroll
      for (int c = 0; c < 2 * C; ++c) sab[q * 2 * C + c] = ok ? ab[size_t(s) * 2 * C + c] : R(0);
    }
    for (int q = threadIdx.x; q < TILE * MD; q += NT) {
      const int qs = q / MD, mm = q - qs * MD;
      const bool ok = qs < ns && m0 + mm < nd;
      if constexpr (kMdPacked<KIND, R, MD>) {
        // (re, im, im, re): the density and its swapped copy for the packed
        // complex multiply-add
        const R xr = ok ? sig[(size_t(sb + qs) * nd + m0 + mm) * 2] : R(0);
        const R xi = ok ? sig[(size_t(sb + qs) * nd + m0 + mm) * 2 + 1] : R(0);
        reinterpret_cast<float4*>(ssig)[q] = make_float4(xr, xi, xi, xr);
      } else {
#pragma unroll
        for (int c = 0; c < C; ++c)
          ssig[q * C + c] = ok ? sig[(size_t(sb + qs) * nd + m0 + mm) * C + c] : R(0);
      }
    }
    __syncthreads();
    if constexpr (kMdPacked<KIND, R, MD>) {
      // FP32 Helmholtz, up to 8 densities per block: each density's complex
      // multiply-add as two packed lanes (re, im): acc += (K_r, K_r) (x_r, x_i)
      // after (-K_i, K_i) (x_i, x_r), each lane rounded as the scalar form in
      // the scalar form's order.
      float2 tr2[TPT][MD];
#pragma unroll
      for (int t = 0; t < TPT; ++t)
#pragma unroll
        for (int m = 0; m < MD; ++m) tr2[t][m] = make_float2(0.f, 0.f);
#pragma unroll 2
      for (int j = 0; j < TILE; ++j) {
        const R4 a = sg0[j];
        const R2 b = sg1[j];
        const R4 sv4 = reinterpret_cast<const R4*>(sab)[j];
        const float4* sv = reinterpret_cast<const float4*>(ssig) + j * MD;
#pragma unroll
        for (int t = 0; t < TPT; ++t) {
          float kr_ = 0.f, ki_ = 0.f;
          pair_helm(tx[t], ty[t], tz[t], a, b, sv4, k, kim, thr2, CK, kr_, ki_, tab);
          const float2 kk = make_float2(kr_, kr_), kn = make_float2(-ki_, ki_);
#pragma unroll
          for (int m = 0; m < MD; ++m) {
            const float4 x = sv[m];
            tr2[t][m] = __ffma2_rn(kk, make_float2(x.x, x.y),
                                   __ffma2_rn(kn, make_float2(x.z, x.w), tr2[t][m]));
          }
        }
      }
#pragma unroll
      for (int t = 0; t < TPT; ++t)
#pragma unroll
        for (int m = 0; m < MD; ++m) {
          acc[t][m][0] += double(tr2[t][m].x);
          acc[t][m][C - 1] += double(tr2[t][m].y);
        }
    } else if constexpr (sizeof(R) == 4 && KIND == 0) {
      // FP32 Laplace: two densities per packed multiply-add (fma.rn.f32x2,
      // each lane rounded as the scalar form).
      constexpr int NP = MD / 2;
      float2 tr2[TPT][NP];
#pragma unroll
      for (int t = 0; t < TPT; ++t)
#pragma unroll
        for (int m = 0; m < NP; ++m) tr2[t][m] = make_float2(0.f, 0.f);
#pragma unroll 2
      for (int j = 0; j < TILE; ++j) {
        const R4 a = sg0[j];
        const R2 b = sg1[j];
        const R2 sv2 = reinterpret_cast<const R2*>(sab)[j];
        const float2* sv = reinterpret_cast<const float2*>(ssig + j * MD);
#pragma unroll
        for (int t = 0; t < TPT; ++t) {
          float kv = 0.f;
          pair_lap<R>(tx[t], ty[t], tz[t], a, b, sv2, thr2, kv);
          const float2 kk = make_float2(kv, kv);
#pragma unroll
          for (int m = 0; m < NP; ++m) tr2[t][m] = __ffma2_rn(kk, sv[m], tr2[t][m]);
        }
      }
#pragma unroll
      for (int t = 0; t < TPT; ++t)
#pragma unroll
        for (int m = 0; m < NP; ++m) {
          acc[t][2 * m][0] += double(tr2[t][m].x);
          acc[t][2 * m + 1][0] += double(tr2[t][m].y);
        }
    } else {
      // FP32: tile sums in FP32, added to the FP64 sums after each tile;
      // FP64: straight into the FP64 sums (a second set of FP64 tile sums
      // would only cost registers)
      constexpr bool kTileSums = sizeof(R) == 4;
      R tr[kTileSums ? TPT : 1][kTileSums ? MD : 1][C];
      auto T = [&](int t, int m, int c) -> R& {
        if constexpr (kTileSums)
          return tr[t][m][c];
        else
          return reinterpret_cast<R&>(acc[t][m][c]);
      };
      if constexpr (kTileSums) {
#pragma unroll
        for (int t = 0; t < TPT; ++t)
#pragma unroll
          for (int m = 0; m < MD; ++m)
#pragma unroll
            for (int c = 0; c < C; ++c) tr[t][m][c] = R(0);
      }
#pragma unroll 2
      for (int j = 0; j < TILE; ++j) {
        const R4 a = sg0[j];
        const R2 b = sg1[j];
        if constexpr (KIND == 1) {
          const R4 s = reinterpret_cast<const R4*>(sab)[j];
#pragma unroll
          for (int t = 0; t < TPT; ++t) {
            R kr_ = R(0), ki_ = R(0);
            pair_helm(tx[t], ty[t], tz[t], a, b, s, k, kim, thr2, CK, kr_, ki_, tab);
            const R4* sv = reinterpret_cast<const R4*>(ssig) + j * (MD / 2);
#pragma unroll
            for (int m2 = 0; m2 < MD / 2; ++m2) {
              const R4 x = sv[m2];  // densities 2*m2 and 2*m2+1
              T(t, 2 * m2, 0) = fma(kr_, x.x, fma(-ki_, x.y, T(t, 2 * m2, 0)));
              T(t, 2 * m2, 1) = fma(kr_, x.y, fma(ki_, x.x, T(t, 2 * m2, 1)));
              T(t, 2 * m2 + 1, 0) = fma(kr_, x.z, fma(-ki_, x.w, T(t, 2 * m2 + 1, 0)));
              T(t, 2 * m2 + 1, 1) = fma(kr_, x.w, fma(ki_, x.z, T(t, 2 * m2 + 1, 1)));
            }
          }
        } else {
          const R2 s = reinterpret_cast<const R2*>(sab)[j];
#pragma unroll
          for (int t = 0; t < TPT; ++t) {
            R kv = R(0);
            pair_lap<R>(tx[t], ty[t], tz[t], a, b, s, thr2, kv);
            const R* sv = ssig + j * MD;
#pragma unroll
            for (int m = 0; m < MD; ++m) T(t, m, 0) = fma(kv, sv[m], T(t, m, 0));
          }
        }
      }
      if constexpr (kTileSums) {
#pragma unroll
        for (int t = 0; t < TPT; ++t)
#pragma unroll
          for (int m = 0; m < MD; ++m)
#pragma unroll
            for (int c = 0; c < C; ++c) acc[t][m][c] += double(tr[t][m][c]);
      }
    }
  }
#pragma unroll
  for (int t = 0; t < TPT; ++t) {
    const int64_t it = tbase + threadIdx.x + int64_t(t) * NT;
    if (it >= ntarg) continue;
#pragma unroll
    for (int m = 0; m < MD; ++m) {
      if (m0 + m >= nd) continue;
      const size_t o = (size_t(by) * ntarg + it) * nd + m0 + m;
#pragma unroll
      for (int c = 0; c < C; ++c) partial[C * o + c] = acc[t][m][c];
    }
  }
}

template <int KIND, typename R, int NT, int TPT, int MD, int TILE, bool CK>
__global__ void __launch_bounds__(NT) far_md_kernel(Geometry g, KParams kp,
                                                    const R* __restrict__ ab,
                                                    const R* __restrict__ sig, int nd,
                                                    double* __restrict__ partial,
                                                    int64_t chunk_len) {
  constexpr int C = (KIND == 1) ? 2 : 1;
  __shared__ typename Vec<R>::T4 sg0[TILE];
  __shared__ typename Vec<R>::T2 sg1[TILE];
  __shared__ __align__(16) R sab[TILE * 2 * C];
  __shared__ __align__(16) R ssig[TILE * MD * kMdSigWords<KIND, R, MD>];
  __shared__ double2 stab[sizeof(R) == 8 && KIND == 1 ? kFarTrigN : 1];
  const double2* tab = nullptr;
  if constexpr (sizeof(R) == 8 && KIND == 1) {
    fill_far_trig_table(stab);  // published by the first __syncthreads of the tile loop
    tab = stab;
  }
  far_md_block<KIND, R, NT, TPT, MD, TILE, CK>(g, kp, ab, sig, nd, partial, chunk_len, blockIdx.x,
                                               blockIdx.y, blockIdx.z, tab, sg0, sg1, sab, ssig);
}

// sigma_over[s][m] = (imat sigma_patch)[s][m] without scaling (several
// densities); feeds far_md_kernel.
template <typename R, int CPLX>
__device__ __forceinline__ void oversample_body(const Geometry& g, const double* __restrict__ sigma,
                                                R* __restrict__ sover, int nd, int p, double* sh,
                                                const int32_t* __restrict__ sdest = nullptr) {
  const int ps = g.pstart[p], np = g.pstart[p + 1] - ps;
  const int os = g.ostart[p], nf = g.ostart[p + 1] - os;
  const double* M = g.imat + g.cmoff[g.pclass[p]];
  const int C = CPLX ? 2 : 1;
  for (int q = threadIdx.x; q < np * nd * C; q += blockDim.x) sh[q] = sigma[size_t(ps) * nd * C + q];
  __syncthreads();
  for (int q = threadIdx.x; q < nf * nd; q += blockDim.x) {
    const int l = q / nd, m = q - l * nd;
    const double* row = M + size_t(l) * np;
    double sr = 0, si = 0;
    for (int j = 0; j < np; ++j) {
      const double mv = row[j];
      sr = fma(mv, sh[C * (j * nd + m)], sr);
      if (CPLX) si = fma(mv, sh[C * (j * nd + m) + 1], si);
    }
    const size_t o = size_t(sdest ? sdest[os + l] : os + l) * nd + m;
    sover[C * o] = R(sr);
    if (CPLX) sover[C * o + 1] = R(si);
  }
}

template <typename R, int CPLX>
__global__ void oversample_kernel(Geometry g, const double* __restrict__ sigma,
                                  R* __restrict__ sover, int nd, const int32_t* __restrict__ sdest) {
  extern __shared__ double sh[];
  oversample_body<R, CPLX>(g, sigma, sover, nd, blockIdx.x, sh, sdest);
}

// Per-source constants a_s = alpha w_s/(4pi), b_s = beta w_s/(4pi).
template <typename R, int CPLX>
__global__ void source_consts_kernel(Geometry g, KParams kp, R* __restrict__ ab,
                                     const int32_t* __restrict__ sdest) {
  for (int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < g.nptso;
       s += int64_t(gridDim.x) * blockDim.x) {
    const double f = g.sw[s] * kOver4Pi;
    const int64_t o = sdest ? int64_t(sdest[s]) : s;
    if (CPLX) {
      ab[4 * o + 0] = R(kp.ar * f);
      ab[4 * o + 1] = R(kp.ai * f);
      ab[4 * o + 2] = R(kp.br * f);
      ab[4 * o + 3] = R(kp.bi * f);
    } else {
      ab[2 * o + 0] = R(kp.ar * f);
      ab[2 * o + 1] = R(kp.br * f);
    }
  }
}

// ---------------------------------------------------------------------------
// (c) combine: far partials + near-correction SpMM, one warp per target row
// ---------------------------------------------------------------------------
template <typename W>
struct Vec2;
template <>
struct Vec2<float> {
  using T = float2;
};
template <>
struct Vec2<double> {
  using T = double2;
};

constexpr int kCombineThreads = 256;  // 8 warps = 8 consecutive target rows per block
constexpr int kCombineUnroll = 4;     // W_eff entries per lane in flight
// Blocks per SM the one-density form is compiled for (48 registers): 5 % faster
// on the 35,840-node matvec than 4 blocks (64 registers); 6 and 8 blocks, and
// 8 entries per lane in flight, measured slower.
constexpr int kCombineMinBlocks = 5;


// Rows 8*bx .. 8*bx+7 (one warp each) of the near correction plus the far
// partial sums.
// Near correction of row i for 2..8 densities.  A lane takes D = min(nd,
// KD) consecutive densities of one W_eff entry (the sigma values of a node's
// densities are contiguous); the warp's lanes are (entry slot, density
// group) pairs -- Q = the number of groups rounded up to a power of two
// groups side by side, G = 32 / Q entries of the row at a time -- and the
// slots are summed by shuffles at the end.  Near pairs are taken 32 at a
// time (one lane-parallel load of their first nodes and entry offsets);
// where all 32 have the same node count the row's entries run as one flat
// range, two entries per lane in flight.  nd = 4: 0.20 ms on the 35,840-node
// matvec against 0.63 ms with the lanes over densities (the wide form); at
// nd = 16 the same scheme with one density per lane measured 0.72 against
// 0.62 ms, so the wide form serves more than 8 densities.
template <int CPLX, typename W, int kD>
__device__ __forceinline__ void combine_row_md(const Geometry& g, const Near& nr,
                                               const W* __restrict__ weff,
                                               const double* __restrict__ sigma,
                                               const double* __restrict__ partial, int nchunks,
                                               double* __restrict__ pot, int nd, int64_t i,
                                               int lane) {
  const int64_t ntarg = g.ntarg;
  const int64_t k0 = nr.row_ptr[i], k1 = nr.row_ptr[i + 1];
  constexpr unsigned kFull = 0xffffffffu;
  const int D = nd < kD ? nd : kD;
  const int ngroups = (nd + D - 1) / D;
  int Q = 1;
  while (Q < ngroups && Q < 32) Q <<= 1;
  const int G = 32 / Q, ql = lane & (Q - 1), slot = lane / Q;
  for (int qb = 0; qb < ngroups; qb += Q) {
    const int m0 = (qb + ql) * D;
    const int dn = m0 < nd ? (nd - m0 < D ? nd - m0 : D) : 0;  // densities of this lane
    double ar[kD], ai[kD];
#pragma unroll
    for (int d = 0; d < kD; ++d) ar[d] = ai[d] = 0.0;
    // far-field partial sums, chunks spread over the entry slots
    if (dn > 0)
      for (int c = slot; c < nchunks; c += G) {
        const size_t o = (size_t(c) * ntarg + i) * nd + m0;
#pragma unroll
        for (int d = 0; d < kD; ++d)
          if (d < dn) {
            if (CPLX) {
              const double2 v = reinterpret_cast<const double2*>(partial)[o + d];
              ar[d] += v.x;
              ai[d] += v.y;
            } else {
              ar[d] += partial[o + d];
            }
          }
      }
    // one entry: weight w times the lane's densities of node
    auto entry = [&](int64_t we, int node) {
      const size_t so = size_t(node) * nd + m0;
      if (CPLX) {
        const typename Vec2<W>::T wv = reinterpret_cast<const typename Vec2<W>::T*>(weff)[we];
        const double wr = double(wv.x), wi = double(wv.y);
#pragma unroll
        for (int d = 0; d < kD; ++d)
          if (d < dn) {
            const double2 sv = reinterpret_cast<const double2*>(sigma)[so + d];
            ar[d] = fma(wr, sv.x, fma(-wi, sv.y, ar[d]));
            ai[d] = fma(wr, sv.y, fma(wi, sv.x, ai[d]));
          }
      } else {
        const double w = double(weff[we]);
#pragma unroll
        for (int d = 0; d < kD; ++d)
          if (d < dn) ar[d] = fma(w, sigma[so + d], ar[d]);
      }
    };
    for (int64_t kc = k0; kc < k1; kc += 32) {
      const int nkc = int(k1 - kc < 32 ? k1 - kc : 32);
      int psl = 0, npl = 0;
      int64_t wbl = 0;
      if (lane < nkc) {
        psl = nr.nps[kc + lane];
        wbl = nr.wofs[kc + lane];
        npl = int(nr.wofs[kc + lane + 1] - wbl);
      }
      const int np0 = __shfl_sync(kFull, npl, 0);
      const int64_t e0 = __shfl_sync(kFull, wbl, 0);
      if (__all_sync(kFull, lane >= nkc || npl == np0)) {
        // entry e of the group belongs to pair e / np0 (exact in FP32, as
        // in the one-density form)
        const int ne = nkc * np0;
        const float inv = 1.0f / float(np0);
        // (the same trip count on every lane: the shuffles need the whole warp)
        constexpr int U = 2;  // entries per lane in flight
        for (int eb = 0; eb < ne; eb += U * G) {
          int node[U], ee[U];
          bool ok[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int e = eb + u * G + slot;
            ee[u] = e;
            ok[u] = e < ne && dn > 0;
            const int kk = e < ne ? int((float(e) + 0.5f) * inv) : 0;
            const int psk = __shfl_sync(kFull, psl, kk);
            node[u] = psk + (e - kk * np0);
          }
#pragma unroll
          for (int u = 0; u < U; ++u)
            if (ok[u]) entry(e0 + ee[u], node[u]);
        }
      } else {
        for (int j = 0; j < nkc; ++j) {
          const int ps = __shfl_sync(kFull, psl, j), np = __shfl_sync(kFull, npl, j);
          const int64_t wb = __shfl_sync(kFull, wbl, j);
          if (dn == 0) continue;
          for (int mm = slot; mm < np; mm += G) entry(wb + mm, ps + mm);
        }
      }
    }
#pragma unroll
    for (int d = 0; d < kD; ++d)
      for (int off = Q; off < 32; off <<= 1) {
        ar[d] += __shfl_xor_sync(kFull, ar[d], off);
        if (CPLX) ai[d] += __shfl_xor_sync(kFull, ai[d], off);
      }
    if (slot == 0)
#pragma unroll
      for (int d = 0; d < kD; ++d)
        if (d < dn) {
          const size_t o = size_t(i) * nd + m0 + d;
          if (CPLX) {
            pot[2 * o] = ar[d];
            pot[2 * o + 1] = ai[d];
          } else {
            pot[o] = ar[d];
          }
        }
  }
}

// More than 8 densities: the lanes run over densities, every lane over the
// whole row (1.43 ms at nd = 64 on the 35,840-node matvec, where the slot
// forms measured 1.6-2.3 ms).
template <int CPLX, typename W>
__device__ __forceinline__ void combine_row_wide(const Geometry& g, const Near& nr,
                                                 const W* __restrict__ weff,
                                                 const double* __restrict__ sigma,
                                                 const double* __restrict__ partial,
                                                 int nchunks, double* __restrict__ pot, int nd,
                                                 int64_t i, int lane) {
  const int64_t ntarg = g.ntarg;
  const int64_t k0 = nr.row_ptr[i], k1 = nr.row_ptr[i + 1];
  for (int m = lane; m < nd; m += 32) {
    double ar = 0, ai = 0;
    for (int c = 0; c < nchunks; ++c) {
      const size_t o = (size_t(c) * ntarg + i) * nd + m;
      if (CPLX) {
        ar += partial[2 * o];
        ai += partial[2 * o + 1];
      } else {
        ar += partial[o];
      }
    }
    for (int64_t k = k0; k < k1; ++k) {
      const int p = nr.col[k];
      const int ps = g.pstart[p], np = g.pstart[p + 1] - ps;
      const int64_t wb = nr.wofs[k];
      for (int mm = 0; mm < np; ++mm) {
        const size_t so = size_t(ps + mm) * nd + m;
        if (CPLX) {
          const double wr = double(weff[2 * (wb + mm)]), wi = double(weff[2 * (wb + mm) + 1]);
          const double sr = sigma[2 * so], si = sigma[2 * so + 1];
          ar = fma(wr, sr, fma(-wi, si, ar));
          ai = fma(wr, si, fma(wi, sr, ai));
        } else {
          ar = fma(double(weff[wb + mm]), sigma[so], ar);
        }
      }
    }
    const size_t o = size_t(i) * nd + m;
    if (CPLX) {
      pot[2 * o] = ar;
      pot[2 * o + 1] = ai;
    } else {
      pot[o] = ar;
    }
  }
}

// MODE: the form of the row's work, by density count -- kCombineOne (nd ==
// 1), kCombineMd4 (nd <= 8), kCombineWide (more) -- each compiled as its own
// kernel so that each has its own register budget.
constexpr int kCombineOne = 0, kCombineMd4 = 1, kCombineWide = 2;
inline int combine_mode(int nd) {
  return nd == 1 ? kCombineOne : nd <= 8 ? kCombineMd4 : kCombineWide;
}

template <int CPLX, typename W, int MODE>
__device__ __forceinline__ void combine_rows(const Geometry& g, const Near& nr,
                                             const W* __restrict__ weff,
                                             const double* __restrict__ sigma,
                                             const double* __restrict__ partial, int nchunks,
                                             double* __restrict__ pot, int nd, int64_t bx) {
  const int lane = threadIdx.x & 31;
  const int64_t i = (int64_t(bx) * blockDim.x + threadIdx.x) >> 5;
  const int64_t ntarg = g.ntarg;
  if constexpr (MODE == kCombineOne) {
    __shared__ double sred[32][8][2];
    // the row's range and its first 32 near pairs are loaded before the
    // partial-sum phase and its barrier, so their latency overlaps it
    int64_t k0 = 0, k1 = 0;
    if (i < ntarg) {
      k0 = nr.row_ptr[i];
      k1 = nr.row_ptr[i + 1];
    }
    int ps_pre = 0, np_pre = 0;
    int64_t wb_pre = 0;
    if (i < ntarg && lane < k1 - k0) {
      ps_pre = nr.nps[k0 + lane];
      wb_pre = nr.wofs[k0 + lane];
      np_pre = int(nr.wofs[k0 + lane + 1] - wb_pre);
    }
    // far-field partial sums of the block's 8 rows, read cooperatively: thread
    // t takes row t % 8 of chunks t / 8, t / 8 + 32, ..., so every warp load
    // covers four whole 8-row segments
    {
      const int r = threadIdx.x & 7, c0 = threadIdx.x >> 3;
      const int64_t row = int64_t(bx) * 8 + r;
      double pr = 0, pi = 0;
      if (row < ntarg)
        for (int c = c0; c < nchunks; c += 32) {
          const size_t o = size_t(c) * ntarg + row;
          if (CPLX) {
            const double2 v = reinterpret_cast<const double2*>(partial)[o];
            pr += v.x;
            pi += v.y;
          } else {
            pr += partial[o];
          }
        }
      sred[c0][r][0] = pr;
      sred[c0][r][1] = pi;
    }
    __syncthreads();
    if (i >= ntarg) return;
    const int wrow = threadIdx.x >> 5;
    double ar = sred[lane][wrow][0], ai = sred[lane][wrow][1];
    // Near patches of the row, 32 at a time: one lane-parallel load of their
    // first nodes and entry offsets (no dependent index loads), then the
    // row's W_eff span (contiguous: wofs[k+1] = wofs[k] + np) streamed with
    // coalesced loads, kCombineUnroll entries per lane in flight.
    constexpr unsigned kFull = 0xffffffffu;
    constexpr int kU = kCombineUnroll;
    for (int64_t kc = k0; kc < k1; kc += 32) {
      const int nkc = int(k1 - kc < 32 ? k1 - kc : 32);
      int ps = ps_pre, np = np_pre;
      int64_t wb = wb_pre;
      if (kc != k0) {
        ps = np = 0;
        wb = 0;
        if (lane < nkc) {
          ps = nr.nps[kc + lane];
          wb = nr.wofs[kc + lane];
          np = int(nr.wofs[kc + lane + 1] - wb);
        }
      }
      const int np0 = __shfl_sync(kFull, np, 0);
      const int64_t e0 = __shfl_sync(kFull, wb, 0);
      if (__all_sync(kFull, lane >= nkc || np == np0)) {
        // every patch of this group has np0 nodes: entry e belongs to patch
        // e / np0 (exact in FP32: the fraction stays >= 0.5/np0 from an integer)
        const int ne = nkc * np0;
        const float inv = 1.0f / float(np0);
        for (int eb = 0; eb < ne; eb += 32 * kU) {
          W wr[kU], wi[kU];  // W_eff stays in its storage precision until the FMA
          double sr[kU], si[kU];
#pragma unroll
          for (int u = 0; u < kU; ++u) {
            const int e = eb + 32 * u + lane;
            const bool ok = e < ne;
            const int kk = ok ? int((float(e) + 0.5f) * inv) : 0;
            const int psk = __shfl_sync(kFull, ps, kk);
            wr[u] = wi[u] = W(0);
            sr[u] = si[u] = 0.0;
            if (ok) {
              const int node = psk + (e - kk * np0);
              if (CPLX) {
                const typename Vec2<W>::T wv =
                    reinterpret_cast<const typename Vec2<W>::T*>(weff)[e0 + e];
                const double2 sv = reinterpret_cast<const double2*>(sigma)[node];
                wr[u] = wv.x;
                wi[u] = wv.y;
                sr[u] = sv.x;
                si[u] = sv.y;
              } else {
                wr[u] = weff[e0 + e];
                sr[u] = sigma[node];
              }
            }
          }
#pragma unroll
          for (int u = 0; u < kU; ++u) {
            const double a = double(wr[u]), b = double(wi[u]);
            if (CPLX) {
              ar = fma(a, sr[u], fma(-b, si[u], ar));
              ai = fma(a, si[u], fma(b, sr[u], ai));
            } else {
              ar = fma(a, sr[u], ar);
            }
          }
        }
      } else {
        // mixed patch sizes: one patch of the group at a time
        for (int j = 0; j < nkc; ++j) {
          const int psj = __shfl_sync(kFull, ps, j);
          const int npj = __shfl_sync(kFull, np, j);
          const int64_t wbj = __shfl_sync(kFull, wb, j);
          for (int mm = lane; mm < npj; mm += 32) {
            if (CPLX) {
              const double wr = double(weff[2 * (wbj + mm)]);
              const double wi = double(weff[2 * (wbj + mm) + 1]);
              const double sr = sigma[2 * (psj + mm)], si = sigma[2 * (psj + mm) + 1];
              ar = fma(wr, sr, fma(-wi, si, ar));
              ai = fma(wr, si, fma(wi, sr, ai));
            } else {
              ar = fma(double(weff[wbj + mm]), sigma[psj + mm], ar);
            }
          }
        }
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      ar += __shfl_xor_sync(0xffffffffu, ar, off);
      if (CPLX) ai += __shfl_xor_sync(0xffffffffu, ai, off);
    }
    if (lane == 0) {
      if (CPLX) {
        pot[2 * i] = ar;
        pot[2 * i + 1] = ai;
      } else {
        pot[i] = ar;
      }
    }
    return;
  } else {
    if (i >= ntarg) return;
    if constexpr (MODE == kCombineMd4)
      combine_row_md<CPLX, W, 4>(g, nr, weff, sigma, partial, nchunks, pot, nd, i, lane);
    else
      combine_row_wide<CPLX, W>(g, nr, weff, sigma, partial, nchunks, pot, nd, i, lane);
  }
}

// Blocks per SM each form is compiled for.  The several-density forms at 4
// (64 registers, no spills): unconstrained they took 96 (wide) and 127
// registers and 2 blocks per SM, and measured 0.89 against 0.62 ms at
// nd = 16, 1.73 against 1.42 ms at nd = 64, 0.25 against 0.20 ms at nd = 4
// on the 35,840-node matvec.
template <int MODE>
constexpr int kCombineBlocks = MODE == kCombineOne ? kCombineMinBlocks : 4;

template <int CPLX, typename W, int MODE>
__global__ void __launch_bounds__(kCombineThreads, kCombineBlocks<MODE>)
    combine_kernel(Geometry g, Near nr, const W* __restrict__ weff,
                   const double* __restrict__ sigma, const double* __restrict__ partial,
                   int nchunks, double* __restrict__ pot, int nd) {
  combine_rows<CPLX, W, MODE>(g, nr, weff, sigma, partial, nchunks, pot, nd, blockIdx.x);
}

// ---------------------------------------------------------------------------
// fold: W_eff = wnear - (smooth oversampled contribution) for each near pair
//
// MATCH32 = 0: the smooth part is the exact FP64 kernel (FP64 matvec path).
// MATCH32 = 1: the smooth part is evaluated with the FP32 far kernel's own
// arithmetic (same block-centred coordinates, same pair functions), so that
// the FP32 far field's error on near pairs -- where n.(t-s) = O(r^2) cancels
// in single precision -- is removed exactly by the subtraction; only the
// well-separated pairs are then left to the FP32 far sum.
// MATCH32 = 2: refold an FP32 W_eff from the FP64 one (wnear = W_eff f64):
// out = W_eff64 + exact part - FP32-matched part.
// The FP32 coordinates are centred as the FP32 far field centres them: on
// the first target of the target's 512-target block, or on g.tcen[3 i ..]
// (the leaf centre of the hierarchical far field) when that is set.
// ---------------------------------------------------------------------------
constexpr int kFarBlockTargetsF32 = 512;  // kFarThreads * kTptF32 (checked below)

template <int CPLX, int MATCH32, typename OUT>
__global__ void fold_kernel(Geometry g, Near nr, KParams kp, const double* __restrict__ wnear,
                            OUT* __restrict__ weff, int64_t k0, int64_t k1) {
  extern __shared__ double sh[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* a = sh + size_t(warp) * g.max_nf * 2;
  // find the row of pair k (near pairs k0 .. k1 - 1) by binary search over row_ptr
  const int64_t k = k0 + int64_t(blockIdx.x) * (blockDim.x >> 5) + warp;
  if (k >= k1) return;
  int64_t lo = 0, hi = g.ntarg;  // row_ptr[lo] <= k < row_ptr[hi]
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (nr.row_ptr[mid] <= k)
      lo = mid;
    else
      hi = mid;
  }
  const int64_t i = lo;
  const double tx = g.tx[i], ty = g.ty[i], tz = g.tz[i];
  const int p = nr.col[k];
  const int ps = g.pstart[p], np = g.pstart[p + 1] - ps;
  const int os = g.ostart[p], nf = g.ostart[p + 1] - os;
  const double* M = g.imat + g.cmoff[g.pclass[p]];
  const double thr2 = kp.thresh * kp.thresh;
  // centre of target i's FP32 coordinates in the far field
  const int64_t tb = (i / kFarBlockTargetsF32) * kFarBlockTargetsF32;
  const double cx = g.tcen ? g.tcen[3 * i] : g.tx[tb];
  const double cy = g.tcen ? g.tcen[3 * i + 1] : g.ty[tb];
  const double cz = g.tcen ? g.tcen[3 * i + 2] : g.tz[tb];
  const float tx32 = float(tx - cx), ty32 = float(ty - cy), tz32 = float(tz - cz);
  for (int l = lane; l < nf; l += 32) {
    const int s = os + l;
    double vr = 0, vi = 0, fr = 0, fi = 0;
    if (MATCH32) {
      const float4 g0 = make_float4(float(g.sx[s] - cx), float(g.sy[s] - cy), float(g.sz[s] - cz),
                                    float(g.snx[s]));
      const float2 g1 = make_float2(float(g.sny[s]), float(g.snz[s]));
      const float thr2f = float(thr2);
      const double f = g.sw[s] * kOver4Pi;
      if (CPLX) {
        // unit charge and unit dipole responses of the FP32 pair function
        float gr = 0, gi = 0, dr = 0, di = 0;
        pair_helm(tx32, ty32, tz32, g0, g1, make_float4(1.f, 0.f, 0.f, 0.f), float(kp.kr),
                  float(kp.ki), thr2f, kp.ki != 0.0, gr, gi);
        pair_helm(tx32, ty32, tz32, g0, g1, make_float4(0.f, 0.f, 1.f, 0.f), float(kp.kr),
                  float(kp.ki), thr2f, kp.ki != 0.0, dr, di);
        vr = (kp.ar * gr - kp.ai * gi + kp.br * dr - kp.bi * di) * f;
        vi = (kp.ar * gi + kp.ai * gr + kp.br * di + kp.bi * dr) * f;
      } else {
        float pc = 0, pd = 0;
        pair_lap<float>(tx32, ty32, tz32, g0, g1, make_float2(1.f, 0.f), thr2f, pc);
        pair_lap<float>(tx32, ty32, tz32, g0, g1, make_float2(0.f, 1.f), thr2f, pd);
        vr = (kp.ar * pc + kp.br * pd) * f;
      }
      if (MATCH32 == 1) {
        a[2 * l] = vr;
        a[2 * l + 1] = vi;
        continue;
      }
      fr = vr;
      fi = vi;
      vr = vi = 0;
    }
    const double dx = tx - g.sx[s], dy = ty - g.sy[s], dz = tz - g.sz[s];
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 >= thr2) {
      const double r = sqrt(r2), rinv = 1.0 / r;
      const double dn = dx * g.snx[s] + dy * g.sny[s] + dz * g.snz[s];
      const double f = g.sw[s] * kOver4Pi;
      if (CPLX) {
        double sn, cs;
        sincos(kp.kr * r, &sn, &cs);
        const double damp = exp(-kp.ki * r);
        const double er = cs * damp * rinv, ei = sn * damp * rinv;  // e^{ikr}/r
        // (1 - i k r) with complex k: 1 + ki r - i kr r
        const double qr = dn * rinv * rinv * (1.0 + kp.ki * r), qi = -dn * rinv * rinv * kp.kr * r;
        // alpha + beta*q
        const double cr = kp.ar + kp.br * qr - kp.bi * qi;
        const double ci = kp.ai + kp.br * qi + kp.bi * qr;
        vr = (cr * er - ci * ei) * f;
        vi = (cr * ei + ci * er) * f;
      } else {
        vr = (kp.ar + kp.br * dn * rinv * rinv) * rinv * f;
      }
    }
    if (MATCH32 == 2) {
      vr = fr - vr;
      vi = fi - vi;
    }
    a[2 * l] = vr;
    a[2 * l + 1] = vi;
  }
  __syncwarp();
  const int64_t wb = nr.wofs[k];
  for (int mm = lane; mm < np; mm += 32) {
    double sr = 0, si = 0;
    for (int l = 0; l < nf; ++l) {
      const double mv = M[size_t(l) * np + mm];
      sr = fma(a[2 * l], mv, sr);
      si = fma(a[2 * l + 1], mv, si);
    }
    if (CPLX) {
      weff[2 * (wb + mm)] = OUT(wnear[2 * (wb + mm)] - sr);
      weff[2 * (wb + mm) + 1] = OUT(wnear[2 * (wb + mm) + 1] - si);
    } else {
      weff[wb + mm] = OUT(wnear[wb + mm] - sr);
    }
  }
}

// Direct far-field evaluation from caller strengths: pack (charge, dipole
// strength) per source into the far kernel's layout, scaled by 1/(4 pi).
template <typename R, int CPLX>
__global__ void pack_strengths_kernel(const double* __restrict__ charge,
                                      const double* __restrict__ dipstr, int64_t ns,
                                      R* __restrict__ str, const int32_t* __restrict__ sdest) {
  for (int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < ns;
       s += int64_t(gridDim.x) * blockDim.x) {
    const int64_t o = sdest ? int64_t(sdest[s]) : s;
    if (CPLX) {
      str[4 * o + 0] = R(charge[2 * s] * kOver4Pi);
      str[4 * o + 1] = R(charge[2 * s + 1] * kOver4Pi);
      str[4 * o + 2] = R(dipstr[2 * s] * kOver4Pi);
      str[4 * o + 3] = R(dipstr[2 * s + 1] * kOver4Pi);
    } else {
      str[2 * o + 0] = R(charge[s] * kOver4Pi);
      str[2 * o + 1] = R(dipstr[s] * kOver4Pi);
    }
  }
}

// pot[i] = sum over chunks of partial[c][i]
template <int CPLX>
__global__ void reduce_partials_kernel(const double* __restrict__ partial, int nchunks,
                                       int64_t ntarg, double* __restrict__ pot) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < ntarg;
       i += int64_t(gridDim.x) * blockDim.x) {
    double ar = 0, ai = 0;
    for (int c = 0; c < nchunks; ++c) {
      const size_t o = size_t(c) * ntarg + i;
      if (CPLX) {
        ar += partial[2 * o];
        ai += partial[2 * o + 1];
      } else {
        ar += partial[o];
      }
    }
    if (CPLX) {
      pot[2 * i] = ar;
      pot[2 * i + 1] = ai;
    } else {
      pot[i] = ar;
    }
  }
}

__global__ void to_f32_kernel(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    out[i] = float(in[i]);
}

// ---------------------------------------------------------------------------
// GMRES vector kernels.  Vectors hold npts nodes x nd densities (point-major).
// The nodes form segments (one per surface of a batch); system
// sys = seg(node) * nd + density is one independent linear system, so every
// inner product is taken per system and every coefficient is per system.
// Reductions run over chunks: contiguous node ranges inside one segment.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int sys_of(const Segs& sg, int64_t e, int nd) {
  const int64_t pt = e / nd;
  const int seg = sg.node_seg ? sg.node_seg[pt] : 0;
  return seg * nd + int(e - pt * nd);
}

// partial[((k*nd + d)*nchunk + c)] = sum over chunk c of wts * conj(V_k) w
template <int CPLX>
__global__ void mdot_partial_kernel(const double* __restrict__ V, int64_t ldv, int m,
                                    const double* __restrict__ w, const double* __restrict__ wts,
                                    int nd, Segs sg, double* __restrict__ partial) {
  __shared__ double2 red[256];
  const int tid = threadIdx.x;
  const int rows = blockDim.x / nd;  // blockDim.x is a multiple of nd
  const int dd = tid % nd, r = tid / nd;
  const int c = blockIdx.x;
  const int64_t lo = sg.chunk_lo[c], hi = sg.chunk_hi[c];
  if (32 % nd == 0) {
    // nd divides the warp: each warp takes whole vectors k = warp, warp + nw,
    // ... over the chunk (lane = row (lane / nd), density lane % nd), sums
    // its rows with xor shuffles over offsets nd .. 16, and writes; no
    // barriers
    const int warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    const int wr = 32 / nd, ld = lane % nd, lr = lane / nd;
    for (int k = warp; k < m; k += nw) {
      const double* v = V + size_t(k) * ldv;
      double sr = 0, si = 0;
      for (int64_t pt = lo + lr; pt < hi; pt += wr) {
        const int64_t e = pt * nd + ld;
        const double wt = wts[pt];
        if (CPLX) {
          const double vr = v[2 * e], vi = v[2 * e + 1], xr = w[2 * e], xi = w[2 * e + 1];
          sr += wt * (vr * xr + vi * xi);
          si += wt * (vr * xi - vi * xr);
        } else {
          sr += wt * v[e] * w[e];
        }
      }
      for (int off = 16; off >= nd; off >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, off);
        si += __shfl_xor_sync(0xffffffffu, si, off);
      }
      if (lane < nd) {
        const size_t o = (size_t(k) * nd + lane) * sg.nchunk + c;
        partial[2 * o] = sr;
        partial[2 * o + 1] = si;
      }
    }
    return;
  }
  for (int k = 0; k < m; ++k) {
    const double* v = V + size_t(k) * ldv;
    double sr = 0, si = 0;
    for (int64_t pt = lo + r; pt < hi; pt += rows) {
      const int64_t e = pt * nd + dd;
      const double wt = wts[pt];
      if (CPLX) {
        const double vr = v[2 * e], vi = v[2 * e + 1], xr = w[2 * e], xi = w[2 * e + 1];
        sr += wt * (vr * xr + vi * xi);
        si += wt * (vr * xi - vi * xr);
      } else {
        sr += wt * v[e] * w[e];
      }
    }
    {
      red[tid] = make_double2(sr, si);
      __syncthreads();
      if (tid < nd) {
        double ar = 0, ai = 0;
        for (int q = 0; q < rows; ++q) {
          ar += red[q * nd + tid].x;
          ai += red[q * nd + tid].y;
        }
        const size_t o = (size_t(k) * nd + tid) * sg.nchunk + c;
        partial[2 * o] = ar;
        partial[2 * o + 1] = ai;
      }
      __syncthreads();
    }
  }
}

// out[2*(k*nsys + sys)] = sum of the partials of the chunks of sys's segment
__global__ void mdot_final_kernel(const double* __restrict__ partial, int nd, Segs sg,
                                  double* __restrict__ out) {
  __shared__ double red[2][32];
  const int nsys = sg.nseg * nd;
  const int b = blockIdx.x;  // flattened (k, sys)
  const int k = b / nsys, sys = b - k * nsys;
  const int seg = sys / nd, d = sys - seg * nd;
  const int c0 = sg.seg_chunk0[seg], c1 = sg.seg_chunk0[seg + 1];
  const size_t base = (size_t(k) * nd + d) * sg.nchunk;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double sr = 0, si = 0;
  for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
    sr += partial[2 * (base + c)];
    si += partial[2 * (base + c) + 1];
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    sr += __shfl_xor_sync(0xffffffffu, sr, off);
    si += __shfl_xor_sync(0xffffffffu, si, off);
  }
  if (lane == 0) {
    red[0][warp] = sr;
    red[1][warp] = si;
  }
  __syncthreads();
  if (warp == 0) {
    sr = lane < nw ? red[0][lane] : 0.0;
    si = lane < nw ? red[1][lane] : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, off);
      si += __shfl_xor_sync(0xffffffffu, si, off);
    }
    if (lane == 0) {
      out[2 * b] = sr;
      out[2 * b + 1] = si;
    }
  }
}

// w[e] -= sum_k h[k, sys(e)] V_k[e]
template <int CPLX>
__global__ void maxpy_kernel(const double* __restrict__ V, int64_t ldv, int m,
                             const double* __restrict__ h, double* __restrict__ w, int64_t n,
                             int nd, Segs sg) {
  const int nsys = sg.nseg * nd;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int sy = sys_of(sg, e, nd);
    if (CPLX) {
      double xr = w[2 * e], xi = w[2 * e + 1];
      for (int k = 0; k < m; ++k) {
        const double hr = h[2 * (k * nsys + sy)], hi = h[2 * (k * nsys + sy) + 1];
        const double vr = V[size_t(k) * ldv + 2 * e], vi = V[size_t(k) * ldv + 2 * e + 1];
        xr -= hr * vr - hi * vi;
        xi -= hr * vi + hi * vr;
      }
      w[2 * e] = xr;
      w[2 * e + 1] = xi;
    } else {
      double x = w[e];
      for (int k = 0; k < m; ++k) x -= h[2 * (k * nsys + sy)] * V[size_t(k) * ldv + e];
      w[e] = x;
    }
  }
}

// y[e] = sum_k c[k, sys(e)] V_k[e]
template <int CPLX>
__global__ void combo_kernel(const double* __restrict__ V, int64_t ldv, int m,
                             const double* __restrict__ c, double* __restrict__ y, int64_t n,
                             int nd, Segs sg) {
  const int nsys = sg.nseg * nd;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int sy = sys_of(sg, e, nd);
    double xr = 0, xi = 0;
    for (int k = 0; k < m; ++k) {
      const double cr = c[2 * (k * nsys + sy)], ci = c[2 * (k * nsys + sy) + 1];
      if (CPLX) {
        const double vr = V[size_t(k) * ldv + 2 * e], vi = V[size_t(k) * ldv + 2 * e + 1];
        xr += cr * vr - ci * vi;
        xi += cr * vi + ci * vr;
      } else {
        xr += cr * V[size_t(k) * ldv + e];
      }
    }
    if (CPLX) {
      y[2 * e] = xr;
      y[2 * e + 1] = xi;
    } else {
      y[e] = xr;
    }
  }
}

// y = a*x + b*y, scalar complex a, b
template <int CPLX>
__global__ void axpby_kernel(const double* __restrict__ x, double* __restrict__ y, double ar,
                             double ai, double br, double bi, int64_t n) {
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    if (CPLX) {
      const double xr = x[2 * e], xi = x[2 * e + 1], yr = y[2 * e], yi = y[2 * e + 1];
      y[2 * e] = ar * xr - ai * xi + br * yr - bi * yi;
      y[2 * e + 1] = ar * xi + ai * xr + br * yi + bi * yr;
    } else {
      y[e] = ar * x[e] + br * y[e];
    }
  }
}

// y[e] = a[sys(e)] * x[e] + b * y[e], a complex per system (device)
template <int CPLX>
__global__ void axpbys_kernel(const double* __restrict__ x, double* __restrict__ y,
                              const double* __restrict__ a, double br, double bi, int64_t n,
                              int nd, Segs sg) {
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int sy = sys_of(sg, e, nd);
    const double ar = a[2 * sy], ai = a[2 * sy + 1];
    if (CPLX) {
      const double xr = x[2 * e], xi = x[2 * e + 1], yr = y[2 * e], yi = y[2 * e + 1];
      y[2 * e] = ar * xr - ai * xi + br * yr - bi * yi;
      y[2 * e + 1] = ar * xi + ai * xr + br * yi + bi * yr;
    } else {
      y[e] = ar * x[e] + br * y[e];
    }
  }
}

// y[e] = s[sys(e)] * x[e], s complex per system (device)
template <int CPLX>
__global__ void dscale_kernel(const double* __restrict__ x, double* __restrict__ y,
                              const double* __restrict__ s, int64_t n, int nd, Segs sg) {
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int sy = sys_of(sg, e, nd);
    const double sr = s[2 * sy], si = s[2 * sy + 1];
    if (CPLX) {
      const double xr = x[2 * e], xi = x[2 * e + 1];
      y[2 * e] = sr * xr - si * xi;
      y[2 * e + 1] = sr * xi + si * xr;
    } else {
      y[e] = sr * x[e];
    }
  }
}

inline int grid_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return int(b);
}

// Far-kernel launch shapes.
constexpr int kFarThreads = 128;
constexpr int kFarTile = 128;
static_assert(kFarTile == kFarTileSources, "source tiles of the box table");
static_assert(kFarBlockTargetsF32 == kFarBlockTargets32, "target blocks of the box table");
constexpr int kTptF32 = 4;
constexpr int kTptF64 = 2;
static_assert(kFarThreads * kTptF32 == kFarBlockTargetsF32,
              "the FP32 fold must centre coordinates exactly like the FP32 far kernel");

}  // namespace

int far_nchunks(int64_t ntarg, int64_t nptso, int kind, int precision, int nd, int num_sms) {
  (void)kind;
  const int tpt = precision == 1 ? kTptF32 : kTptF64;
  const int64_t tblocks = (ntarg + int64_t(kFarThreads) * tpt - 1) / (int64_t(kFarThreads) * tpt);
  const int64_t want = int64_t(num_sms) * 6;  // blocks in flight over the chip
  int64_t s = (want + tblocks * nd - 1) / (tblocks * nd);
  const int64_t maxs = std::max<int64_t>(1, nptso / (2 * kFarTile));
  s = std::max<int64_t>(1, std::min<int64_t>(s, maxs));
  return int(s);
}

cudaError_t launch_strengths(const Geometry& g, const KParams& kp, const MatvecArgs& a,
                             cudaStream_t st) {
  const int cplx = kp.kind == 1;
  const size_t sh = size_t(g.max_np) * a.nd * (cplx ? 2 : 1) * sizeof(double);
  if (sh > 200 * 1024) return cudaErrorInvalidValue;
  const dim3 grid(static_cast<unsigned>(g.npatches)), block(128);
  if (a.precision == 1) {
    if (sh > 48 * 1024) {
      cudaFuncSetAttribute(strengths_kernel<float, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sh));
      cudaFuncSetAttribute(strengths_kernel<float, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sh));
    }
    if (cplx)
      strengths_kernel<float, 1><<<grid, block, sh, st>>>(g, kp, a.sigma, (float*)a.strengths, a.nd, a.sdest);
    else
      strengths_kernel<float, 0><<<grid, block, sh, st>>>(g, kp, a.sigma, (float*)a.strengths, a.nd, a.sdest);
  } else {
    if (sh > 48 * 1024) {
      cudaFuncSetAttribute(strengths_kernel<double, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sh));
      cudaFuncSetAttribute(strengths_kernel<double, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sh));
    }
    if (cplx)
      strengths_kernel<double, 1><<<grid, block, sh, st>>>(g, kp, a.sigma, (double*)a.strengths, a.nd, a.sdest);
    else
      strengths_kernel<double, 0><<<grid, block, sh, st>>>(g, kp, a.sigma, (double*)a.strengths, a.nd, a.sdest);
  }
  count();
  return cudaGetLastError();
}

namespace {
// Far-kernel shapes.  Every f32 variant keeps kFarThreads*kTptF32 = 512
// targets per block (the FP32 fold centres coordinates per 512 targets).
template <int KIND, typename R, int NT, int TPT, bool CK>
cudaError_t launch_far_t(const Geometry& g, const KParams& kp, const MatvecArgs& a,
                         cudaStream_t st) {
  const int64_t per_block = int64_t(NT) * TPT;
  const int64_t tblocks = (g.ntarg + per_block - 1) / per_block;
  int64_t chunk = (g.nptso + a.nchunks - 1) / a.nchunks;
  chunk = ((chunk + kFarTile - 1) / kFarTile) * kFarTile;
  const dim3 grid(static_cast<unsigned>(tblocks), static_cast<unsigned>(a.nchunks),
                  static_cast<unsigned>(a.nd));
  far_kernel<KIND, R, NT, TPT, kFarTile, CK><<<grid, NT, 0, st>>>(
      g, kp, static_cast<const R*>(a.strengths), a.partial, chunk, a.nd);
  return cudaGetLastError();
}

template <int KIND, typename R, int NT, int TPT, bool CK>
int occupancy_t() {
  int b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, far_kernel<KIND, R, NT, TPT, kFarTile, CK>, NT,
                                                0);
  return b;
}

// (threads, targets per thread) of each variant
constexpr int kF32Shapes[3][2] = {{128, 4}, {64, 8}, {256, 2}};
constexpr int kF64Shapes[3][2] = {{128, 2}, {64, 4}, {256, 1}};

template <int KIND, typename R, bool CK, int V>
cudaError_t far_dispatch(const Geometry& g, const KParams& kp, const MatvecArgs& a,
                         cudaStream_t st, int* occ) {
  constexpr bool F32 = sizeof(R) == 4;
  constexpr int NT = F32 ? kF32Shapes[V][0] : kF64Shapes[V][0];
  constexpr int TPT = F32 ? kF32Shapes[V][1] : kF64Shapes[V][1];
  if (occ) {
    *occ = occupancy_t<KIND, R, NT, TPT, CK>();
    return cudaSuccess;
  }
  return launch_far_t<KIND, R, NT, TPT, CK>(g, kp, a, st);
}

template <int KIND, typename R, bool CK>
cudaError_t far_variant(int v, const Geometry& g, const KParams& kp, const MatvecArgs& a,
                        cudaStream_t st, int* occ) {
  switch (v) {
    case 1:
      return far_dispatch<KIND, R, CK, 1>(g, kp, a, st, occ);
    case 2:
      return far_dispatch<KIND, R, CK, 2>(g, kp, a, st, occ);
    default:
      return far_dispatch<KIND, R, CK, 0>(g, kp, a, st, occ);
  }
}

// multi-density shapes (threads, targets per thread, densities per block):
// one class per density-group size, chosen by nd (<= 4, <= 8, more), and
// three block shapes per class for the autotuner.
constexpr int kMdShapes[3][3][3] = {
    {{128, 1, 4}, {128, 2, 4}, {256, 1, 4}},
    {{128, 1, 8}, {128, 2, 8}, {64, 2, 8}},
    {{128, 1, 16}, {64, 1, 16}, {256, 1, 16}}};

inline int md_class(int nd) { return nd <= 4 ? 0 : (nd <= 8 ? 1 : 2); }

template <int KIND, typename R, bool CK, int CL, int V>
cudaError_t far_md_dispatch(const Geometry& g, const KParams& kp, const MatvecArgs& a,
                            cudaStream_t st, int* occ) {
  constexpr int NT = kMdShapes[CL][V][0], TPT = kMdShapes[CL][V][1], MD = kMdShapes[CL][V][2];
  if (occ) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        occ, far_md_kernel<KIND, R, NT, TPT, MD, kFarTile, CK>, NT, 0);
    return cudaSuccess;
  }
  const int64_t tblocks = (g.ntarg + int64_t(NT) * TPT - 1) / (int64_t(NT) * TPT);
  const int groups = (a.nd + MD - 1) / MD;
  int64_t chunk = (g.nptso + a.nchunks - 1) / a.nchunks;
  chunk = ((chunk + kFarTile - 1) / kFarTile) * kFarTile;
  const dim3 grid(static_cast<unsigned>(tblocks), static_cast<unsigned>(a.nchunks),
                  static_cast<unsigned>(groups));
  far_md_kernel<KIND, R, NT, TPT, MD, kFarTile, CK><<<grid, NT, 0, st>>>(
      g, kp, static_cast<const R*>(a.ab), static_cast<const R*>(a.strengths), a.nd, a.partial,
      chunk);
  return cudaGetLastError();
}

template <int KIND, typename R, bool CK, int CL>
cudaError_t far_md_class(int v, const Geometry& g, const KParams& kp, const MatvecArgs& a,
                         cudaStream_t st, int* occ) {
  switch (v) {
    case 1:
      return far_md_dispatch<KIND, R, CK, CL, 1>(g, kp, a, st, occ);
    case 2:
      return far_md_dispatch<KIND, R, CK, CL, 2>(g, kp, a, st, occ);
    default:
      return far_md_dispatch<KIND, R, CK, CL, 0>(g, kp, a, st, occ);
  }
}

template <int KIND, typename R, bool CK>
cudaError_t far_md_variant(int v, const Geometry& g, const KParams& kp, const MatvecArgs& a,
                           cudaStream_t st, int* occ) {
  switch (md_class(a.nd)) {
    case 0:
      return far_md_class<KIND, R, CK, 0>(v, g, kp, a, st, occ);
    case 1:
      return far_md_class<KIND, R, CK, 1>(v, g, kp, a, st, occ);
    default:
      return far_md_class<KIND, R, CK, 2>(v, g, kp, a, st, occ);
  }
}

cudaError_t far_md_any(const Geometry& g, const KParams& kp, const MatvecArgs& a, cudaStream_t st,
                       int* occ) {
  const bool ck = kp.kind == 1 && kp.ki != 0.0;
  int v = a.far_variant;
  if (v >= 3) {
    if (far_tc_group(v, a.nd, a.precision, kp.kind) > 0) return far_tc(v, g, kp, a, st, occ);
    if (occ) {  // not a shape of this path: the autotuner skips it
      *occ = 0;
      return cudaSuccess;
    }
    v = 0;
  }
  if (a.precision == 1) {
    if (kp.kind == 1)
      return ck ? far_md_variant<1, float, true>(v, g, kp, a, st, occ)
                : far_md_variant<1, float, false>(v, g, kp, a, st, occ);
    return far_md_variant<0, float, false>(v, g, kp, a, st, occ);
  }
  if (kp.kind == 1)
    return ck ? far_md_variant<1, double, true>(v, g, kp, a, st, occ)
              : far_md_variant<1, double, false>(v, g, kp, a, st, occ);
  return far_md_variant<0, double, false>(v, g, kp, a, st, occ);
}

cudaError_t far_any(const Geometry& g, const KParams& kp, const MatvecArgs& a, cudaStream_t st,
                    int* occ) {
  const bool ck = kp.kind == 1 && kp.ki != 0.0;
  const int v = a.far_variant;
  if (v >= 3 && occ) {  // the tensor-core shapes are multi-density only
    *occ = 0;
    return cudaSuccess;
  }
  if (a.precision == 1) {
    if (kp.kind == 1)
      return ck ? far_variant<1, float, true>(v, g, kp, a, st, occ)
                : far_variant<1, float, false>(v, g, kp, a, st, occ);
    return far_variant<0, float, false>(v, g, kp, a, st, occ);
  }
  if (kp.kind == 1)
    return ck ? far_variant<1, double, true>(v, g, kp, a, st, occ)
              : far_variant<1, double, false>(v, g, kp, a, st, occ);
  return far_variant<0, double, false>(v, g, kp, a, st, occ);
}
}  // namespace

namespace {
// ---- batched matvec kernels ----------------------------------------------------
template <typename R, int CPLX>
__global__ void batch_strengths_kernel(const BatchSurf* __restrict__ bs,
                                       const int2* __restrict__ items, int nitems,
                                       const double* const* __restrict__ xref,
                                       R* __restrict__ str, int nd, int over) {
  extern __shared__ double sh[];
  const double* x = *xref;
  constexpr int C = CPLX ? 2 : 1;
  for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
    const int2 it = items[w];
    const BatchSurf& S = bs[it.x];
    if (S.live && *S.live == 0) continue;  // uniform over the block
    const Geometry g = S.g;
    if (over)
      oversample_body<R, CPLX>(g, x + S.vofs * nd * C, str + S.sofs * nd * C, nd, it.y, sh);
    else
      strengths_body<R, CPLX>(g, S.kp, x + S.vofs * nd * C, str + S.sofs * nd * 2 * C, nd, it.y,
                              sh);
    __syncthreads();
  }
}

// Next work item of a persistent batch kernel, taken from a counter that the
// launch sequence zeroes before the kernel: thread 0 draws, the block reads
// it, and the second barrier keeps thread 0's next draw from overwriting the
// slot before every thread has read it (items are then handed out in list
// order, largest first, as blocks become free).
__device__ __forceinline__ int next_item(int* counter, int* slot) {
  if (threadIdx.x == 0) *slot = atomicAdd(counter, 1);
  __syncthreads();
  const int w = *slot;
  __syncthreads();
  return w;
}

template <int KIND, typename R, int NT, int TPT, int TILE, bool CK>
__global__ void __launch_bounds__(NT)
    batch_far_kernel(const BatchSurf* __restrict__ bs, const int4* __restrict__ items, int nitems,
                     const R* __restrict__ str, double* __restrict__ partial, int nd, int prec,
                     int* __restrict__ counter) {
  constexpr int SW = (KIND == 1) ? 4 : 2;
  constexpr bool X2 = sizeof(R) == 4;
  __shared__ float4 tile[X2 ? TILE * kFarX2Words<KIND> : 1];
  __shared__ typename Vec<R>::T4 sg0[X2 ? 1 : TILE];
  __shared__ typename Vec<R>::T2 sg1[X2 ? 1 : TILE];
  __shared__ R sst[X2 ? 1 : TILE * SW];
  __shared__ double2 stab[sizeof(R) == 8 && KIND == 1 ? kFarTrigN : 1];
  const double2* tab = nullptr;
  if constexpr (sizeof(R) == 8 && KIND == 1) {
    fill_far_trig_table(stab);
    tab = stab;
  }
  __syncthreads();
  __shared__ int s_w;
  for (;;) {
    const int w = next_item(counter, &s_w);
    if (w >= nitems) break;
    const int4 it = items[w];
    const BatchSurf& S = bs[it.x];
    if (S.live && *S.live == 0) continue;  // uniform over the block
    const Geometry g = S.g;
    const KParams kp = S.kp;
    if constexpr (X2)
      far_block_x2<KIND, NT, TPT, TILE, CK>(g, kp, str + S.sofs * nd * SW, partial + S.pofs[prec],
                                            S.chunk_len[prec], nd, it.y, it.z, it.w, tile);
    else
      far_block<KIND, R, NT, TPT, TILE, CK>(g, kp, str + S.sofs * nd * SW,
                                            partial + S.pofs[prec], S.chunk_len[prec], nd, it.y,
                                            it.z, it.w, tab, sg0, sg1, sst);
    __syncthreads();
  }
}

template <int KIND, typename R, int NT, int TPT, int MD, int TILE, bool CK>
__global__ void __launch_bounds__(NT)
    batch_far_md_kernel(const BatchSurf* __restrict__ bs, const int4* __restrict__ items,
                        int nitems, const R* __restrict__ sig, double* __restrict__ partial,
                        int nd, int prec, int* __restrict__ counter) {
  constexpr int C = (KIND == 1) ? 2 : 1;
  __shared__ typename Vec<R>::T4 sg0[TILE];
  __shared__ typename Vec<R>::T2 sg1[TILE];
  __shared__ __align__(16) R sab[TILE * 2 * C];
  __shared__ __align__(16) R ssig[TILE * MD * kMdSigWords<KIND, R, MD>];
  __shared__ double2 stab[sizeof(R) == 8 && KIND == 1 ? kFarTrigN : 1];
  const double2* tab = nullptr;
  if constexpr (sizeof(R) == 8 && KIND == 1) {
    fill_far_trig_table(stab);
    tab = stab;
  }
  __syncthreads();
  __shared__ int s_w;
  for (;;) {
    const int w = next_item(counter, &s_w);
    if (w >= nitems) break;
    const int4 it = items[w];
    const BatchSurf& S = bs[it.x];
    if (S.live && *S.live == 0) continue;  // uniform over the block
    const Geometry g = S.g;
    const KParams kp = S.kp;
    far_md_block<KIND, R, NT, TPT, MD, TILE, CK>(
        g, kp, static_cast<const R*>(S.ab[prec]), sig + S.sofs * nd * C, nd,
        partial + S.pofs[prec], S.chunk_len[prec], it.y, it.z, it.w, tab, sg0, sg1, sab, ssig);
    __syncthreads();
  }
}

template <int CPLX, typename W, int MODE>
__global__ void __launch_bounds__(kCombineThreads, kCombineBlocks<MODE>)
    batch_combine_kernel(const BatchSurf* __restrict__ bs, const int2* __restrict__ items,
                         int nitems, const double* const* __restrict__ xref,
                         double* const* __restrict__ yref, const double* __restrict__ partial,
                         int nd, int prec) {
  const double* x = *xref;
  double* y = *yref;
  constexpr int C = CPLX ? 2 : 1;
  for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
    const int2 it = items[w];
    const BatchSurf& S = bs[it.x];
    if (S.live && *S.live == 0) {
      // converged surface: zero rows, so no stale value enters the solver
      const int64_t row = int64_t(it.y) * 8 + (threadIdx.x >> 5);
      if (row < S.g.ntarg) {
        double* yr = y + (S.vofs + row) * nd * C;
        for (int j = threadIdx.x & 31; j < nd * C; j += 32) yr[j] = 0.0;
      }
      __syncthreads();
      continue;
    }
    const Geometry g = S.g;
    const Near nr = S.nr;
    combine_rows<CPLX, W, MODE>(g, nr, static_cast<const W*>(S.weff[prec]), x + S.vofs * nd * C,
                          partial + S.pofs[prec], S.nchunks[prec], y + S.vofs * nd * C, nd, it.y);
    __syncthreads();
  }
}

template <int KIND, typename R, bool CK, int V>
cudaError_t batch_far_dispatch(const BatchArgs& a, cudaStream_t st, int* occ) {
  constexpr bool F32 = sizeof(R) == 4;
  constexpr int NT = F32 ? kF32Shapes[V][0] : kF64Shapes[V][0];
  constexpr int TPT = F32 ? kF32Shapes[V][1] : kF64Shapes[V][1];
  auto kern = batch_far_kernel<KIND, R, NT, TPT, kFarTile, CK>;
  if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, NT, 0);
  kern<<<a.grid_far, NT, 0, st>>>(a.surfs, a.far_items, a.nfar_items,
                                  static_cast<const R*>(a.str), a.partial, a.nd, a.precision,
                                  a.far_counter);
  return cudaGetLastError();
}

template <int KIND, typename R, bool CK, int CL, int V>
cudaError_t batch_far_md_dispatch(const BatchArgs& a, cudaStream_t st, int* occ) {
  constexpr int NT = kMdShapes[CL][V][0], TPT = kMdShapes[CL][V][1], MD = kMdShapes[CL][V][2];
  auto kern = batch_far_md_kernel<KIND, R, NT, TPT, MD, kFarTile, CK>;
  if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, NT, 0);
  kern<<<a.grid_far, NT, 0, st>>>(a.surfs, a.far_items, a.nfar_items,
                                  static_cast<const R*>(a.str), a.partial, a.nd, a.precision,
                                  a.far_counter);
  return cudaGetLastError();
}

template <int KIND, typename R, bool CK>
cudaError_t batch_far_t(const BatchArgs& a, cudaStream_t st, int* occ) {
  const int v = a.variant;
  if (a.nd == 1) {
    switch (v) {
      case 1: return batch_far_dispatch<KIND, R, CK, 1>(a, st, occ);
      case 2: return batch_far_dispatch<KIND, R, CK, 2>(a, st, occ);
      default: return batch_far_dispatch<KIND, R, CK, 0>(a, st, occ);
    }
  }
  switch (md_class(a.nd) * 3 + (v < 0 || v > 2 ? 0 : v)) {
    case 0: return batch_far_md_dispatch<KIND, R, CK, 0, 0>(a, st, occ);
    case 1: return batch_far_md_dispatch<KIND, R, CK, 0, 1>(a, st, occ);
    case 2: return batch_far_md_dispatch<KIND, R, CK, 0, 2>(a, st, occ);
    case 3: return batch_far_md_dispatch<KIND, R, CK, 1, 0>(a, st, occ);
    case 4: return batch_far_md_dispatch<KIND, R, CK, 1, 1>(a, st, occ);
    case 5: return batch_far_md_dispatch<KIND, R, CK, 1, 2>(a, st, occ);
    case 6: return batch_far_md_dispatch<KIND, R, CK, 2, 0>(a, st, occ);
    case 7: return batch_far_md_dispatch<KIND, R, CK, 2, 1>(a, st, occ);
    default: return batch_far_md_dispatch<KIND, R, CK, 2, 2>(a, st, occ);
  }
}

cudaError_t batch_far_any(const BatchArgs& a, cudaStream_t st, int* occ) {
  if (a.precision == 1) {
    if (a.kind == 1) return a.ck ? batch_far_t<1, float, true>(a, st, occ) : batch_far_t<1, float, false>(a, st, occ);
    return batch_far_t<0, float, false>(a, st, occ);
  }
  if (a.kind == 1) return a.ck ? batch_far_t<1, double, true>(a, st, occ) : batch_far_t<1, double, false>(a, st, occ);
  return batch_far_t<0, double, false>(a, st, occ);
}
}  // namespace

void batch_far_shape(int precision, int variant, int nd, int* targets_per_block, int* group) {
  const int v = variant < 0 || variant > 2 ? 0 : variant;
  if (nd == 1) {
    const int(*sh)[2] = precision == 1 ? kF32Shapes : kF64Shapes;
    *targets_per_block = sh[v][0] * sh[v][1];
    *group = 1;
    return;
  }
  const int cl = md_class(nd);
  *targets_per_block = kMdShapes[cl][v][0] * kMdShapes[cl][v][1];
  *group = kMdShapes[cl][v][2];
}

int batch_far_variants(int precision, int nd) {
  (void)precision;
  (void)nd;
  return 3;
}

int batch_far_blocks_per_sm(int kind, int precision, int variant, int nd, bool ck) {
  BatchArgs a;
  a.kind = kind;
  a.precision = precision;
  a.variant = variant;
  a.nd = nd;
  a.ck = ck;
  int occ = 0;
  batch_far_any(a, nullptr, &occ);
  return occ;
}

cudaError_t launch_batch_matvec(const BatchArgs& a, cudaStream_t st) {
  const int cplx = a.kind == 1;
  const size_t sh = size_t(a.max_np) * a.nd * (cplx ? 2 : 1) * sizeof(double);
  if (sh > 200 * 1024) return cudaErrorInvalidValue;
  const int over = a.nd > 1 ? 1 : 0;
  auto strengths = [&](auto kern, auto* out) -> cudaError_t {
    if (sh > 48 * 1024)
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sh));
    kern<<<a.grid_patch, 128, sh, st>>>(a.surfs, a.patch_items, a.npatch_items, a.xref, out, a.nd,
                                        over);
    return cudaGetLastError();
  };
  cudaError_t e;
  if (a.precision == 1)
    e = cplx ? strengths(batch_strengths_kernel<float, 1>, static_cast<float*>(a.str))
             : strengths(batch_strengths_kernel<float, 0>, static_cast<float*>(a.str));
  else
    e = cplx ? strengths(batch_strengths_kernel<double, 1>, static_cast<double*>(a.str))
             : strengths(batch_strengths_kernel<double, 0>, static_cast<double*>(a.str));
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(a.far_counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  e = batch_far_any(a, st, nullptr);
  if (e != cudaSuccess) return e;
  auto combine = [&](auto kern) {
    kern<<<a.grid_row, kCombineThreads, 0, st>>>(a.surfs, a.row_items, a.nrow_items, a.xref,
                                                 a.yref, a.partial, a.nd, a.precision);
  };
  auto by_mode = [&](auto one, auto md4, auto wide) {
    switch (combine_mode(a.nd)) {
      case kCombineOne: combine(one); break;
      case kCombineMd4: combine(md4); break;
      default: combine(wide); break;
    }
  };
  if (cplx) {
    if (a.precision == 1)
      by_mode(batch_combine_kernel<1, float, 0>, batch_combine_kernel<1, float, 1>,
              batch_combine_kernel<1, float, 2>);
    else
      by_mode(batch_combine_kernel<1, double, 0>, batch_combine_kernel<1, double, 1>,
              batch_combine_kernel<1, double, 2>);
  } else {
    if (a.precision == 1)
      by_mode(batch_combine_kernel<0, float, 0>, batch_combine_kernel<0, float, 1>,
              batch_combine_kernel<0, float, 2>);
    else
      by_mode(batch_combine_kernel<0, double, 0>, batch_combine_kernel<0, double, 1>,
              batch_combine_kernel<0, double, 2>);
  }
  count(3);
  return cudaGetLastError();
}

cudaError_t launch_far(const Geometry& g, const KParams& kp, const MatvecArgs& a, cudaStream_t st) {
  if (g.ntarg == 0) return cudaSuccess;
  const cudaError_t e = far_any(g, kp, a, st, nullptr);
  count();
  return e;
}

cudaError_t launch_far_md(const Geometry& g, const KParams& kp, const MatvecArgs& a,
                          cudaStream_t st) {
  if (g.ntarg == 0) return cudaSuccess;
  const cudaError_t e = far_md_any(g, kp, a, st, nullptr);
  count();
  return e;
}

cudaError_t launch_oversample(const Geometry& g, const KParams& kp, const MatvecArgs& a,
                              cudaStream_t st) {
  const int cplx = kp.kind == 1;
  const size_t sh = size_t(g.max_np) * a.nd * (cplx ? 2 : 1) * sizeof(double);
  if (sh > 200 * 1024) return cudaErrorInvalidValue;
  const dim3 grid(static_cast<unsigned>(g.npatches)), block(128);
  auto go = [&](auto kern, auto* out) {
    if (sh > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sh));
    kern<<<grid, block, sh, st>>>(g, a.sigma, out, a.nd, a.sdest);
  };
  if (a.precision == 1) {
    if (cplx)
      go(oversample_kernel<float, 1>, (float*)a.strengths);
    else
      go(oversample_kernel<float, 0>, (float*)a.strengths);
  } else {
    if (cplx)
      go(oversample_kernel<double, 1>, (double*)a.strengths);
    else
      go(oversample_kernel<double, 0>, (double*)a.strengths);
  }
  count();
  return cudaGetLastError();
}

cudaError_t launch_source_consts(const Geometry& g, const KParams& kp, int precision, void* ab,
                                 cudaStream_t st, const int32_t* sdest) {
  if (g.nptso == 0) return cudaSuccess;
  const int b = grid_for(g.nptso, 256);
  if (precision == 1) {
    if (kp.kind == 1)
      source_consts_kernel<float, 1><<<b, 256, 0, st>>>(g, kp, (float*)ab, sdest);
    else
      source_consts_kernel<float, 0><<<b, 256, 0, st>>>(g, kp, (float*)ab, sdest);
  } else {
    if (kp.kind == 1)
      source_consts_kernel<double, 1><<<b, 256, 0, st>>>(g, kp, (double*)ab, sdest);
    else
      source_consts_kernel<double, 0><<<b, 256, 0, st>>>(g, kp, (double*)ab, sdest);
  }
  count();
  return cudaGetLastError();
}

int far_variants() { return 5; }

int far_block_targets(int precision, int variant, int md, int nd) {
  if (md && far_tc_group(variant, nd, precision, 1) > 0) return far_tc_targets();
  const int v = variant < 0 || variant > 2 ? 0 : variant;
  if (md) return kMdShapes[md_class(nd)][v][0] * kMdShapes[md_class(nd)][v][1];
  return precision == 1 ? kF32Shapes[v][0] * kF32Shapes[v][1]
                        : kF64Shapes[v][0] * kF64Shapes[v][1];
}

int far_md_group(int variant, int nd) {
  const int tc = far_tc_group(variant, nd, 1, 1);
  if (tc > 0) return tc;
  return kMdShapes[md_class(nd)][variant < 0 || variant > 2 ? 0 : variant][2];
}

int far_blocks_per_sm(const KParams& kp, int precision, int variant, int md, int nd) {
  MatvecArgs a;
  a.precision = precision;
  a.far_variant = variant;
  a.nd = nd;
  Geometry g;
  int occ = 0;
  if (md)
    far_md_any(g, kp, a, nullptr, &occ);
  else
    far_any(g, kp, a, nullptr, &occ);
  return occ;
}

int far_chunks_for_waves(int64_t ntarg, int64_t nptso, int precision, int variant, int nd,
                         int num_sms, int blocks_per_sm, double waves, int md) {
  const int64_t bt = far_block_targets(precision, variant, md, nd);
  const int64_t tblocks = (ntarg + bt - 1) / bt;
  const int64_t zdim = md ? (nd + far_md_group(variant, nd) - 1) / far_md_group(variant, nd) : nd;
  const double slots = double(num_sms) * std::max(blocks_per_sm, 1) * waves;
  int64_t s = std::max<int64_t>(1, int64_t(slots / double(tblocks * zdim) + 0.5));
  s = std::min<int64_t>(s, std::max<int64_t>(1, (nptso + kFarTile - 1) / kFarTile));
  // drop chunks that the tile rounding would leave empty
  int64_t chunk = (nptso + s - 1) / s;
  chunk = ((chunk + kFarTile - 1) / kFarTile) * kFarTile;
  return int((nptso + chunk - 1) / chunk);
}

cudaError_t launch_combine(const Geometry& g, const Near& nr, const KParams& kp,
                           const MatvecArgs& a, cudaStream_t st) {
  if (g.ntarg == 0) return cudaSuccess;
  const int threads = kCombineThreads;
  const int64_t blocks = (g.ntarg * 32 + threads - 1) / threads;
  const dim3 grid(static_cast<unsigned>(blocks)), block(threads);
  auto go = [&](auto kern, const auto* w) {
    kern<<<grid, block, 0, st>>>(g, nr, w, a.sigma, a.partial, a.nchunks, a.pot, a.nd);
  };
  auto by_mode = [&](auto one, auto md4, auto wide, const auto* w) {
    switch (combine_mode(a.nd)) {
      case kCombineOne: go(one, w); break;
      case kCombineMd4: go(md4, w); break;
      default: go(wide, w); break;
    }
  };
  const float* wf = static_cast<const float*>(a.weff);
  const double* wd = static_cast<const double*>(a.weff);
  if (kp.kind == 1) {
    if (a.weff_f32)
      by_mode(combine_kernel<1, float, 0>, combine_kernel<1, float, 1>,
              combine_kernel<1, float, 2>, wf);
    else
      by_mode(combine_kernel<1, double, 0>, combine_kernel<1, double, 1>,
              combine_kernel<1, double, 2>, wd);
  } else {
    if (a.weff_f32)
      by_mode(combine_kernel<0, float, 0>, combine_kernel<0, float, 1>,
              combine_kernel<0, float, 2>, wf);
    else
      by_mode(combine_kernel<0, double, 0>, combine_kernel<0, double, 1>,
              combine_kernel<0, double, 2>, wd);
  }
  count();
  return cudaGetLastError();
}

cudaError_t launch_fold(const Geometry& g, const Near& nr, const KParams& kp, const double* wnear,
                        void* weff, int match32, cudaStream_t st, int64_t k0, int64_t k1) {
  if (k1 < 0) k1 = nr.nnz;
  if (k1 <= k0) return cudaSuccess;
  const int warps = 4;
  const size_t sh = size_t(warps) * g.max_nf * 2 * sizeof(double);
  if (sh > 48 * 1024) return cudaErrorInvalidValue;  // max_nf <= 289 keeps this <= 18.5 KB
  const dim3 grid(static_cast<unsigned>((k1 - k0 + warps - 1) / warps)), block(32 * warps);
  if (kp.kind == 1) {
    if (match32 == 2)
      fold_kernel<1, 2, float><<<grid, block, sh, st>>>(g, nr, kp, wnear, (float*)weff, k0, k1);
    else if (match32)
      fold_kernel<1, 1, float><<<grid, block, sh, st>>>(g, nr, kp, wnear, (float*)weff, k0, k1);
    else
      fold_kernel<1, 0, double><<<grid, block, sh, st>>>(g, nr, kp, wnear, (double*)weff, k0, k1);
  } else {
    if (match32 == 2)
      fold_kernel<0, 2, float><<<grid, block, sh, st>>>(g, nr, kp, wnear, (float*)weff, k0, k1);
    else if (match32)
      fold_kernel<0, 1, float><<<grid, block, sh, st>>>(g, nr, kp, wnear, (float*)weff, k0, k1);
    else
      fold_kernel<0, 0, double><<<grid, block, sh, st>>>(g, nr, kp, wnear, (double*)weff, k0, k1);
  }
  count();
  return cudaGetLastError();
}

cudaError_t launch_to_f32(const double* in, float* out, int64_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  to_f32_kernel<<<grid_for(n, 256), 256, 0, st>>>(in, out, n);
  count();
  return cudaGetLastError();
}

cudaError_t launch_pack_strengths(int kind, int precision, int64_t ns, const double* charge,
                                  const double* dipstr, void* str, cudaStream_t st,
                                  const int32_t* sdest) {
  if (ns == 0) return cudaSuccess;
  const int b = grid_for(ns, 256);
  if (precision == 1) {
    if (kind == 1)
      pack_strengths_kernel<float, 1><<<b, 256, 0, st>>>(charge, dipstr, ns, (float*)str, sdest);
    else
      pack_strengths_kernel<float, 0><<<b, 256, 0, st>>>(charge, dipstr, ns, (float*)str, sdest);
  } else {
    if (kind == 1)
      pack_strengths_kernel<double, 1><<<b, 256, 0, st>>>(charge, dipstr, ns, (double*)str, sdest);
    else
      pack_strengths_kernel<double, 0><<<b, 256, 0, st>>>(charge, dipstr, ns, (double*)str, sdest);
  }
  count();
  return cudaGetLastError();
}

cudaError_t launch_reduce_partials(int kind, const double* partial, int nchunks, int64_t ntarg,
                                   double* pot, cudaStream_t st) {
  if (ntarg == 0) return cudaSuccess;
  if (kind == 1)
    reduce_partials_kernel<1><<<grid_for(ntarg, 256), 256, 0, st>>>(partial, nchunks, ntarg, pot);
  else
    reduce_partials_kernel<0><<<grid_for(ntarg, 256), 256, 0, st>>>(partial, nchunks, ntarg, pot);
  count();
  return cudaGetLastError();
}

cudaError_t launch_mdot(const double* V, int64_t ldv, int m, const double* w, const double* wts,
                        int nd, int cplx, const Segs& sg, double* partial, double* out,
                        cudaStream_t st) {
  if (m <= 0) return cudaSuccess;
  if (nd < 1 || nd > 256) return cudaErrorInvalidValue;
  const int threads = (256 / nd) * nd;
  if (cplx)
    mdot_partial_kernel<1><<<sg.nchunk, threads, 0, st>>>(V, ldv, m, w, wts, nd, sg, partial);
  else
    mdot_partial_kernel<0><<<sg.nchunk, threads, 0, st>>>(V, ldv, m, w, wts, nd, sg, partial);
  mdot_final_kernel<<<m * sg.nseg * nd, 256, 0, st>>>(partial, nd, sg, out);
  count(2);
  return cudaGetLastError();
}

cudaError_t launch_maxpy(const double* V, int64_t ldv, int m, const double* h, double* w,
                         int64_t n, int nd, int cplx, const Segs& sg, cudaStream_t st) {
  if (m <= 0) return cudaSuccess;
  if (cplx)
    maxpy_kernel<1><<<grid_for(n, 256), 256, 0, st>>>(V, ldv, m, h, w, n, nd, sg);
  else
    maxpy_kernel<0><<<grid_for(n, 256), 256, 0, st>>>(V, ldv, m, h, w, n, nd, sg);
  count();
  return cudaGetLastError();
}

cudaError_t launch_dscale(const double* x, double* y, const double* s, int64_t n, int nd, int cplx,
                          const Segs& sg, cudaStream_t st) {
  if (cplx)
    dscale_kernel<1><<<grid_for(n, 256), 256, 0, st>>>(x, y, s, n, nd, sg);
  else
    dscale_kernel<0><<<grid_for(n, 256), 256, 0, st>>>(x, y, s, n, nd, sg);
  count();
  return cudaGetLastError();
}

cudaError_t launch_axpby(const double* x, double* y, double ar, double ai, double br, double bi,
                         int64_t n, int cplx, cudaStream_t st) {
  if (cplx)
    axpby_kernel<1><<<grid_for(n, 256), 256, 0, st>>>(x, y, ar, ai, br, bi, n);
  else
    axpby_kernel<0><<<grid_for(n, 256), 256, 0, st>>>(x, y, ar, ai, br, bi, n);
  count();
  return cudaGetLastError();
}

cudaError_t launch_axpbys(const double* x, double* y, const double* a, double br, double bi,
                          int64_t n, int nd, int cplx, const Segs& sg, cudaStream_t st) {
  if (cplx)
    axpbys_kernel<1><<<grid_for(n, 256), 256, 0, st>>>(x, y, a, br, bi, n, nd, sg);
  else
    axpbys_kernel<0><<<grid_for(n, 256), 256, 0, st>>>(x, y, a, br, bi, n, nd, sg);
  count();
  return cudaGetLastError();
}

// ---- GMRES least squares on the device (FP64) -------------------------------
// Complex values as (re, im) pairs; one thread per system.
struct Z {
  double r, i;
};
__device__ __forceinline__ Z zmul(Z a, Z b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
__device__ __forceinline__ Z zadd(Z a, Z b) { return {a.r + b.r, a.i + b.i}; }
__device__ __forceinline__ Z zconj(Z a) { return {a.r, -a.i}; }
__device__ __forceinline__ Z zdiv(Z a, Z b) {
  const double d = b.r * b.r + b.i * b.i;
  return {(a.r * b.r + a.i * b.i) / d, (a.i * b.r - a.r * b.i) / d};
}
__device__ __forceinline__ Z zld(const double* p) { return {p[0], p[1]}; }
__device__ __forceinline__ void zst(double* p, Z v) {
  p[0] = v.r;
  p[1] = v.i;
}

// Iteration it of every active system: the new Hessenberg column
// H(0..it, it) = h1 + h2 (the two Gram-Schmidt passes) with zid on the
// diagonal, the previous Givens rotations applied, the new rotation
// (zrotmat_gmres, rotmat_gmres.f:60-100) against the norm of the new
// vector, the rotated residual vector s, the residual estimate
// |s(it+1)| / ||rhs||, and the stopping test; scale = 1/||w|| for the
// systems that go on (0 for the others).  done[q]: 0 active, > 0 iterations
// taken, < 0 zero right-hand side; brk[q] = 1 on a NaN (breakdown).
__global__ void gmres_givens_kernel(int it, int M, int nsys, const double* __restrict__ h1,
                                    const double* __restrict__ h2,
                                    const double* __restrict__ nrm,
                                    const double* __restrict__ zid, double* __restrict__ H,
                                    double* __restrict__ cs, double* __restrict__ sn,
                                    double* __restrict__ sv, const double* __restrict__ bnorm,
                                    const double* __restrict__ eps, int64_t* __restrict__ done,
                                    int* __restrict__ brk, double* __restrict__ errs,
                                    double* __restrict__ scale) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsys) return;
  scale[2 * q] = 0.0;
  scale[2 * q + 1] = 0.0;
  if (done[q] != 0) return;
  double* Hq = H + 2 * (size_t(q) * M + it) * (M + 1);  // column it of system q
  for (int k = 0; k <= it; ++k)
    zst(Hq + 2 * k, zadd(zld(h1 + 2 * (size_t(k) * nsys + q)), zld(h2 + 2 * (size_t(k) * nsys + q))));
  zst(Hq + 2 * it, zadd(zld(Hq + 2 * it), zld(zid + 2 * q)));
  const double wnrm = sqrt(fmax(nrm[2 * q], 0.0));
  double* cq = cs + 2 * size_t(q) * M;
  double* sq = sn + 2 * size_t(q) * M;
  double* vq = sv + 2 * size_t(q) * (M + 1);
  for (int k = 0; k < it; ++k) {
    const Z c = zld(cq + 2 * k), s = zld(sq + 2 * k);
    const Z a = zld(Hq + 2 * k), b = zld(Hq + 2 * (k + 1));
    zst(Hq + 2 * k, zadd(zmul(c, a), zmul(zconj(s), b)));
    const Z ms = {-s.r, -s.i};
    zst(Hq + 2 * (k + 1), zadd(zmul(ms, a), zmul(c, b)));
  }
  const Z a = zld(Hq + 2 * it);
  Z c, s;
  if (a.r == 0.0 && a.i == 0.0) {
    c = {0.0, 0.0};
    s = {1.0, 0.0};
  } else {
    const Z t = zdiv(Z{wnrm, 0.0}, a);
    const double cr = 1.0 / sqrt(1.0 + t.r * t.r + t.i * t.i);
    c = {cr, 0.0};
    s = {t.r * cr, t.i * cr};
  }
  zst(cq + 2 * it, c);
  zst(sq + 2 * it, s);
  zst(Hq + 2 * it, zadd(zmul(c, a), zmul(zconj(s), Z{wnrm, 0.0})));
  const Z v = zld(vq + 2 * it);
  zst(vq + 2 * (it + 1), Z{-(s.r * v.r - s.i * v.i), -(s.r * v.i + s.i * v.r)});
  zst(vq + 2 * it, zmul(c, v));
  const Z vn = zld(vq + 2 * (it + 1));
  const double err = bnorm[q] > 0.0 ? sqrt(vn.r * vn.r + vn.i * vn.i) / bnorm[q] : 0.0;
  errs[size_t(q) * (M + 1) + it] = err;
  if (!(err == err) || !(wnrm == wnrm)) {
    brk[q] = 1;
    done[q] = it + 1;
    return;
  }
  // the new Krylov vector is normalised also when the system stops here: it
  // is the last vector of the basis that carries the residual vector
  if (wnrm > 0.0) scale[2 * q] = 1.0 / wnrm;
  if (err <= eps[q] || it == M - 1 || wnrm == 0.0) done[q] = it + 1;
}

// y = triu(H)^-1 s over the done[q] iterations of system q, written as the
// combination coefficients coef[2 (j nsys + q)], j < mused (zero past done[q]).
__global__ void gmres_backsolve_kernel(int M, int nsys, int mused, const double* __restrict__ H,
                                       const double* __restrict__ sv,
                                       const int64_t* __restrict__ done,
                                       double* __restrict__ coef) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsys) return;
  const int k = done[q] > 0 ? int(done[q]) : 0;
  for (int j = k; j < mused; ++j) zst(coef + 2 * (size_t(j) * nsys + q), Z{0.0, 0.0});
  const double* Hq = H + 2 * size_t(q) * M * (M + 1);
  const double* vq = sv + 2 * size_t(q) * (M + 1);
  for (int j = k - 1; j >= 0; --j) {
    Z acc = zld(vq + 2 * j);
    for (int l = j + 1; l < k; ++l) {
      const Z h = zld(Hq + 2 * (size_t(l) * (M + 1) + j));
      const Z y = zld(coef + 2 * (size_t(l) * nsys + q));
      acc = {acc.r - (h.r * y.r - h.i * y.i), acc.i - (h.r * y.i + h.i * y.r)};
    }
    zst(coef + 2 * (size_t(j) * nsys + q), zdiv(acc, zld(Hq + 2 * (size_t(j) * (M + 1) + j))));
  }
}

// Coefficients z (j = 0..done[q], zero up to mcols) of the GMRES residual
// vector r0 - A V y = V Q^H (0, ..., 0, g_k)^T in the Krylov basis: the
// last rotated residual entry g_k carried back through the rotations
// (G_i^H on entries i, i+1, last rotation first).
__global__ void gmres_resvec_kernel(int M, int nsys, int mcols, const double* __restrict__ cs,
                                    const double* __restrict__ sn,
                                    const double* __restrict__ sv,
                                    const int64_t* __restrict__ done, double* __restrict__ z) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsys) return;
  const int k = done[q] > 0 ? int(done[q]) : 0;
  for (int j = k + 1; j < mcols; ++j) zst(z + 2 * (size_t(j) * nsys + q), Z{0.0, 0.0});
  if (k == 0) {
    zst(z + 2 * size_t(q), Z{0.0, 0.0});
    return;
  }
  const double* cq = cs + 2 * size_t(q) * M;
  const double* sq = sn + 2 * size_t(q) * M;
  Z hi = zld(sv + 2 * (size_t(q) * (M + 1) + k));  // z_k = g_k
  for (int i = k - 1; i >= 0; --i) {
    // (z_i, z_{i+1}) <- (c z_i - conj(s) z_{i+1}, s z_i + c z_{i+1}), z_i = 0
    const Z c = zld(cq + 2 * i), s = zld(sq + 2 * i);
    zst(z + 2 * (size_t(i + 1) * nsys + q), zmul(c, hi));
    hi = Z{-(s.r * hi.r + s.i * hi.i), -(s.r * hi.i - s.i * hi.r)};
  }
  zst(z + 2 * size_t(q), hi);
}

cudaError_t launch_gmres_resvec(int M, int nsys, int mcols, const double* cs, const double* sn,
                                const double* sv, const int64_t* done, double* z,
                                cudaStream_t st) {
  gmres_resvec_kernel<<<(nsys + 63) / 64, 64, 0, st>>>(M, nsys, mcols, cs, sn, sv, done, z);
  count();
  return cudaGetLastError();
}

// kx += r - rn - zid d: the operator applied to a refinement correction d,
// taken from the inner solve's own right-hand side r and residual rn.
template <int CPLX>
__global__ void kx_update_kernel(double* __restrict__ kx, const double* __restrict__ r,
                                 const double* __restrict__ rn, const double* __restrict__ d,
                                 const double* __restrict__ zid, int64_t n, int nd, Segs sg) {
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int sy = sys_of(sg, e, nd);
    const double zr = zid[2 * sy], zi = zid[2 * sy + 1];
    if (CPLX) {
      const double dr = d[2 * e], di = d[2 * e + 1];
      kx[2 * e] += r[2 * e] - rn[2 * e] - (zr * dr - zi * di);
      kx[2 * e + 1] += r[2 * e + 1] - rn[2 * e + 1] - (zr * di + zi * dr);
    } else {
      kx[e] += r[e] - rn[e] - zr * d[e];
    }
  }
}

cudaError_t launch_kx_update(double* kx, const double* r, const double* rn, const double* d,
                             const double* zid, int64_t n, int nd, int cplx, const Segs& sg,
                             cudaStream_t st) {
  if (cplx)
    kx_update_kernel<1><<<grid_for(n, 256), 256, 0, st>>>(kx, r, rn, d, zid, n, nd, sg);
  else
    kx_update_kernel<0><<<grid_for(n, 256), 256, 0, st>>>(kx, r, rn, d, zid, n, nd, sg);
  count();
  return cudaGetLastError();
}

cudaError_t launch_gmres_givens(int it, int M, int nsys, const double* h1, const double* h2,
                                const double* nrm, const double* zid, double* H, double* cs,
                                double* sn, double* sv, const double* bnorm, const double* eps,
                                int64_t* done, int* brk, double* errs, double* scale,
                                cudaStream_t st) {
  gmres_givens_kernel<<<(nsys + 63) / 64, 64, 0, st>>>(it, M, nsys, h1, h2, nrm, zid, H, cs, sn, sv,
                                                       bnorm, eps, done, brk, errs, scale);
  count();
  return cudaGetLastError();
}

cudaError_t launch_gmres_backsolve(int M, int nsys, int mused, const double* H, const double* sv,
                                   const int64_t* done, double* coef, cudaStream_t st) {
  gmres_backsolve_kernel<<<(nsys + 63) / 64, 64, 0, st>>>(M, nsys, mused, H, sv, done, coef);
  count();
  return cudaGetLastError();
}

cudaError_t launch_combo(const double* V, int64_t ldv, int m, const double* c, double* y,
                         int64_t n, int nd, int cplx, const Segs& sg, cudaStream_t st) {
  if (cplx)
    combo_kernel<1><<<grid_for(n, 256), 256, 0, st>>>(V, ldv, m, c, y, n, nd, sg);
  else
    combo_kernel<0><<<grid_for(n, 256), 256, 0, st>>>(V, ldv, m, c, y, n, nd, sg);
  count();
  return cudaGetLastError();
}

// FFMA throughput probe: every thread runs 8 independent FMA chains; the
// result is stored so the work cannot be removed.  flops = 2 * 8 * iters
// per thread.
__global__ void ffma_peak_kernel(float* out, int iters, float a, float b) {
  float x0 = threadIdx.x * 1e-3f, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5,
        x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 = fmaf(x0, a, b);
      x1 = fmaf(x1, a, b);
      x2 = fmaf(x2, a, b);
      x3 = fmaf(x3, a, b);
      x4 = fmaf(x4, a, b);
      x5 = fmaf(x5, a, b);
      x6 = fmaf(x6, a, b);
      x7 = fmaf(x7, a, b);
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

cudaError_t launch_ffma_peak(float* out, int blocks, int threads, int iters, cudaStream_t st) {
  ffma_peak_kernel<<<blocks, threads, 0, st>>>(out, iters, 0.9999999f, 1e-7f);
  count();
  return cudaGetLastError();
}

// MUFU throughput probe: 8 independent reciprocal-square-root chains per
// thread (rsqrt.approx.ftz.f32, one MUFU operation each; the chains settle at
// 1).  ops = 16 * 8 * iters per thread.
__global__ void mufu_peak_kernel(float* out, int iters) {
  float x0 = 1.0f + threadIdx.x * 1e-3f, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4,
        x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      asm("rsqrt.approx.ftz.f32 %0, %0;" : "+f"(x0));
      asm("rsqrt.approx.ftz.f32 %0, %0;" : "+f"(x1));
      asm("rsqrt.approx.ftz.f32 %0, %0;" : "+f"(x2));
      asm("rsqrt.approx.ftz.f32 %0, %0;" : "+f"(x3));
      asm("rsqrt.approx.ftz.f32 %0, %0;" : "+f"(x4));
      asm("rsqrt.approx.ftz.f32 %0, %0;" : "+f"(x5));
      asm("rsqrt.approx.ftz.f32 %0, %0;" : "+f"(x6));
      asm("rsqrt.approx.ftz.f32 %0, %0;" : "+f"(x7));
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

cudaError_t launch_mufu_peak(float* out, int blocks, int threads, int iters, cudaStream_t st) {
  mufu_peak_kernel<<<blocks, threads, 0, st>>>(out, iters);
  count();
  return cudaGetLastError();
}

int64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }
void note_launches(int64_t n) { count(n); }

}  // namespace dev
}  // namespace bie
