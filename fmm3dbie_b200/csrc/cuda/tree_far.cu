// Hierarchical far field: device lists and kernels (see tree_far.h and
// host/tree.h for the method).
//
// HBM layout (all built once per plan and precision):
//   sorted targets tx,ty,tz f64 and tperm (sorted -> original index);
//   sorted oversampled sources sx..snz f64 (strengths arrive in this order);
//   target nodes TNodeD: parent, proxy grid, target range, first target
//     proxy, and two entry ranges: pent (PP and PC: sources seen by the
//     node's targets) and cent (CP and CC: sources seen by its proxies);
//   entries EntryD {kind, b, e}: kind 0/1 = sorted sources [b, e) with /
//     without the self-interaction test, kind 2 = source proxies [b, e);
//   proxy coordinates of the source nodes (spx..) and target nodes (tpx..);
//   upward work items (source node chunk -> partial proxy charges) and the
//     per-node reduction table.
// Per matvec: proxy charges qhat and proxy potentials phi (far precision,
// complex interleaved, nd densities), partial proxy charges (f64).
//
// Kernels (one thread block per work item, densities on grid y):
//   tree_up_kernel     partial proxy charges of a chunk of <= 2048 sources:
//                      thread (i, j, l-range) of the grid accumulates
//                      sum_s c_s Lx_i Ly_j Lz_l + d_s n_s . grad(Lx_i Ly_j Lz_l);
//   tree_reduce_kernel sums the chunks of each node;
//   tree_eval_kernel   <PROXYT = 1> proxy potentials of 128 proxies of a
//                      target node from its CP and CC entries;
//                      <PROXYT = 0> the far field of one target leaf (<= 128
//                      targets): the PP and PC entries of the leaf and of
//                      every ancestor, then the ancestors' proxy potentials
//                      interpolated to the targets.
// Pair arithmetic is that of the direct far kernels (pair.cuh); FP32
// coordinates are centred on the work item's box centre.
#include "tree_far.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <type_traits>

#include "pair.cuh"

namespace bie {
namespace dev {
namespace {

constexpr int kP = tree::kMaxP;

struct TNodeD {
  int parent, np0, np1, np2;
  int64_t b, e, tpoff, pe0, pe1, ce0, ce1;
  double lo[3], hi[3];
};
struct EntryD {
  int kind, b, e, pad;
};
struct UpItemD {
  int64_t b, e, ubase;
  int np0, np1, np2, pad;
  double lo[3], hi[3];
};
struct RedD {
  int64_t sp0, ubase;
  int nitems, P;
};
struct TreeArgs {
  const TNodeD* tn;
  const EntryD* pent;
  const EntryD* cent;
  const int* leaves;
  const int2* pitems;
  const double *tx, *ty, *tz;
  const int64_t* tperm;
  const double *sx, *sy, *sz, *snx, *sny, *snz;
  const double *tpx, *tpy, *tpz, *spx, *spy, *spz;
};

// Chebyshev points of the second kind and Lagrange normalisations for
// p = 1 .. kP nodes (row p).
__constant__ double cNode[(kP + 1) * kP];
__constant__ double cWt[(kP + 1) * kP];

// L[j] = Lagrange basis j of the p-point grid at u in [-1, 1] (product form:
// w_j prod_{i != j} (u - x_i), stable for u at or near a node).
template <typename R>
__device__ __forceinline__ void lagrange(int p, R u, R* L) {
  R diff[kP];
#pragma unroll
  for (int i = 0; i < kP; ++i) diff[i] = i < p ? u - R(cNode[p * kP + i]) : R(1);
  R pre = R(1);
#pragma unroll
  for (int j = 0; j < kP; ++j) {
    L[j] = pre;
    pre *= diff[j];
  }
  R suf = R(1);
#pragma unroll
  for (int j = kP - 1; j >= 0; --j)
    if (j < p) {
      L[j] *= suf * R(cWt[p * kP + j]);
      suf *= diff[j];
    }
}

// Values and u-derivatives of the basis.
template <typename R>
__device__ __forceinline__ void lagrange_d(int p, R u, R* L, R* D) {
  R diff[kP];
#pragma unroll
  for (int i = 0; i < kP; ++i) diff[i] = i < p ? u - R(cNode[p * kP + i]) : R(1);
  R pre = R(1), dpre = R(0);
#pragma unroll
  for (int j = 0; j < kP; ++j) {
    L[j] = pre;
    D[j] = dpre;
    dpre = fma(dpre, diff[j], pre);
    pre *= diff[j];
  }
  R suf = R(1), dsuf = R(0);
#pragma unroll
  for (int j = kP - 1; j >= 0; --j)
    if (j < p) {
      const R w = R(cWt[p * kP + j]);
      D[j] = fma(D[j], suf, L[j] * dsuf) * w;
      L[j] *= suf * w;
      dsuf = fma(dsuf, diff[j], suf);
      suf *= diff[j];
    }
}

// ---------------------------------------------------------------------------
// upward pass
// ---------------------------------------------------------------------------
constexpr int kUpThreads = 128, kUpTile = 32;
constexpr int64_t kUpChunk = 2048;

// SIG = false: str holds each source's (charge, dipole) strengths per
// density; SIG = true: they are formed as (a_s sigma_m, b_s sigma_m) from
// the oversampled densities sig and the per-source constants ab.
template <int KIND, typename R, bool SIG>
__global__ void __launch_bounds__(kUpThreads)
    tree_up_kernel(const UpItemD* __restrict__ items, TreeArgs ta, const R* __restrict__ str,
                   const R* __restrict__ sig, const R* __restrict__ ab, int nd,
                   double* __restrict__ up_part) {
  constexpr int SW = KIND == 1 ? 4 : 2;
  constexpr int C = KIND == 1 ? 2 : 1;
  __shared__ R sL[3][kP][kUpTile];
  __shared__ R sD[3][kP][kUpTile];  // derivative along the side times the normal component
  __shared__ R sS[kUpTile][SW];
  const UpItemD it = items[blockIdx.x];
  const int m = blockIdx.y, tid = threadIdx.x;
  const int npd[3] = {it.np0, it.np1, it.np2};
  const int pxy = it.np0 * it.np1, pz = it.np2;
  const int lg = min(max(kUpThreads / pxy, 1), pz);  // l-groups per (i, j)
  const int lc = (pz + lg - 1) / lg;                 // l per group
  const int slots = pxy * lg;
  double ctr[3], h[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    ctr[d] = 0.5 * (it.lo[d] + it.hi[d]);
    h[d] = 0.5 * (it.hi[d] - it.lo[d]);
  }
  for (int base = 0; base < slots; base += kUpThreads) {
    const int slot = base + tid;
    const bool act = slot < slots;
    const int ij = act ? slot % pxy : 0, grp = act ? slot / pxy : 0;
    const int i = ij / it.np1, j = ij - (ij / it.np1) * it.np1;
    const int l0 = grp * lc;
    const int nl = act ? max(0, min(lc, pz - l0)) : 0;
    double accr[kP], acci[kP];
#pragma unroll
    for (int l = 0; l < kP; ++l) accr[l] = acci[l] = 0.0;
    for (int64_t sb = it.b; sb < it.e; sb += kUpTile) {
      const int ns = int(it.e - sb < kUpTile ? it.e - sb : kUpTile);
      __syncthreads();
      if (tid < 3 * kUpTile) {
        const int s = tid % kUpTile, d = tid / kUpTile;
        if (s < ns) {
          const int64_t src = sb + s;
          const double x = d == 0 ? ta.sx[src] : (d == 1 ? ta.sy[src] : ta.sz[src]);
          const double nrm = d == 0 ? ta.snx[src] : (d == 1 ? ta.sny[src] : ta.snz[src]);
          const R u = h[d] > 0.0 ? R((x - ctr[d]) / h[d]) : R(0);
          const R sc = h[d] > 0.0 ? R(nrm / h[d]) : R(0);
          R L[kP], D[kP];
          lagrange_d(npd[d], u, L, D);
#pragma unroll
          for (int q = 0; q < kP; ++q)
            if (q < npd[d]) {
              sL[d][q][s] = L[q];
              sD[d][q][s] = D[q] * sc;
            }
        }
      }
      if constexpr (SIG) {
        for (int q = tid; q < ns; q += kUpThreads) {
          const size_t si = size_t(sb + q);
          const R* a = ab + si * SW;
          const R* sg = sig + (si * nd + m) * C;
          if constexpr (KIND == 1) {
            const R sr = sg[0], sim = sg[1];
            sS[q][0] = fma(a[0], sr, -a[1] * sim);
            sS[q][1] = fma(a[0], sim, a[1] * sr);
            sS[q][2] = fma(a[2], sr, -a[3] * sim);
            sS[q][3] = fma(a[2], sim, a[3] * sr);
          } else {
            sS[q][0] = a[0] * sg[0];
            sS[q][1] = a[1] * sg[0];
          }
        }
      } else {
        for (int q = tid; q < ns * SW; q += kUpThreads)
          sS[q / SW][q % SW] = str[(size_t(sb + q / SW) * nd + m) * SW + q % SW];
      }
      __syncthreads();
      if (nl > 0) {
        R tr[kP], ti[kP];
#pragma unroll
        for (int l = 0; l < kP; ++l) tr[l] = ti[l] = R(0);
        for (int s = 0; s < ns; ++s) {
          const R lx = sL[0][i][s], dx = sD[0][i][s], ly = sL[1][j][s], dy = sD[1][j][s];
          const R v = lx * ly, gxy = fma(dx, ly, lx * dy);
          R ar, ai = R(0), br, bi = R(0);
          if constexpr (KIND == 1) {
            ar = fma(sS[s][0], v, sS[s][2] * gxy);
            ai = fma(sS[s][1], v, sS[s][3] * gxy);
            br = sS[s][2] * v;
            bi = sS[s][3] * v;
          } else {
            ar = fma(sS[s][0], v, sS[s][1] * gxy);
            br = sS[s][1] * v;
          }
#pragma unroll
          for (int l = 0; l < kP; ++l)
            if (l < nl) {
              const R lz = sL[2][l0 + l][s], dz = sD[2][l0 + l][s];
              tr[l] = fma(ar, lz, fma(br, dz, tr[l]));
              if constexpr (KIND == 1) ti[l] = fma(ai, lz, fma(bi, dz, ti[l]));
            }
        }
#pragma unroll
        for (int l = 0; l < kP; ++l) {
          accr[l] += double(tr[l]);
          acci[l] += double(ti[l]);
        }
      }
    }
#pragma unroll
    for (int l = 0; l < kP; ++l)
      if (l < nl) {
        const int64_t k = int64_t(i * it.np1 + j) * pz + l0 + l;
        double* o = up_part + ((it.ubase + k) * nd + m) * C;
        o[0] = accr[l];
        if constexpr (C == 2) o[1] = acci[l];
      }
  }
}

// qhat[(sp0 + k) nd + m] = sum over the node's chunks of the partial charges.
template <typename R, int C>
__global__ void tree_reduce_kernel(const RedD* __restrict__ reds, const double* __restrict__ up_part,
                                   int nd, R* __restrict__ qhat) {
  const RedD r = reds[blockIdx.x];
  const int per = nd * C;
  for (int q = threadIdx.x; q < r.P * per; q += blockDim.x) {
    const int k = q / per, rem = q - k * per;
    double s = 0.0;
    for (int c = 0; c < r.nitems; ++c) s += up_part[(r.ubase + int64_t(c) * r.P + k) * per + rem];
    qhat[(r.sp0 + k) * per + rem] = R(s);
  }
}

// ---------------------------------------------------------------------------
// list evaluation
// ---------------------------------------------------------------------------
constexpr int kEvThreads = 128, kEvTile = 128;

template <int KIND, typename R, bool CK, bool PROXYT>
__global__ void __launch_bounds__(kEvThreads)
    tree_eval_kernel(TreeArgs ta, KParams kp, const R* __restrict__ str,
                     const R* __restrict__ qhat, R* __restrict__ phi,
                     double* __restrict__ partial, int nd) {
  using R2 = typename Vec<R>::T2;
  using R4 = typename Vec<R>::T4;
  constexpr int SW = KIND == 1 ? 4 : 2;
  constexpr int C = KIND == 1 ? 2 : 1;
  __shared__ R4 sg0[kEvTile];
  __shared__ R2 sg1[kEvTile];
  __shared__ R4 sst[kEvTile];
  __shared__ R2 sphi[PROXYT ? 1 : tree::kMaxProxies];
  __shared__ double2 stab[sizeof(R) == 8 && KIND == 1 ? kFarTrigN : 1];
  const double2* tab = nullptr;
  if constexpr (sizeof(R) == 8 && KIND == 1) {
    fill_far_trig_table(stab);  // published by the first __syncthreads below
    tab = stab;
  }
  const int tid = threadIdx.x, m = blockIdx.y;
  int node;
  int64_t k0 = 0;
  if constexpr (PROXYT) {
    const int2 pi = ta.pitems[blockIdx.x];
    node = pi.x;
    k0 = pi.y;
  } else {
    node = ta.leaves[blockIdx.x];
  }
  const TNodeD tn = ta.tn[node];
  // FP32 shifts coordinates to the node centre; FP64 keeps them absolute so
  // that t - s of a close pair stays exact (as the direct far kernels do)
  constexpr bool kShift = sizeof(R) == 4;
  const double cx = kShift ? 0.5 * (tn.lo[0] + tn.hi[0]) : 0.0,
               cy = kShift ? 0.5 * (tn.lo[1] + tn.hi[1]) : 0.0,
               cz = kShift ? 0.5 * (tn.lo[2] + tn.hi[2]) : 0.0;
  bool act, wact;  // this thread's / this warp's targets exist
  double x = cx, y = cy, z = cz;
  if constexpr (PROXYT) {
    const int64_t P = int64_t(tn.np0) * tn.np1 * tn.np2;
    act = k0 + tid < P;
    wact = k0 + (tid & ~31) < P;
    if (act) {
      const int64_t q = tn.tpoff + k0 + tid;
      x = ta.tpx[q];
      y = ta.tpy[q];
      z = ta.tpz[q];
    }
  } else {
    act = tn.b + tid < tn.e;
    wact = tn.b + (tid & ~31) < tn.e;
    if (act) {
      const int64_t q = tn.b + tid;
      x = ta.tx[q];
      y = ta.ty[q];
      z = ta.tz[q];
    }
  }
  const R tx = R(x - cx), ty = R(y - cy), tz = R(z - cz);
  const R thr2 = R(kp.thresh * kp.thresh), k = R(kp.kr), kim = R(kp.ki);
  double accr = 0.0, acci = 0.0;
  int n = node;
  int64_t e0 = PROXYT ? tn.ce0 : tn.pe0, e1 = PROXYT ? tn.ce1 : tn.pe1;
  const EntryD* ents = PROXYT ? ta.cent : ta.pent;
  while (true) {
    for (int64_t q = e0; q < e1; ++q) {
      const EntryD en = ents[q];
      for (int sb = en.b; sb < en.e; sb += kEvTile) {
        const int ns = min(kEvTile, en.e - sb);
        __syncthreads();
        for (int qq = tid; qq < ns; qq += kEvThreads) {
          const int s = sb + qq;
          if (en.kind == 2) {
            sg0[qq] = R4{R(ta.spx[s] - cx), R(ta.spy[s] - cy), R(ta.spz[s] - cz), R(0)};
            const R* qp = qhat + (size_t(s) * nd + m) * C;
            sst[qq] = R4{qp[0], C == 2 ? qp[C - 1] : R(0), R(0), R(0)};
          } else {
            sg0[qq] = R4{R(ta.sx[s] - cx), R(ta.sy[s] - cy), R(ta.sz[s] - cz), R(ta.snx[s])};
            sg1[qq] = R2{R(ta.sny[s]), R(ta.snz[s])};
            const R* sp = str + (size_t(s) * nd + m) * SW;
            if constexpr (SW == 4)
              sst[qq] = R4{sp[0], sp[1], sp[2], sp[3]};
            else
              sst[qq] = R4{sp[0], sp[1], R(0), R(0)};
          }
        }
        __syncthreads();
        R pr = R(0), pi = R(0);
        if (!wact) {
          // a warp without targets only helps load the tiles
        } else if (en.kind == 2) {
#pragma unroll 4
          for (int j = 0; j < ns; ++j) pair_charge<KIND>(tx, ty, tz, sg0[j], sst[j], k, kim, CK, pr, pi, tab);
        } else if (en.kind == 1) {
#pragma unroll 4
          for (int j = 0; j < ns; ++j) {
            if constexpr (KIND == 1) {
              pair_helm<false>(tx, ty, tz, sg0[j], sg1[j], sst[j], k, kim, thr2, CK, pr, pi, tab);
            } else {
              const R4 s = sst[j];
              pair_lap<R, false>(tx, ty, tz, sg0[j], sg1[j], R2{s.x, s.y}, thr2, pr);
            }
          }
        } else {
#pragma unroll 4
          for (int j = 0; j < ns; ++j) {
            if constexpr (KIND == 1) {
              pair_helm<true>(tx, ty, tz, sg0[j], sg1[j], sst[j], k, kim, thr2, CK, pr, pi, tab);
            } else {
              const R4 s = sst[j];
              pair_lap<R, true>(tx, ty, tz, sg0[j], sg1[j], R2{s.x, s.y}, thr2, pr);
            }
          }
        }
        accr += double(pr);
        acci += double(pi);
      }
    }
    if (PROXYT) break;
    n = ta.tn[n].parent;
    if (n < 0) break;
    e0 = ta.tn[n].pe0;
    e1 = ta.tn[n].pe1;
  }
  if constexpr (!PROXYT) {
    // downward pass: proxy potentials of the leaf's ancestors (and its own)
    for (int a = node; a >= 0; a = ta.tn[a].parent) {
      const TNodeD an = ta.tn[a];
      if (an.tpoff < 0) continue;
      const int P = an.np0 * an.np1 * an.np2;
      __syncthreads();
      for (int q = tid; q < P; q += kEvThreads) {
        const R* pp = phi + (size_t(an.tpoff + q) * nd + m) * C;
        sphi[q] = R2{pp[0], C == 2 ? pp[C - 1] : R(0)};
      }
      __syncthreads();
      if (act) {
        const double h0 = 0.5 * (an.hi[0] - an.lo[0]), h1 = 0.5 * (an.hi[1] - an.lo[1]),
                     h2 = 0.5 * (an.hi[2] - an.lo[2]);
        const R u0 = h0 > 0.0 ? R((x - 0.5 * (an.lo[0] + an.hi[0])) / h0) : R(0);
        const R u1 = h1 > 0.0 ? R((y - 0.5 * (an.lo[1] + an.hi[1])) / h1) : R(0);
        const R u2 = h2 > 0.0 ? R((z - 0.5 * (an.lo[2] + an.hi[2])) / h2) : R(0);
        R Lx[kP], Ly[kP], Lz[kP];
        lagrange(an.np0, u0, Lx);
        lagrange(an.np1, u1, Ly);
        lagrange(an.np2, u2, Lz);
        R sr = R(0), si = R(0);
        for (int i = 0; i < an.np0; ++i)
          for (int j = 0; j < an.np1; ++j) {
            const R w = Lx[i] * Ly[j];
            const R2* ph = sphi + (i * an.np1 + j) * an.np2;
            R tr = R(0), ti = R(0);
#pragma unroll
            for (int l = 0; l < kP; ++l)
              if (l < an.np2) {
                tr = fma(Lz[l], ph[l].x, tr);
                ti = fma(Lz[l], ph[l].y, ti);
              }
            sr = fma(w, tr, sr);
            si = fma(w, ti, si);
          }
        accr += double(sr);
        acci += double(si);
      }
    }
  }
  if (!act) return;
  if constexpr (PROXYT) {
    R* o = phi + (size_t(tn.tpoff + k0 + tid) * nd + m) * C;
    o[0] = R(accr);
    if constexpr (C == 2) o[1] = R(acci);
  } else {
    const int64_t it = ta.tperm[tn.b + tid];
    double* o = partial + (size_t(it) * nd + m) * C;
    o[0] = accr;
    if constexpr (C == 2) o[1] = acci;
  }
}

// Several densities per block (MD of them, densities m0 .. m0 + MD - 1 on
// grid y).  The charge and dipole strengths of a layer potential are both
// proportional to the oversampled density, c_m = a_s sigma_m and
// d_m = b_s sigma_m (a_s = alpha w_s/(4 pi), b_s = beta w_s/(4 pi)), so each
// pair's kernel value K = a_s G + b_s D is formed once from its unit
// responses (pair_helm_unit) and applied to every density with one complex
// multiply-add; proxy charges use G alone.  sig: sigma_over in tree order,
// ab: (a_s, b_s) in tree order.  Otherwise as tree_eval_kernel.
constexpr int kMdTile = 64;

template <int KIND, typename R, bool CK, bool PROXYT, int MD>
__global__ void __launch_bounds__(kEvThreads)
    tree_eval_md_kernel(TreeArgs ta, KParams kp, const R* __restrict__ sig,
                        const R* __restrict__ ab, const R* __restrict__ qhat,
                        R* __restrict__ phi, double* __restrict__ partial, int nd) {
  using R2 = typename Vec<R>::T2;
  using R4 = typename Vec<R>::T4;
  constexpr int SW = KIND == 1 ? 4 : 2;
  constexpr int C = KIND == 1 ? 2 : 1;
  __shared__ R4 sg0[kMdTile];
  __shared__ R2 sg1[kMdTile];
  __shared__ R4 sab[kMdTile];  // (a_s, b_s) of particle sources
  // the densities (or proxy charges) of the list phase and the proxy
  // potentials of the downward phase share one buffer
  constexpr size_t kSstBytes = sizeof(R) * kMdTile * MD * C;
  constexpr size_t kPhiBytes = PROXYT ? 0 : sizeof(R2) * tree::kMaxProxies;
  __shared__ __align__(16) unsigned char sbuf[kSstBytes > kPhiBytes ? kSstBytes : kPhiBytes];
  R(*sst)[MD][C] = reinterpret_cast<R(*)[MD][C]>(sbuf);
  R2* sphi = reinterpret_cast<R2*>(sbuf);
  __shared__ double2 stab[sizeof(R) == 8 && KIND == 1 ? kFarTrigN : 1];
  const double2* tab = nullptr;
  if constexpr (sizeof(R) == 8 && KIND == 1) {
    fill_far_trig_table(stab);  // published by the first __syncthreads below
    tab = stab;
  }
  const int tid = threadIdx.x;
  const int m0 = blockIdx.y * MD;
  const int nm = min(MD, nd - m0);
  int node;
  int64_t k0 = 0;
  if constexpr (PROXYT) {
    const int2 pi = ta.pitems[blockIdx.x];
    node = pi.x;
    k0 = pi.y;
  } else {
    node = ta.leaves[blockIdx.x];
  }
  const TNodeD tn = ta.tn[node];
  // FP32 shifts coordinates to the node centre; FP64 keeps them absolute so
  // that t - s of a close pair stays exact (as the direct far kernels do)
  constexpr bool kShift = sizeof(R) == 4;
  const double cx = kShift ? 0.5 * (tn.lo[0] + tn.hi[0]) : 0.0,
               cy = kShift ? 0.5 * (tn.lo[1] + tn.hi[1]) : 0.0,
               cz = kShift ? 0.5 * (tn.lo[2] + tn.hi[2]) : 0.0;
  bool act, wact;
  double x = cx, y = cy, z = cz;
  if constexpr (PROXYT) {
    const int64_t P = int64_t(tn.np0) * tn.np1 * tn.np2;
    act = k0 + tid < P;
    wact = k0 + (tid & ~31) < P;
    if (act) {
      const int64_t q = tn.tpoff + k0 + tid;
      x = ta.tpx[q];
      y = ta.tpy[q];
      z = ta.tpz[q];
    }
  } else {
    act = tn.b + tid < tn.e;
    wact = tn.b + (tid & ~31) < tn.e;
    if (act) {
      const int64_t q = tn.b + tid;
      x = ta.tx[q];
      y = ta.ty[q];
      z = ta.tz[q];
    }
  }
  const R tx = R(x - cx), ty = R(y - cy), tz = R(z - cz);
  const R thr2 = R(kp.thresh * kp.thresh), k = R(kp.kr), kim = R(kp.ki);
  double accr[MD], acci[MD];
#pragma unroll
  for (int mm = 0; mm < MD; ++mm) accr[mm] = acci[mm] = 0.0;
  int n = node;
  int64_t e0 = PROXYT ? tn.ce0 : tn.pe0, e1 = PROXYT ? tn.ce1 : tn.pe1;
  const EntryD* ents = PROXYT ? ta.cent : ta.pent;
  while (true) {
    for (int64_t q = e0; q < e1; ++q) {
      const EntryD en = ents[q];
      for (int sb = en.b; sb < en.e; sb += kMdTile) {
        const int ns = min(kMdTile, en.e - sb);
        __syncthreads();
        for (int qq = tid; qq < ns; qq += kEvThreads) {
          const int s = sb + qq;
          if (en.kind == 2) {
            sg0[qq] = R4{R(ta.spx[s] - cx), R(ta.spy[s] - cy), R(ta.spz[s] - cz), R(0)};
          } else {
            sg0[qq] = R4{R(ta.sx[s] - cx), R(ta.sy[s] - cy), R(ta.sz[s] - cz), R(ta.snx[s])};
            sg1[qq] = R2{R(ta.sny[s]), R(ta.snz[s])};
            const R* a = ab + size_t(s) * SW;
            sab[qq] = SW == 4 ? R4{a[0], a[1], a[2], a[3]} : R4{a[0], R(0), a[1], R(0)};
          }
        }
        {
          const R* src = en.kind == 2 ? qhat : sig;
          for (int qq = tid; qq < ns * MD * C; qq += kEvThreads) {
            const int sj = qq / (MD * C), rem = qq - sj * (MD * C);
            const int mm = rem / C, c = rem - mm * C;
            sst[sj][mm][c] = mm < nm ? src[(size_t(sb + sj) * nd + m0 + mm) * C + c] : R(0);
          }
        }
        __syncthreads();
        if (!wact) continue;  // a warp without targets only helps load the tiles
        // FP32: tile sums in FP32, added to the FP64 sums after the tile;
        // FP64: straight into the FP64 sums
        constexpr bool kTileSums = sizeof(R) == 4;
        R trs[kTileSums ? MD : 1], tis[kTileSums ? MD : 1];
        auto tr = [&](int mm) -> R& {
          if constexpr (kTileSums) return trs[mm]; else return reinterpret_cast<R&>(accr[mm]);
        };
        auto ti = [&](int mm) -> R& {
          if constexpr (kTileSums) return tis[mm]; else return reinterpret_cast<R&>(acci[mm]);
        };
        if constexpr (kTileSums) {
#pragma unroll
          for (int mm = 0; mm < MD; ++mm) trs[mm] = tis[mm] = R(0);
        }
        if (en.kind == 2) {
          for (int j = 0; j < ns; ++j) {
            R gr = R(0), gi = R(0);
            pair_charge<KIND>(tx, ty, tz, sg0[j], R4{R(1), R(0), R(0), R(0)}, k, kim, CK, gr, gi, tab);
#pragma unroll
            for (int mm = 0; mm < MD; ++mm) {
              const R qr = sst[j][mm][0];
              if constexpr (KIND == 1) {
                const R qi = sst[j][mm][1];
                tr(mm) = fma(qr, gr, fma(-qi, gi, tr(mm)));
                ti(mm) = fma(qr, gi, fma(qi, gr, ti(mm)));
              } else {
                tr(mm) = fma(qr, gr, tr(mm));
              }
            }
          }
        } else {
          const bool chk = en.kind == 0;
          for (int j = 0; j < ns; ++j) {
            const R4 w = sab[j];  // (a_r, a_i, b_r, b_i); Laplace (a, 0, b, 0)
            if constexpr (KIND == 1) {
              R gr, gi, dr, di;
              if (chk)
                pair_helm_unit<true>(tx, ty, tz, sg0[j], sg1[j], k, kim, thr2, CK, gr, gi, dr, di, tab);
              else
                pair_helm_unit<false>(tx, ty, tz, sg0[j], sg1[j], k, kim, thr2, CK, gr, gi, dr, di, tab);
              // K = a G + b D
              const R kr_ = fma(w.x, gr, fma(-w.y, gi, fma(w.z, dr, -w.w * di)));
              const R ki_ = fma(w.x, gi, fma(w.y, gr, fma(w.z, di, w.w * dr)));
#pragma unroll
              for (int mm = 0; mm < MD; ++mm) {
                const R2 sv = *reinterpret_cast<const R2*>(sst[j][mm]);
                tr(mm) = fma(sv.x, kr_, fma(-sv.y, ki_, tr(mm)));
                ti(mm) = fma(sv.x, ki_, fma(sv.y, kr_, ti(mm)));
              }
            } else {
              R g, dd;
              if (chk)
                pair_lap_unit<R, true>(tx, ty, tz, sg0[j], sg1[j], thr2, g, dd);
              else
                pair_lap_unit<R, false>(tx, ty, tz, sg0[j], sg1[j], thr2, g, dd);
              const R kv = fma(w.x, g, w.z * dd);
#pragma unroll
              for (int mm = 0; mm < MD; ++mm) tr(mm) = fma(sst[j][mm][0], kv, tr(mm));
            }
          }
        }
        if constexpr (kTileSums) {
#pragma unroll
          for (int mm = 0; mm < MD; ++mm) {
            accr[mm] += double(trs[mm]);
            acci[mm] += double(tis[mm]);
          }
        }
      }
    }
    if (PROXYT) break;
    n = ta.tn[n].parent;
    if (n < 0) break;
    e0 = ta.tn[n].pe0;
    e1 = ta.tn[n].pe1;
  }
  if constexpr (!PROXYT) {
    // downward pass, one density at a time through the shared buffer
    for (int a = node; a >= 0; a = ta.tn[a].parent) {
      const TNodeD an = ta.tn[a];
      if (an.tpoff < 0) continue;
      const int P = an.np0 * an.np1 * an.np2;
      R Lx[kP], Ly[kP], Lz[kP];
      {
        const double h0 = 0.5 * (an.hi[0] - an.lo[0]), h1 = 0.5 * (an.hi[1] - an.lo[1]),
                     h2 = 0.5 * (an.hi[2] - an.lo[2]);
        const R u0 = h0 > 0.0 ? R((x - 0.5 * (an.lo[0] + an.hi[0])) / h0) : R(0);
        const R u1 = h1 > 0.0 ? R((y - 0.5 * (an.lo[1] + an.hi[1])) / h1) : R(0);
        const R u2 = h2 > 0.0 ? R((z - 0.5 * (an.lo[2] + an.hi[2])) / h2) : R(0);
        lagrange(an.np0, u0, Lx);
        lagrange(an.np1, u1, Ly);
        lagrange(an.np2, u2, Lz);
      }
      for (int mm = 0; mm < nm; ++mm) {
        __syncthreads();
        for (int q = tid; q < P; q += kEvThreads) {
          const R* pp = phi + (size_t(an.tpoff + q) * nd + m0 + mm) * C;
          sphi[q] = R2{pp[0], C == 2 ? pp[C - 1] : R(0)};
        }
        __syncthreads();
        if (!act) continue;
        R sr = R(0), si = R(0);
        for (int i = 0; i < an.np0; ++i)
          for (int j = 0; j < an.np1; ++j) {
            const R w = Lx[i] * Ly[j];
            const R2* ph = sphi + (i * an.np1 + j) * an.np2;
            R qr = R(0), qi = R(0);
#pragma unroll
            for (int l = 0; l < kP; ++l)
              if (l < an.np2) {
                qr = fma(Lz[l], ph[l].x, qr);
                qi = fma(Lz[l], ph[l].y, qi);
              }
            sr = fma(w, qr, sr);
            si = fma(w, qi, si);
          }
        // mm is runtime: add through a register-indexed loop
#pragma unroll
        for (int q2 = 0; q2 < MD; ++q2)
          if (q2 == mm) {
            accr[q2] += double(sr);
            acci[q2] += double(si);
          }
      }
    }
  }
  if (!act) return;
#pragma unroll
  for (int mm = 0; mm < MD; ++mm) {
    if (mm >= nm) break;
    if constexpr (PROXYT) {
      R* o = phi + (size_t(tn.tpoff + k0 + tid) * nd + m0 + mm) * C;
      o[0] = R(accr[mm]);
      if constexpr (C == 2) o[1] = R(acci[mm]);
    } else {
      const int64_t it = ta.tperm[tn.b + tid];
      double* o = partial + (size_t(it) * nd + m0 + mm) * C;
      o[0] = accr[mm];
      if constexpr (C == 2) o[1] = acci[mm];
    }
  }
}

template <int KIND, typename R, bool CK, int MD>
void launch_md(const TreeArgs& ta, const KParams& kp, int npitems, int nleaf, const R* sig,
               const R* ab, const R* qhat, R* phi, double* partial, int nd, cudaStream_t st,
               int& launches) {
  const unsigned gy = unsigned((nd + MD - 1) / MD);
  if (npitems > 0) {
    tree_eval_md_kernel<KIND, R, CK, true, MD><<<dim3(unsigned(npitems), gy), kEvThreads, 0, st>>>(
        ta, kp, sig, ab, qhat, phi, partial, nd);
    ++launches;
  }
  if (nleaf > 0) {
    tree_eval_md_kernel<KIND, R, CK, false, MD><<<dim3(unsigned(nleaf), gy), kEvThreads, 0, st>>>(
        ta, kp, sig, ab, qhat, phi, partial, nd);
    ++launches;
  }
}

template <int KIND, typename R, bool CK>
cudaError_t run_t(const TreeArgs& ta, const KParams& kp, int nup, const UpItemD* up, int nred,
                  const RedD* red, int npitems, int nleaf, const R* str, const R* sig,
                  const R* ab, double* up_part, R* qhat, R* phi, double* partial, int nd,
                  cudaStream_t st) {
  constexpr int C = KIND == 1 ? 2 : 1;
  int launches = 0;
  const bool md = nd >= 2;  // several densities: from sig and ab
  if (nup > 0) {
    const dim3 grid{unsigned(nup), unsigned(nd), 1u};
    if (md)
      tree_up_kernel<KIND, R, true><<<grid, kUpThreads, 0, st>>>(up, ta, nullptr, sig, ab, nd, up_part);
    else
      tree_up_kernel<KIND, R, false><<<grid, kUpThreads, 0, st>>>(up, ta, str, nullptr, nullptr, nd,
                                                                  up_part);
    tree_reduce_kernel<R, C><<<unsigned(nred), 256, 0, st>>>(red, up_part, nd, qhat);
    launches += 2;
  }
  if (md) {
    // one kernel evaluation per pair for a group of densities
    if (nd <= 4)
      launch_md<KIND, R, CK, 4>(ta, kp, npitems, nleaf, sig, ab, qhat, phi, partial, nd, st, launches);
    else if (nd <= 8)
      launch_md<KIND, R, CK, 8>(ta, kp, npitems, nleaf, sig, ab, qhat, phi, partial, nd, st, launches);
    else
      launch_md<KIND, R, CK, 16>(ta, kp, npitems, nleaf, sig, ab, qhat, phi, partial, nd, st, launches);
  } else {
    if (npitems > 0) {
      tree_eval_kernel<KIND, R, CK, true>
          <<<dim3(unsigned(npitems), 1u), kEvThreads, 0, st>>>(ta, kp, str, qhat, phi, partial, nd);
      ++launches;
    }
    if (nleaf > 0) {
      tree_eval_kernel<KIND, R, CK, false>
          <<<dim3(unsigned(nleaf), 1u), kEvThreads, 0, st>>>(ta, kp, str, qhat, phi, partial, nd);
      ++launches;
    }
  }
  note_launches(launches);
  return cudaGetLastError();
}

}  // namespace
}  // namespace dev

namespace {
#define TF_CUDA(call)                                                     \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                              \
      set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
      return e_ == cudaErrorMemoryAllocation ? kErrNoMem : kErrCuda;      \
    }                                                                     \
  } while (0)

template <class T>
cudaError_t put(DBuf<T>& b, const T* h, size_t n, cudaStream_t st) {
  cudaError_t e = b.alloc(std::max<size_t>(n, 1));
  if (e != cudaSuccess || n == 0) return e;
  return cudaMemcpyAsync(b.p, h, n * sizeof(T), cudaMemcpyHostToDevice, st);
}
template <class T>
cudaError_t put_raw(DBuf<char>& b, const std::vector<T>& h, cudaStream_t st) {
  const size_t bytes = h.size() * sizeof(T);
  cudaError_t e = b.alloc(std::max<size_t>(bytes, 16));
  if (e != cudaSuccess || bytes == 0) return e;
  return cudaMemcpyAsync(b.p, h.data(), bytes, cudaMemcpyHostToDevice, st);
}
std::vector<double> get(const double* d, int64_t n) {
  std::vector<double> h(size_t(std::max<int64_t>(n, 0)));
  if (n > 0) cudaMemcpy(h.data(), d, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost);
  return h;
}
// proxy grid coordinates of a node (k = (i np1 + j) np2 + l)
void grid_points(const tree::Node& nd, std::vector<double>& px, std::vector<double>& py,
                 std::vector<double>& pz) {
  double xs[3][tree::kMaxP], w[tree::kMaxP];
  for (int d = 0; d < 3; ++d) {
    double u[tree::kMaxP];
    tree::cheb_nodes(nd.np[d], u, w);
    const double c = 0.5 * (nd.lo[d] + nd.hi[d]), h = 0.5 * (nd.hi[d] - nd.lo[d]);
    for (int q = 0; q < nd.np[d]; ++q) xs[d][q] = c + h * u[q];
  }
  for (int i = 0; i < nd.np[0]; ++i)
    for (int j = 0; j < nd.np[1]; ++j)
      for (int l = 0; l < nd.np[2]; ++l) {
        px.push_back(xs[0][i]);
        py.push_back(xs[1][j]);
        pz.push_back(xs[2][l]);
      }
}
}  // namespace

int TreeFar::build(const dev::Geometry& g, const tree::Params& prm, double thresh,
                   cudaStream_t st, const dev::KParams* kp, int precision) {
  const auto t0 = std::chrono::steady_clock::now();
  prm_ = prm;
  ntarg_ = g.ntarg;
  nptso_ = g.nptso;
  if (ntarg_ <= 0 || nptso_ <= 0) {
    set_last_error("tree far field: no targets or sources");
    return kErrArg;
  }
  if (nptso_ >= (int64_t(1) << 31)) {
    set_last_error("tree far field: more than 2^31 sources");
    return kErrArg;
  }
  TF_CUDA(cudaStreamSynchronize(st));
  const std::vector<double> htx = get(g.tx, ntarg_), hty = get(g.ty, ntarg_), htz = get(g.tz, ntarg_);
  const std::vector<double> hsx = get(g.sx, nptso_), hsy = get(g.sy, nptso_), hsz = get(g.sz, nptso_);
  const std::vector<double> hnx = get(g.snx, nptso_), hny = get(g.sny, nptso_), hnz = get(g.snz, nptso_);
  double ext = 0.0;
  for (const auto* v : {&htx, &hty, &htz, &hsx, &hsy, &hsz})
    for (double c : *v) ext = std::max(ext, 2.0 * std::fabs(c));
  const double sep_min = thresh + std::ldexp(ext, -12);
  tree::Tree T, S;
  tree::build_tree(ntarg_, htx.data(), hty.data(), htz.data(), prm.leaf_t, T);
  tree::build_tree(nptso_, hsx.data(), hsy.data(), hsz.data(), prm.leaf_s, S);
  // target leaves must fit one thread block; only more than 128 coincident
  // targets (which no split separates) exceed it
  for (const auto& nd : T.nodes)
    if (nd.nchild == 0 && nd.n() > dev::kEvThreads) {
      set_last_error("tree far field: more than 128 coincident targets");
      return kErrArg;
    }
  tree::set_proxies(T, prm);
  tree::set_proxies(S, prm);
  std::vector<tree::Interaction> ia;
  tree::traverse(T, S, prm, sep_min, ia);
  const int nT = int(T.nodes.size()), nS = int(S.nodes.size());
  // ---- proxies in use -------------------------------------------------------
  std::vector<int64_t> spoff(nS, -1), tpoff(nT, -1);
  for (const auto& x : ia) {
    if (x.kind == tree::kPC || x.kind == tree::kCC) spoff[x.s] = 0;
    if (x.kind == tree::kCP || x.kind == tree::kCC) tpoff[x.t] = 0;
  }
  std::vector<double> spx, spy, spz, tpx, tpy, tpz;
  for (int s = 0; s < nS; ++s)
    if (spoff[s] == 0) {
      spoff[s] = int64_t(spx.size());
      grid_points(S.nodes[s], spx, spy, spz);
    }
  for (int t = 0; t < nT; ++t)
    if (tpoff[t] == 0) {
      tpoff[t] = int64_t(tpx.size());
      grid_points(T.nodes[t], tpx, tpy, tpz);
    }
  if (spx.size() >= (size_t(1) << 31)) {
    set_last_error("tree far field: too many source proxies");
    return kErrArg;
  }
  // ---- entries per target node ------------------------------------------------
  std::vector<int64_t> pcnt(nT + 1, 0), ccnt(nT + 1, 0);
  for (const auto& x : ia) {
    if (x.kind == tree::kCP || x.kind == tree::kCC)
      ++ccnt[x.t + 1];
    else
      ++pcnt[x.t + 1];
  }
  std::partial_sum(pcnt.begin(), pcnt.end(), pcnt.begin());
  std::partial_sum(ccnt.begin(), ccnt.end(), ccnt.begin());
  std::vector<dev::EntryD> pent(static_cast<size_t>(pcnt[nT])), cent(static_cast<size_t>(ccnt[nT]));
  {
    std::vector<int64_t> pf(pcnt.begin(), pcnt.end() - 1), cf(ccnt.begin(), ccnt.end() - 1);
    for (const auto& x : ia) {
      const tree::Node& tn = T.nodes[x.t];
      const tree::Node& sn = S.nodes[x.s];
      double d2 = 0.0;
      for (int d = 0; d < 3; ++d) d2 += (tn.c[d] - sn.c[d]) * (tn.c[d] - sn.c[d]);
      const int pk = std::sqrt(d2) - tn.r - sn.r > sep_min ? 1 : 0;
      dev::EntryD en{0, 0, 0, 0};
      switch (x.kind) {
        case tree::kPPCheck:
          en = {0, int(sn.b), int(sn.e), 0};
          break;
        case tree::kPP:
          en = {1, int(sn.b), int(sn.e), 0};
          break;
        case tree::kCP:
          en = {pk, int(sn.b), int(sn.e), 0};
          break;
        default:  // kPC, kCC: the source node's proxies
          en = {2, int(spoff[x.s]), int(spoff[x.s] + sn.nprox()), 0};
          break;
      }
      if (x.kind == tree::kCP || x.kind == tree::kCC)
        cent[size_t(cf[x.t]++)] = en;
      else
        pent[size_t(pf[x.t]++)] = en;
    }
    // entries of a node grouped by kind (fewer divergent tile loops)
    auto by_kind = [](const dev::EntryD& a, const dev::EntryD& b) {
      return a.kind != b.kind ? a.kind < b.kind : a.b < b.b;
    };
    for (int t = 0; t < nT; ++t) {
      std::sort(pent.begin() + pcnt[t], pent.begin() + pcnt[t + 1], by_kind);
      std::sort(cent.begin() + ccnt[t], cent.begin() + ccnt[t + 1], by_kind);
    }
  }
  std::vector<dev::TNodeD> tnodes(nT);
  for (int t = 0; t < nT; ++t) {
    const tree::Node& nd = T.nodes[t];
    dev::TNodeD& o = tnodes[t];
    o.parent = nd.parent;
    o.np0 = std::max(nd.np[0], 1);
    o.np1 = std::max(nd.np[1], 1);
    o.np2 = std::max(nd.np[2], 1);
    o.b = nd.b;
    o.e = nd.e;
    o.tpoff = tpoff[t];
    o.pe0 = pcnt[t];
    o.pe1 = pcnt[t + 1];
    o.ce0 = ccnt[t];
    o.ce1 = ccnt[t + 1];
    for (int d = 0; d < 3; ++d) {
      o.lo[d] = nd.lo[d];
      o.hi[d] = nd.hi[d];
    }
  }
  // ---- work items, largest first ----------------------------------------------
  auto entry_cost = [](const dev::EntryD& en) { return double(en.e - en.b); };
  std::vector<std::pair<double, int>> lw;
  stats_ = TreeStats();
  double pair_evals = 0.0, down_evals = 0.0;
  for (int t = 0; t < nT; ++t) {
    const tree::Node& nd = T.nodes[t];
    if (nd.nchild != 0 || nd.n() == 0) continue;
    double c = 0.0, dn = 0.0;
    for (int a = t; a >= 0; a = T.nodes[a].parent) {
      for (int64_t q = pcnt[a]; q < pcnt[a + 1]; ++q) c += entry_cost(pent[size_t(q)]);
      if (tpoff[a] >= 0) dn += T.nodes[a].nprox();
    }
    pair_evals += c * double(nd.n());
    down_evals += dn * double(nd.n());
    lw.push_back({c * double(dev::kEvThreads) + dn * nd.n(), t});
  }
  std::sort(lw.begin(), lw.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  std::vector<int> leaves;
  for (const auto& x : lw) leaves.push_back(x.second);
  std::vector<std::pair<double, int2>> pw;
  for (int t = 0; t < nT; ++t) {
    if (tpoff[t] < 0) continue;
    double c = 0.0;
    for (int64_t q = ccnt[t]; q < ccnt[t + 1]; ++q) c += entry_cost(cent[size_t(q)]);
    const int P = T.nodes[t].nprox();
    pair_evals += c * P;
    for (int k = 0; k < P; k += dev::kEvThreads)
      pw.push_back({c * std::min(dev::kEvThreads, P - k), make_int2(t, k)});
  }
  std::sort(pw.begin(), pw.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  std::vector<int2> pitems;
  for (const auto& x : pw) pitems.push_back(x.second);
  std::vector<std::pair<double, dev::UpItemD>> uw;
  std::vector<dev::RedD> reds;
  int64_t ubase = 0;
  double up_evals = 0.0;
  for (int s = 0; s < nS; ++s) {
    if (spoff[s] < 0) continue;
    const tree::Node& nd = S.nodes[s];
    const int P = nd.nprox();
    dev::RedD r{spoff[s], ubase, 0, P};
    for (int64_t b = nd.b; b < nd.e; b += dev::kUpChunk) {
      dev::UpItemD u{};
      u.b = b;
      u.e = std::min(nd.e, b + dev::kUpChunk);
      u.ubase = ubase + int64_t(r.nitems) * P;
      u.np0 = nd.np[0];
      u.np1 = nd.np[1];
      u.np2 = nd.np[2];
      for (int d = 0; d < 3; ++d) {
        u.lo[d] = nd.lo[d];
        u.hi[d] = nd.hi[d];
      }
      uw.push_back({double(u.e - u.b) * P, u});
      ++r.nitems;
    }
    up_evals += double(nd.n()) * P;
    ubase += int64_t(r.nitems) * P;
    reds.push_back(r);
  }
  std::stable_sort(uw.begin(), uw.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  std::vector<dev::UpItemD> ups;
  for (const auto& x : uw) ups.push_back(x.second);
  up_len_ = ubase;
  // ---- sorted geometry, permutations, leaf centres -------------------------------
  std::vector<double> stx(ntarg_), sty(ntarg_), stz(ntarg_), ssx(nptso_), ssy(nptso_), ssz(nptso_),
      snx(nptso_), sny(nptso_), snz(nptso_), tcen(size_t(3) * ntarg_);
  for (int64_t q = 0; q < ntarg_; ++q) {
    const int64_t o = T.perm[q];
    stx[q] = htx[o];
    sty[q] = hty[o];
    stz[q] = htz[o];
  }
  std::vector<int32_t> sdest(nptso_);
  for (int64_t q = 0; q < nptso_; ++q) {
    const int64_t o = S.perm[q];
    ssx[q] = hsx[o];
    ssy[q] = hsy[o];
    ssz[q] = hsz[o];
    snx[q] = hnx[o];
    sny[q] = hny[o];
    snz[q] = hnz[o];
    sdest[o] = int32_t(q);
  }
  for (const auto& nd : T.nodes) {
    if (nd.nchild != 0) continue;
    for (int64_t q = nd.b; q < nd.e; ++q)
      for (int d = 0; d < 3; ++d) tcen[size_t(3) * T.perm[q] + d] = nd.c[d];
  }
  // ---- upload ------------------------------------------------------------------
  double hn[(tree::kMaxP + 1) * tree::kMaxP] = {}, hw[(tree::kMaxP + 1) * tree::kMaxP] = {};
  for (int p = 1; p <= tree::kMaxP; ++p) tree::cheb_nodes(p, hn + p * tree::kMaxP, hw + p * tree::kMaxP);
  TF_CUDA(cudaMemcpyToSymbolAsync(dev::cNode, hn, sizeof(hn), 0, cudaMemcpyHostToDevice, st));
  TF_CUDA(cudaMemcpyToSymbolAsync(dev::cWt, hw, sizeof(hw), 0, cudaMemcpyHostToDevice, st));
  TF_CUDA(put(tx_, stx.data(), stx.size(), st));
  TF_CUDA(put(ty_, sty.data(), sty.size(), st));
  TF_CUDA(put(tz_, stz.data(), stz.size(), st));
  TF_CUDA(put(sx_, ssx.data(), ssx.size(), st));
  TF_CUDA(put(sy_, ssy.data(), ssy.size(), st));
  TF_CUDA(put(sz_, ssz.data(), ssz.size(), st));
  TF_CUDA(put(snx_, snx.data(), snx.size(), st));
  TF_CUDA(put(sny_, sny.data(), sny.size(), st));
  TF_CUDA(put(snz_, snz.data(), snz.size(), st));
  TF_CUDA(put(tcen_, tcen.data(), tcen.size(), st));
  TF_CUDA(put(tperm_, T.perm.data(), T.perm.size(), st));
  TF_CUDA(put(sdest_, sdest.data(), sdest.size(), st));
  TF_CUDA(put(tpx_, tpx.data(), tpx.size(), st));
  TF_CUDA(put(tpy_, tpy.data(), tpy.size(), st));
  TF_CUDA(put(tpz_, tpz.data(), tpz.size(), st));
  TF_CUDA(put(spx_, spx.data(), spx.size(), st));
  TF_CUDA(put(spy_, spy.data(), spy.size(), st));
  TF_CUDA(put(spz_, spz.data(), spz.size(), st));
  TF_CUDA(put(leaves_, leaves.data(), leaves.size(), st));
  TF_CUDA(put(pitems_, pitems.data(), pitems.size(), st));
  TF_CUDA(put_raw(tnodes_, tnodes, st));
  TF_CUDA(put_raw(pent_, pent, st));
  TF_CUDA(put_raw(cent_, cent, st));
  TF_CUDA(put_raw(upitems_, ups, st));
  TF_CUDA(put_raw(reds_, reds, st));
  if (kp && g.sw) {
    // per-source (a_s, b_s) in tree order for several densities at once
    const size_t rs = precision == 1 ? sizeof(float) : sizeof(double);
    TF_CUDA(ab_.alloc(size_t(nptso_) * (kp->kind == 1 ? 4 : 2) * rs));
    TF_CUDA(dev::launch_source_consts(g, *kp, precision, ab_.p, st, sdest_.p));
    ab_precision_ = precision;
  }
  TF_CUDA(cudaStreamSynchronize(st));  // host vectors above feed async copies
  nleaf_ = int(leaves.size());
  npitems_ = int(pitems.size());
  nup_ = int(ups.size());
  nred_ = int(reds.size());
  stats_.tnodes = nT;
  stats_.snodes = nS;
  stats_.leaves = nleaf_;
  stats_.proxy_items = npitems_;
  stats_.up_items = nup_;
  for (const auto& x : ia) ++stats_.interactions[x.kind];
  stats_.pair_evals = pair_evals;
  stats_.up_evals = up_evals;
  stats_.down_evals = down_evals;
  stats_.source_proxies = int64_t(spx.size());
  stats_.target_proxies = int64_t(tpx.size());
  stats_.build_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return kOk;
}

int TreeFar::ensure_scratch(int nd, int precision) {
  const int C = 2;  // room for complex values
  const size_t rs = precision == 1 ? sizeof(float) : sizeof(double);
  TF_CUDA(up_part_.alloc(std::max<size_t>(1, size_t(up_len_) * nd * C)));
  TF_CUDA(qhat_.alloc(std::max<size_t>(16, size_t(stats_.source_proxies) * nd * C * rs)));
  TF_CUDA(phi_.alloc(std::max<size_t>(16, size_t(stats_.target_proxies) * nd * C * rs)));
  return kOk;
}

cudaError_t TreeFar::run(int precision, int nd, const dev::KParams& kp, const void* str_sorted,
                         double* partial, cudaStream_t st, const void* sig_sorted) {
  if (nd < 1 || nd > 65535) return cudaErrorInvalidValue;
  if (nd >= 2 && (!sig_sorted || !ab_.p || ab_precision_ != precision)) return cudaErrorInvalidValue;
  if (ensure_scratch(nd, precision) != kOk) return cudaErrorMemoryAllocation;
  dev::TreeArgs ta;
  ta.tn = reinterpret_cast<const dev::TNodeD*>(tnodes_.p);
  ta.pent = reinterpret_cast<const dev::EntryD*>(pent_.p);
  ta.cent = reinterpret_cast<const dev::EntryD*>(cent_.p);
  ta.leaves = leaves_.p;
  ta.pitems = pitems_.p;
  ta.tx = tx_.p;
  ta.ty = ty_.p;
  ta.tz = tz_.p;
  ta.tperm = tperm_.p;
  ta.sx = sx_.p;
  ta.sy = sy_.p;
  ta.sz = sz_.p;
  ta.snx = snx_.p;
  ta.sny = sny_.p;
  ta.snz = snz_.p;
  ta.tpx = tpx_.p;
  ta.tpy = tpy_.p;
  ta.tpz = tpz_.p;
  ta.spx = spx_.p;
  ta.spy = spy_.p;
  ta.spz = spz_.p;
  const auto* up = reinterpret_cast<const dev::UpItemD*>(upitems_.p);
  const auto* red = reinterpret_cast<const dev::RedD*>(reds_.p);
  const bool ck = kp.kind == 1 && kp.ki != 0.0;
  auto go = [&](auto kind_c, auto ck_c, auto* tag) {
    using R = std::remove_pointer_t<decltype(tag)>;
    constexpr int KIND = decltype(kind_c)::value;
    constexpr bool CK = decltype(ck_c)::value;
    return dev::run_t<KIND, R, CK>(ta, kp, nup_, up, nred_, red, npitems_, nleaf_,
                                   static_cast<const R*>(str_sorted),
                                   static_cast<const R*>(sig_sorted),
                                   reinterpret_cast<const R*>(ab_.p), up_part_.p,
                                   reinterpret_cast<R*>(qhat_.p), reinterpret_cast<R*>(phi_.p),
                                   partial, nd, st);
  };
  using I0 = std::integral_constant<int, 0>;
  using I1 = std::integral_constant<int, 1>;
  using BF = std::false_type;
  using BT = std::true_type;
  if (precision == 1) {
    float* f = nullptr;
    if (kp.kind == 0) return go(I0{}, BF{}, f);
    return ck ? go(I1{}, BT{}, f) : go(I1{}, BF{}, f);
  }
  double* d = nullptr;
  if (kp.kind == 0) return go(I0{}, BF{}, d);
  return ck ? go(I1{}, BT{}, d) : go(I1{}, BF{}, d);
}

}  // namespace bie
