// Device near-field quadrature generator (see nearquad_gpu.h).
//
// One warp per (target, patch) pair of the row-sparse near list, taken from
// a global work counter (self pairs first: they cost the most).  A warp
// integrates one parameter-space triangle at a time: each lane evaluates
// one rule node -- the patch basis (Koornwinder on triangles, tensor
// Legendre/Chebyshev on quads), the geometry sum over the patch
// coefficients and the kernel -- and writes the basis row to shared
// memory; the lanes then switch to one basis index each and accumulate
// sum_q K_q w_q P_l(y_q) over the chunk.  The refinement stack of the
// adaptive rule (vertices, level and the integral vector of every pending
// triangle) lives in a per-warp slice of global scratch; DFS order and the
// acceptance test follow the host generator (host/nearquad.cpp:190-247).
// The self rule (host/nearquad.cpp:251-311) flattens (sub-triangle, sinh
// node, Duffy node) into one index the lanes stride over.
#include "nearquad_gpu.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../host/basis.h"
#include "plan.h"
#include "basis_dev.cuh"
#include "trig_table.cuh"

namespace bie {
namespace {

constexpr int kNqMaxLevel = 18;
// Integral vectors per warp: at most 1 + 3 * 17 + 4 = 56 pending triangles
// (one other root, three siblings per level, four at the deepest level) and
// four children computed above the top.
constexpr int kNqSlots = 64;
constexpr int kNqStackDoubles = 8;  // per pending triangle: 6 vertex coordinates, level, cache index
constexpr int kNqMaxSteps = 1 << 16;
constexpr int kNqSubDoubles = 8 * 8 + 8;  // 8 self sub-triangles x 8, then the count
constexpr double kNqOver4Pi = 0.07957747154594767;
// Basis values of a chunk of 32 rule nodes in shared memory: one row of
// kNqPS doubles per basis function, node index fastest (the pad keeps
// 16-byte row starts and makes the lanes' 16-byte reads of one column pair
// fall in distinct banks).
constexpr int kNqPS = 34;
constexpr unsigned kFull = 0xffffffffu;

struct NqType {
  int iptype, norder, np, nv;
  int rule;            // 0..2: 8, 10 or 12 points per direction
  int uvs, wts, umat;  // arena offsets of nodes (2 np), weights (np), umat (np x np)
  double vert[8];      // corners of the reference domain
};

struct NqArgs {
  double zr, zi, ar, ai, br, bi, eps;
  const double* coefs;  // srccoefs, 9 per node
  const NqType* types;
  const int* ptype;
  const int64_t* pstart;  // first node of each patch, 0-based
  double* ptol;           // per-patch refinement tolerance
  const double* arena;
  int rule_off[3], rule_nq[3];  // xi[nq], eta[nq], w[nq] consecutive
  int self_off, nself;          // Gauss-Legendre x[nself], w[nself]
  const double* targ;           // 3 x nt
  const double* uvt;            // 2 x nt
  const longlong2* items;       // (pair, target); self pairs first, then by patch
  int64_t item_lo, item_hi;     // this launch's item range
  int64_t nself_items, npatches;
  // Cache of the uniform refinement levels 0..cache_levels of every root
  // triangle of the patches in the current group: per triangle (root r,
  // heap index h) and rule node q, the geometry xyz, unit normal and
  // |J| w_q area2 (7 x nq, node fastest) followed by the basis values
  // (np x nq, node fastest).
  double* cache;
  const int64_t* coff;  // per patch: offset of its block in `cache` (-1: not in this group)
  int cache_levels;     // -1: no cache
  int cache_h;          // triangles per root: (4^(cache_levels+1) - 1) / 3
  const int64_t* col_ind;
  const int64_t* iquad;
  double* wout;
  double* scratch;
  int64_t scratch_per_warp;
  int np_max, warp_doubles;
  unsigned long long* next;  // this launch's item counter
  unsigned long long* stat;  // [0] kernel evaluations, [1] capped pairs
};

// Combined-field kernel (alpha G + beta dG/dn_y) / 4pi at target x of the
// source y with unit normal nr (host/nearquad.cpp LapComb / HelmComb).
// 1/r from rsqrt; e^{i Re(k) r} from the block's sine/cosine table; the
// decay e^{-Im(k) r} only for complex wavenumbers.
template <bool CPLX>
__device__ __forceinline__ void kernel_val(const NqArgs& a, const double2* tab, const double* y,
                                           const double* nr, const double* x, double& re,
                                           double& im) {
  const double dx = x[0] - y[0], dy = x[1] - y[1], dz = x[2] - y[2];
  const double d = dx * nr[0] + dy * nr[1] + dz * nr[2];
  const double r2 = dx * dx + dy * dy + dz * dz;
  const double ir = rsqrt(r2);
  const double r = r2 * ir;
  const double dr3 = d * ir * ir * ir;
  if (!CPLX) {
    re = (a.br * dr3 + a.ar * ir) * kNqOver4Pi;
    im = 0.0;
    return;
  }
  // (beta d (1 - ikr) / r^3 + alpha / r) e^{ikr},  1 - ikr = (1 + zi r) - i zr r
  const double omr = 1.0 + a.zi * r, omi = -a.zr * r;
  const double tr = (a.br * omr - a.bi * omi) * dr3 + a.ar * ir;
  const double ti = (a.br * omi + a.bi * omr) * dr3 + a.ai * ir;
  double s, c;
  dev::sincos_tab(a.zr * r, tab, s, c);
  const double m = (a.zi != 0.0 ? exp(-a.zi * r) : 1.0) * kNqOver4Pi;
  re = (tr * c - ti * s) * m;
  im = (tr * s + ti * c) * m;
}

// One rule node: basis values -> prow[l * kNqPS], kernel value -> (kr, ki);
// returns |J|.
template <bool CPLX>
__device__ double node_val(const NqArgs& a, const double2* tab, const NqType* T, const double* c,
                           double u, double v, double* prow, const double* x, double& kr,
                           double& ki) {
  double g[9];
  basis_geom<true, true>(T->iptype, T->norder, u, v, c, prow, kNqPS, g);
  const double n0 = g[4] * g[8] - g[5] * g[7];
  const double n1 = g[5] * g[6] - g[3] * g[8];
  const double n2 = g[3] * g[7] - g[4] * g[6];
  const double j2 = n0 * n0 + n1 * n1 + n2 * n2;
  const double inv = rsqrt(j2);
  const double nr[3] = {n0 * inv, n1 * inv, n2 * inv};
  kernel_val<CPLX>(a, tab, g, nr, x, kr, ki);
  return j2 * inv;
}

// Lanes own basis indices l = lane, lane + 32, ...: acc_l += sum over the
// chunk's nv nodes of kv_q P_l,q (P rows of kNqPS doubles and kv in shared
// memory; node pairs read as one 16-byte load, two partial sums per
// component to halve the dependent FMA chain).
template <bool CPLX>
__device__ __forceinline__ void accumulate(const double* P, const double* kv, int nv, int np,
                                           double* acc, int lane) {
  const double2* kv2 = reinterpret_cast<const double2*>(kv);
  for (int l = lane; l < np; l += 32) {
    const double* row = P + l * kNqPS;
    double s0r = 0.0, s0i = 0.0, s1r = 0.0, s1i = 0.0;
    auto step = [&](int q) {
      const double2 p = *reinterpret_cast<const double2*>(row + q);
      const double2 k0 = kv2[q], k1 = kv2[q + 1];
      s0r = fma(k0.x, p.x, s0r);
      s1r = fma(k1.x, p.y, s1r);
      if (CPLX) {
        s0i = fma(k0.y, p.x, s0i);
        s1i = fma(k1.y, p.y, s1i);
      }
    };
    if (nv == 32) {
#pragma unroll
      for (int q = 0; q < 32; q += 2) step(q);
    } else {
      int q = 0;
      for (; q + 1 < nv; q += 2) step(q);
      if (q < nv) {
        const double2 k0 = kv2[q];
        s0r = fma(k0.x, row[q], s0r);
        if (CPLX) s0i = fma(k0.y, row[q], s0i);
      }
    }
    acc[2 * l] += s0r + s1r;
    acc[2 * l + 1] += s0i + s1i;
  }
}

// Asynchronous copy of the chunk's basis values: rows l < np of nv doubles
// from src + l * nq (16-byte aligned: nq and the chunk start are even) to
// P + l * kNqPS, as 16-byte cp.async pieces strided over the lanes (an odd
// last column by plain loads).  Completed by cp_async_wait_all() and a
// __syncwarp().
__device__ __forceinline__ void copy_chunk_async(double* P, const double* src, int nq, int nv,
                                                 int np, int lane) {
  auto piece = [&](int l, int j) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(P + l * kNqPS + 2 * j));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa),
                 "l"(src + size_t(l) * nq + 2 * j)
                 : "memory");
  };
  if (nv == 32) {
    for (int l = lane >> 4; l < np; l += 2) piece(l, lane & 15);
  } else {
    const int hv = nv >> 1;
    for (int i = lane; i < np * hv; i += 32) piece(i / hv, i % hv);
    if (nv & 1)
      for (int l = lane; l < np; l += 32) P[l * kNqPS + nv - 1] = __ldg(src + size_t(l) * nq + nv - 1);
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Child q of the 4-way split of parameter triangle v (host/nearquad.cpp
// PatchTree::children): the three corner triangles, then the middle one.
__device__ __forceinline__ void child_tri(const double* v, int q, double* o) {
  const double m01x = 0.5 * (v[0] + v[2]), m01y = 0.5 * (v[1] + v[3]);
  const double m12x = 0.5 * (v[2] + v[4]), m12y = 0.5 * (v[3] + v[5]);
  const double m20x = 0.5 * (v[4] + v[0]), m20y = 0.5 * (v[5] + v[1]);
  if (q == 0) {
    o[0] = v[0], o[1] = v[1], o[2] = m01x, o[3] = m01y, o[4] = m20x, o[5] = m20y;
  } else if (q == 1) {
    o[0] = m01x, o[1] = m01y, o[2] = v[2], o[3] = v[3], o[4] = m12x, o[5] = m12y;
  } else if (q == 2) {
    o[0] = m20x, o[1] = m20y, o[2] = m12x, o[3] = m12y, o[4] = v[4], o[5] = v[5];
  } else {
    o[0] = m01x, o[1] = m01y, o[2] = m12x, o[3] = m12y, o[4] = m20x, o[5] = m20y;
  }
}

// Integral vector over the parameter triangle v6 of K(x, y) P_l(y) dA -> dst.
// cached: the triangle's cache block (geometry and basis rows at the rule
// nodes) or null, in which case they are evaluated here.
template <bool CPLX>
__device__ void tri_integral(const NqArgs& a, const double2* tab, const NqType* T, const double* c,
                             const double* v6, const double* cached, const double* x, double* P,
                             double* kv, double* acc, double* dst, int lane) {
  const int np = T->np;
  const int nq = a.rule_nq[T->rule];
  for (int l = lane; l < np; l += 32) acc[2 * l] = acc[2 * l + 1] = 0.0;
  if (cached) {
    for (int q0 = 0; q0 < nq; q0 += 32) {
      const int q = q0 + lane;
      const int nv = min(32, nq - q0);
      // basis rows of the chunk into the P buffer while the kernel values
      // are computed
      copy_chunk_async(P, cached + 7 * nq + q0, nq, nv, np, lane);
      if (q < nq) {
        const double y[3] = {__ldg(cached + q), __ldg(cached + nq + q), __ldg(cached + 2 * nq + q)};
        const double nr[3] = {__ldg(cached + 3 * nq + q), __ldg(cached + 4 * nq + q),
                              __ldg(cached + 5 * nq + q)};
        const double wq = __ldg(cached + 6 * nq + q);
        double kr, ki;
        kernel_val<CPLX>(a, tab, y, nr, x, kr, ki);
        kv[2 * lane] = kr * wq;
        kv[2 * lane + 1] = ki * wq;
      }
      cp_async_wait_all();
      __syncwarp();
      accumulate<CPLX>(P, kv, nv, np, acc, lane);
      __syncwarp();
    }
    for (int l = lane; l < np; l += 32) {
      dst[2 * l] = acc[2 * l];
      dst[2 * l + 1] = acc[2 * l + 1];
    }
    return;
  }
  const double* rule = a.arena + a.rule_off[T->rule];
  const double ax = v6[2] - v6[0], ay = v6[3] - v6[1];
  const double bx = v6[4] - v6[0], by = v6[5] - v6[1];
  const double area2 = fabs(ax * by - ay * bx);
  for (int q0 = 0; q0 < nq; q0 += 32) {
    const int q = q0 + lane;
    if (q < nq) {
      const double xi = rule[q], eta = rule[nq + q], w = rule[2 * nq + q];
      double kr, ki;
      const double jn = node_val<CPLX>(a, tab, T, c, v6[0] + xi * ax + eta * bx,
                                       v6[1] + xi * ay + eta * by, P + lane, x, kr, ki);
      const double s = jn * w * area2;
      kv[2 * lane] = kr * s;
      kv[2 * lane + 1] = ki * s;
    }
    __syncwarp();
    accumulate<CPLX>(P, kv, min(32, nq - q0), np, acc, lane);
    __syncwarp();
  }
  for (int l = lane; l < np; l += 32) {
    dst[2 * l] = acc[2 * l];
    dst[2 * l + 1] = acc[2 * l + 1];
  }
}

// Adaptive integral for a target off the patch (host/nearquad.cpp:190-247):
// pop a triangle, integrate its four children, accept their sum when it
// agrees with the parent to tol (max over l) or at level 18, else push them.
template <bool CPLX>
__device__ void near_integral(const NqArgs& a, const double2* tab, const NqType* T, const double* c,
                              const double* pcache, const double* x, double tol, double* P,
                              double* kv, double* acc, double* out, double* vec, double* stk,
                              int lane, unsigned long long& nev, int& capped) {
  const int np = T->np, vs = 2 * a.np_max;
  const int nq = a.rule_nq[T->rule];
  const int H = a.cache_h;
  const size_t tri_doubles = size_t(7 + np) * nq;
  auto block = [&](int ci) { return ci >= 0 ? pcache + size_t(ci) * tri_doubles : nullptr; };
  for (int l = lane; l < np; l += 32) out[2 * l] = out[2 * l + 1] = 0.0;
  const double* V = T->vert;
  const int nroots = T->nv == 3 ? 1 : 2;
  int sp = 0;
  for (int r = 0; r < nroots; ++r) {
    const double v6[6] = {V[0], V[1], V[2 + 2 * r], V[3 + 2 * r], V[4 + 2 * r], V[5 + 2 * r]};
    const int ci = pcache ? r * H : -1;
    if (lane == 0) {
      for (int i = 0; i < 6; ++i) stk[kNqStackDoubles * sp + i] = v6[i];
      stk[kNqStackDoubles * sp + 6] = 0.0;
      stk[kNqStackDoubles * sp + 7] = double(ci);
    }
    tri_integral<CPLX>(a, tab, T, c, v6, block(ci), x, P, kv, acc, vec + size_t(sp) * vs, lane);
    nev += nq;
    ++sp;
  }
  __syncwarp();
  int steps = 0;
  while (sp > 0) {
    if (++steps > kNqMaxSteps) {
      capped = 1;
      break;
    }
    const int top = sp - 1;
    const double* e = stk + kNqStackDoubles * top;
    const double v[6] = {e[0], e[1], e[2], e[3], e[4], e[5]};
    const int lev = int(e[6]);
    const int ci = int(e[7]);
    // children of a cached triangle above the last cached level are cached:
    // heap index h -> 4h + 1 + q within the same root
    const int cc = (ci >= 0 && lev < a.cache_levels) ? (ci / H) * H + 4 * (ci % H) + 1 : -1;

    for (int q = 0; q < 4; ++q) {
      double cv[6];
      child_tri(v, q, cv);
      tri_integral<CPLX>(a, tab, T, c, cv, block(cc >= 0 ? cc + q : -1), x, P, kv, acc,
                         vec + size_t(sp + q) * vs, lane);
    }
    nev += 4 * nq;
    double err = 0.0;
    const double* par = vec + size_t(top) * vs;
    for (int l = lane; l < np; l += 32) {
      double sr = 0.0, si = 0.0;
      for (int q = 0; q < 4; ++q) {
        sr += vec[size_t(sp + q) * vs + 2 * l];
        si += vec[size_t(sp + q) * vs + 2 * l + 1];
      }
      acc[2 * l] = sr;
      acc[2 * l + 1] = si;
      const double dr = sr - par[2 * l], di = si - par[2 * l + 1];
      err = fmax(err, CPLX ? sqrt(dr * dr + di * di) : fabs(dr));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) err = fmax(err, __shfl_xor_sync(kFull, err, o));
    if (err <= tol || lev >= kNqMaxLevel) {
      for (int l = lane; l < np; l += 32) {
        out[2 * l] += acc[2 * l];
        out[2 * l + 1] += acc[2 * l + 1];
      }
      sp = top;
    } else {
      for (int q = 0; q < 4; ++q)
        for (int l = lane; l < np; l += 32) {
          vec[size_t(top + q) * vs + 2 * l] = vec[size_t(sp + q) * vs + 2 * l];
          vec[size_t(top + q) * vs + 2 * l + 1] = vec[size_t(sp + q) * vs + 2 * l + 1];
        }
      if (lane == 0)
        for (int q = 0; q < 4; ++q) {
          double cv[6];
          child_tri(v, q, cv);
          for (int i = 0; i < 6; ++i) stk[kNqStackDoubles * (top + q) + i] = cv[i];
          stk[kNqStackDoubles * (top + q) + 6] = double(lev + 1);
          stk[kNqStackDoubles * (top + q) + 7] = double(cc >= 0 ? cc + q : -1);
        }
      sp = top + 4;
    }
    __syncwarp();
  }
}

// Singular integral for a target at (u0, v0) on the patch
// (host/nearquad.cpp:251-311): the patch split at the target's foot points
// on the edges into triangles, each with a Duffy map in s and a sinh map in
// the angle-like variable anchored at the closest edge point.
template <bool CPLX>
__device__ void self_integral(const NqArgs& a, const double2* tab, const NqType* T, const double* c,
                              double u0,
                              double v0, double* P, double* kv, double* acc, double* sub,
                              int lane, unsigned long long& nev) {
  const int np = T->np, nself = a.nself;
  double g[9];
  basis_geom<false, true>(T->iptype, T->norder, u0, v0, c, nullptr, 0, g);
  const double x0[3] = {g[0], g[1], g[2]};
  const double g11 = g[3] * g[3] + g[4] * g[4] + g[5] * g[5];
  const double g12 = g[3] * g[6] + g[4] * g[7] + g[5] * g[8];
  const double g22 = g[6] * g[6] + g[7] * g[7] + g[8] * g[8];
  auto gdot = [&](double ax, double ay, double bx, double by) {
    return ax * (g11 * bx + g12 * by) + ay * (g12 * bx + g22 * by);
  };
  if (lane == 0) {
    int ns = 0;
    const int nv = T->nv;
    for (int e = 0; e < nv; ++e) {
      const double ax = T->vert[2 * e], ay = T->vert[2 * e + 1];
      const double bx = T->vert[2 * ((e + 1) % nv)], by = T->vert[2 * ((e + 1) % nv) + 1];
      const double dx = bx - ax, dy = by - ay;
      const double tau = gdot(u0 - ax, v0 - ay, dx, dy) / gdot(dx, dy, dx, dy);
      double Pp[2][2], Qp[2][2];
      int nsub;
      if (tau <= 0.0) {
        Pp[0][0] = ax, Pp[0][1] = ay, Qp[0][0] = bx, Qp[0][1] = by, nsub = 1;
      } else if (tau >= 1.0) {
        Pp[0][0] = bx, Pp[0][1] = by, Qp[0][0] = ax, Qp[0][1] = ay, nsub = 1;
      } else {
        const double fx = ax + tau * dx, fy = ay + tau * dy;
        Pp[0][0] = fx, Pp[0][1] = fy, Qp[0][0] = ax, Qp[0][1] = ay;
        Pp[1][0] = fx, Pp[1][1] = fy, Qp[1][0] = bx, Qp[1][1] = by;
        nsub = 2;
      }
      for (int sb = 0; sb < nsub; ++sb) {
        const double a0 = Pp[sb][0] - u0, a1 = Pp[sb][1] - v0;
        const double b0 = Qp[sb][0] - Pp[sb][0], b1 = Qp[sb][1] - Pp[sb][1];
        const double det = fabs(a0 * b1 - a1 * b0);
        if (det <= 1e-300) continue;
        const double h = sqrt(gdot(a0, a1, a0, a1));
        const double L = sqrt(gdot(b0, b1, b0, b1));
        double* o = sub + 8 * ns;
        o[0] = a0, o[1] = a1, o[2] = b0, o[3] = b1, o[4] = det, o[5] = h / L;
        o[6] = asinh(L / h);
        ++ns;
      }
    }
    sub[64] = double(ns);
  }
  __syncwarp();
  const int nsub = int(sub[64]);
  const double* xs = a.arena + a.self_off;
  const double* ws = xs + nself;
  for (int l = lane; l < np; l += 32) acc[2 * l] = acc[2 * l + 1] = 0.0;
  const int per = nself * nself, total = nsub * per;
  for (int q0 = 0; q0 < total; q0 += 32) {
    const int q = q0 + lane;
    if (q < total) {
      const int si = q / per, rem = q - si * per;
      const int iw = rem / nself, is = rem - iw * nself;
      const double* o = sub + 8 * si;
      const double W = o[6];
      const double w = 0.5 * W * (xs[iw] + 1.0);
      const double t = o[5] * sinh(w);
      const double dtw = o[5] * cosh(w) * 0.5 * W * ws[iw];
      const double ex = o[0] + t * o[2], ey = o[1] + t * o[3];
      const double s = 0.5 * (xs[is] + 1.0);
      const double jac = s * o[4] * dtw * 0.5 * ws[is];
      double kr, ki;
      const double jn = node_val<CPLX>(a, tab, T, c, u0 + s * ex, v0 + s * ey,
                                       P + lane, x0, kr, ki);
      kv[2 * lane] = kr * jn * jac;
      kv[2 * lane + 1] = ki * jn * jac;
    }
    __syncwarp();
    accumulate<CPLX>(P, kv, min(32, total - q0), np, acc, lane);
    __syncwarp();
  }
  nev += total;
}

// Per-patch tolerance 0.1 * eps * sqrt(min_j |J(u_j, v_j)| w_j); one warp
// per patch.
__global__ void __launch_bounds__(256) nq_tol_kernel(NqArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t p = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (p >= a.npatches) return;
  const NqType* T = a.types + a.ptype[p];
  const double* c = a.coefs + 9 * a.pstart[p];
  double jw = 1e300;
  for (int j = lane; j < T->np; j += 32) {
    double g[9];
    basis_geom<false>(T->iptype, T->norder, a.arena[T->uvs + 2 * j], a.arena[T->uvs + 2 * j + 1],
                      c, nullptr, 0, g);
    const double n0 = g[4] * g[8] - g[5] * g[7];
    const double n1 = g[5] * g[6] - g[3] * g[8];
    const double n2 = g[3] * g[7] - g[4] * g[6];
    jw = fmin(jw, sqrt(n0 * n0 + n1 * n1 + n2 * n2) * a.arena[T->wts + j]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) jw = fmin(jw, __shfl_xor_sync(kFull, jw, o));
  if (lane == 0) a.ptol[p] = 0.1 * a.eps * sqrt(jw);
}

// Cache blocks of the patches [p0, p0 + n): one block per (patch, root,
// heap index h < cache_h), threads over the rule nodes.  Heap order: the
// children of h are 4h+1..4h+4 in child_tri order.
__global__ void __launch_bounds__(128) nq_cache_kernel(NqArgs a, int64_t p0) {
  const int H = a.cache_h;
  const int64_t p = p0 + int64_t(blockIdx.x) / (2 * H);
  const int rem = int(int64_t(blockIdx.x) % (2 * H));
  const int r = rem / H, h = rem % H;
  const NqType* T = a.types + a.ptype[p];
  if (r >= (T->nv == 3 ? 1 : 2)) return;
  const double* V = T->vert;
  double v[6] = {V[0], V[1], V[2 + 2 * r], V[3 + 2 * r], V[4 + 2 * r], V[5 + 2 * r]};
  int digit[8], nd = 0;
  for (int k = h; k > 0 && nd < 8; k = (k - 1) / 4) digit[nd++] = (k - 1) % 4;
  for (int i = nd - 1; i >= 0; --i) {
    double o[6];
    child_tri(v, digit[i], o);
    for (int j = 0; j < 6; ++j) v[j] = o[j];
  }
  const int np = T->np, nq = a.rule_nq[T->rule];
  const double* rule = a.arena + a.rule_off[T->rule];
  const double* c = a.coefs + 9 * a.pstart[p];
  double* blk = a.cache + a.coff[p] + size_t(r * H + h) * size_t(7 + np) * nq;
  const double ax = v[2] - v[0], ay = v[3] - v[1];
  const double bx = v[4] - v[0], by = v[5] - v[1];
  const double area2 = fabs(ax * by - ay * bx);
  for (int q = threadIdx.x; q < nq; q += blockDim.x) {
    const double xi = rule[q], eta = rule[nq + q], w = rule[2 * nq + q];
    double g[9];
    basis_geom<true>(T->iptype, T->norder, v[0] + xi * ax + eta * bx, v[1] + xi * ay + eta * by,
                     c, blk + 7 * nq + q, nq, g);
    const double n0 = g[4] * g[8] - g[5] * g[7];
    const double n1 = g[5] * g[6] - g[3] * g[8];
    const double n2 = g[3] * g[7] - g[4] * g[6];
    const double j2 = n0 * n0 + n1 * n1 + n2 * n2;
    const double inv = rsqrt(j2);  // as node_val, so cached and evaluated nodes agree
    const double jn = j2 * inv;
    blk[q] = g[0];
    blk[nq + q] = g[1];
    blk[2 * nq + q] = g[2];
    blk[3 * nq + q] = n0 * inv;
    blk[4 * nq + q] = n1 * inv;
    blk[5 * nq + q] = n2 * inv;
    blk[6 * nq + q] = jn * w * area2;
  }
}

template <bool CPLX>
__global__ void __launch_bounds__(256) nq_pair_kernel(NqArgs a) {
  extern __shared__ __align__(16) double nq_smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double2* tab = reinterpret_cast<double2*>(nq_smem);  // (cos, sin)(2 pi j / 256)
  if (CPLX) dev::fill_trig_table(tab);
  __syncthreads();
  double* P = nq_smem + 2 * dev::kTrigN + size_t(wib) * a.warp_doubles;
  double* kv = P + kNqPS * a.np_max;
  double* acc = kv + 64;
  double* out = acc + 2 * a.np_max;
  double* sub = out + 2 * a.np_max;
  double* csh = sub + kNqSubDoubles;  // the patch's coefficients, 10 per basis function
  const int64_t gw = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  double* vec = a.scratch + gw * a.scratch_per_warp;
  double* stk = vec + size_t(kNqSlots) * 2 * a.np_max;
  unsigned long long nev = 0;
  int capped = 0;
  for (;;) {
    long long idx = 0;
    if (lane == 0) idx = a.item_lo + (long long)atomicAdd(a.next, 1ull);
    idx = __shfl_sync(kFull, idx, 0);
    if (idx >= a.item_hi) break;
    const longlong2 it = a.items[idx];
    const int64_t k = it.x, t = it.y;
    const int64_t p = a.col_ind[k] - 1;
    const NqType* T = a.types + a.ptype[p];
    const int np = T->np;
    {
      const double* cg = a.coefs + 9 * a.pstart[p];
      for (int i = lane; i < 9 * np; i += 32) csh[10 * (i / 9) + i % 9] = __ldg(cg + i);
      for (int i = lane; i < np; i += 32) csh[10 * i + 9] = 0.0;
    }
    __syncwarp();
    const double* c = csh;
    double* res;
    if (idx < a.nself_items) {
      self_integral<CPLX>(a, tab, T, c, a.uvt[2 * t], a.uvt[2 * t + 1], P, kv, acc, sub, lane,
                          nev);
      res = acc;
    } else {
      const double* pcache =
          (a.cache_levels >= 0 && a.coff[p] >= 0) ? a.cache + a.coff[p] : nullptr;
      near_integral<CPLX>(a, tab, T, c, pcache, a.targ + 3 * t, a.ptol[p], P, kv, acc, out, vec,
                          stk, lane, nev, capped);
      res = out;
    }
    __syncwarp();
    // nodal weights: w_j = sum_l I_l umat(l, j)
    const double* U = a.arena + T->umat;
    const int64_t base = a.iquad[k] - 1;
    for (int j = lane; j < np; j += 32) {
      double re = 0.0, im = 0.0;
      for (int l = 0; l < np; ++l) {
        const double u = U[l * np + j];
        re = fma(res[2 * l], u, re);
        if (CPLX) im = fma(res[2 * l + 1], u, im);
      }
      if (CPLX) {
        a.wout[2 * (base + j)] = re;
        a.wout[2 * (base + j) + 1] = im;
      } else {
        a.wout[base + j] = re;
      }
    }
    __syncwarp();
  }
  if (lane == 0) {
    atomicAdd(a.stat, nev);
    if (capped) atomicAdd(a.stat + 1, 1ull);
  }
}

template <class T>
cudaError_t upload(DBuf<T>& d, const T* h, size_t n, cudaStream_t st) {
  cudaError_t e = d.alloc(std::max<size_t>(n, 1));
  if (e != cudaSuccess || n == 0) return e;
  return cudaMemcpyAsync(d.p, h, n * sizeof(T), cudaMemcpyHostToDevice, st);
}

}  // namespace

int getnearquad_gpu(const Surf& s, int ndt, int64_t nt, const double* targs,
                    const int64_t* ipatch_id, const double* uvs_targ, double eps, int kind,
                    cdouble zk, cdouble alpha, cdouble beta, int64_t nnz, const int64_t* row_ptr,
                    const int64_t* col_ind, const int64_t* iquad, int64_t nquad,
                    double* wnear_dev, cudaStream_t st, NearQuadStats* stats) {
  if (stats) *stats = NearQuadStats{};
  if (nnz == 0) return kOk;
  if (nnz < 0 || nt <= 0 || ndt < 3 || !targs || !row_ptr || !col_ind || !iquad || !wnear_dev ||
      s.npatches <= 0 || !s.srccoefs) {
    set_last_error("getnearquad_gpu: invalid arguments");
    return kErrArg;
  }
  if (row_ptr[0] != 1 || row_ptr[nt] - 1 != nnz || iquad[nnz] - 1 != nquad) {
    set_last_error("getnearquad_gpu: row_ptr / iquad inconsistent with nnz / nquad");
    return kErrArg;
  }
  // patch types, their node/weight/umat tables and the rules
  std::map<std::pair<int, int>, int> tmap;
  std::vector<NqType> types;
  std::vector<double> arena;
  std::vector<int> ptype(s.npatches);
  std::vector<int64_t> pstart(s.npatches);
  int np_max = 0;
  for (int64_t p = 0; p < s.npatches; ++p) {
    const int ip = int(s.iptype[p]), no = int(s.norders[p]);
    const int np = int(s.npols(p));
    if (!valid_patch(ip, no) || npols_of(ip, no) != np) {
      set_last_error("getnearquad_gpu: patch " + std::to_string(p + 1) + " has an invalid type/order");
      return kErrArg;
    }
    if (np > kNearQuadMaxNp) {
      set_last_error("getnearquad_gpu: patch " + std::to_string(p + 1) + " has " +
                     std::to_string(np) + " basis functions (device limit " +
                     std::to_string(kNearQuadMaxNp) + ")");
      return kErrArg;
    }
    auto key = std::make_pair(ip, no);
    auto f = tmap.find(key);
    if (f == tmap.end()) {
      NqType T{};
      T.iptype = ip;
      T.norder = no;
      T.np = np;
      T.nv = boundary_vertices(ip, T.vert);
      const int ng = nearquad_tri_ng(no);
      T.rule = ng == 8 ? 0 : (ng == 10 ? 1 : 2);
      std::vector<double> uvs(2 * np), umat(size_t(np) * np), vmat(size_t(np) * np), w(np);
      if (disc_exps(ip, no, uvs.data(), umat.data(), vmat.data(), w.data())) {
        set_last_error("getnearquad_gpu: no discretisation tables for a patch type");
        return kErrTables;
      }
      T.uvs = int(arena.size());
      arena.insert(arena.end(), uvs.begin(), uvs.end());
      T.wts = int(arena.size());
      arena.insert(arena.end(), w.begin(), w.end());
      T.umat = int(arena.size());
      arena.insert(arena.end(), umat.begin(), umat.end());
      f = tmap.emplace(key, int(types.size())).first;
      types.push_back(T);
    }
    ptype[p] = f->second;
    pstart[p] = s.start(p);
    np_max = std::max(np_max, np);
  }
  NqArgs a{};
  const int ngs[3] = {8, 10, 12};
  for (int r = 0; r < 3; ++r) {
    std::vector<double> xi, eta, w;
    nearquad_tri_rule(ngs[r], xi, eta, w);
    a.rule_off[r] = int(arena.size());
    a.rule_nq[r] = int(xi.size());
    arena.insert(arena.end(), xi.begin(), xi.end());
    arena.insert(arena.end(), eta.begin(), eta.end());
    arena.insert(arena.end(), w.begin(), w.end());
  }
  a.nself = nearquad_self_order(eps);
  {
    std::vector<double> x(a.nself), w(a.nself);
    gauss_legendre(a.nself, x.data(), w.data());
    a.self_off = int(arena.size());
    arena.insert(arena.end(), x.begin(), x.end());
    arena.insert(arena.end(), w.begin(), w.end());
  }
  // work items, self pairs first, with the checks that keep every device
  // access in bounds: patch index, row of wnear, self parameters
  std::vector<longlong2> items, near_items;
  items.reserve(nt);
  near_items.reserve(nnz);
  for (int64_t t = 0; t < nt; ++t) {
    if (row_ptr[t + 1] < row_ptr[t]) {
      set_last_error("getnearquad_gpu: row_ptr not monotone");
      return kErrArg;
    }
    for (int64_t k = row_ptr[t] - 1; k < row_ptr[t + 1] - 1; ++k) {
      const int64_t p = col_ind[k] - 1;
      if (p < 0 || p >= s.npatches || iquad[k + 1] - iquad[k] != s.npols(p) || iquad[k] < 1) {
        set_last_error("getnearquad_gpu: col_ind / iquad entry " + std::to_string(k + 1) +
                       " out of range");
        return kErrArg;
      }
      const bool self = ipatch_id && ipatch_id[t] == p + 1;
      if (self && !uvs_targ) {
        set_last_error("getnearquad_gpu: on-surface targets need uvs_targ");
        return kErrArg;
      }
      (self ? items : near_items).push_back(make_longlong2(k, t));
    }
  }
  // near pairs grouped by patch (targets in order within a patch), so the
  // warps running at one time share a few patches' cache blocks
  const int64_t nself_items = int64_t(items.size());
  std::vector<int64_t> pfirst(s.npatches + 1, 0);
  for (const auto& it : near_items) ++pfirst[col_ind[it.x]];
  for (int64_t p = 0; p < s.npatches; ++p) pfirst[p + 1] += pfirst[p];
  items.resize(size_t(nself_items) + near_items.size());
  {
    std::vector<int64_t> fill(pfirst.begin(), pfirst.end() - 1);
    for (const auto& it : near_items) items[size_t(nself_items + fill[col_ind[it.x] - 1]++)] = it;
  }
  near_items.clear();
  near_items.shrink_to_fit();
  std::vector<double> targ3(3 * size_t(nt)), uvt(uvs_targ ? 2 * size_t(nt) : 0);
  for (int64_t t = 0; t < nt; ++t)
    for (int i = 0; i < 3; ++i) targ3[3 * t + i] = targs[size_t(ndt) * t + i];
  if (uvs_targ) std::copy(uvs_targ, uvs_targ + 2 * size_t(nt), uvt.begin());

  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int warp_doubles = kNqPS * np_max + 64 + 4 * np_max + kNqSubDoubles + 10 * np_max;
  const size_t warp_bytes = sizeof(double) * size_t(warp_doubles);
  const size_t tab_bytes = sizeof(double) * 2 * dev::kTrigN;
  auto kern = kind == 1 ? nq_pair_kernel<true> : nq_pair_kernel<false>;
  // warps per block: the most resident warps per SM, larger blocks on ties
  int wpb = 0, bps = 0;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(std::min<size_t>(tab_bytes + 8 * warp_bytes, 227u << 10)));
  for (int w = 8; w >= 1 && e == cudaSuccess; --w) {
    if (tab_bytes + w * warp_bytes > (227u << 10)) continue;
    int b = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, 32 * w, tab_bytes + w * warp_bytes);
    if (e == cudaSuccess && b * w > bps * wpb) {
      wpb = w;
      bps = b;
    }
  }
  const size_t smem = tab_bytes + warp_bytes * std::max(wpb, 1);
  if (e != cudaSuccess || bps < 1) {
    set_last_error(std::string("getnearquad_gpu: launch configuration: ") + cudaGetErrorString(e));
    return kErrCuda;
  }
  // cache: uniform levels 0..L of every root triangle (L from
  // BIE_NEARQUAD_CACHE_LEVELS, default 3, at most 5, -1 = none), built for
  // groups of consecutive patches whose blocks fit in the group budget
  // (min(4 GiB, free memory / 4), or BIE_NEARQUAD_CACHE_BUDGET_MB)
  int levels = 3;
  if (const char* ev = std::getenv("BIE_NEARQUAD_CACHE_LEVELS")) levels = std::atoi(ev);
  levels = std::max(-1, std::min(5, levels));
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  size_t budget = std::min<size_t>(size_t(4) << 30, free_b / 4);
  if (const char* ev = std::getenv("BIE_NEARQUAD_CACHE_BUDGET_MB"))
    budget = size_t(std::max(1, std::atoi(ev))) << 20;
  const int H = levels >= 0 ? ((1 << (2 * (levels + 1))) - 1) / 3 : 0;
  std::vector<int64_t> coff(s.npatches, -1);
  std::vector<std::pair<int64_t, int64_t>> groups;  // patch ranges
  size_t cache_doubles = 0;
  if (levels >= 0) {
    size_t used = 0;
    int64_t g0 = 0;
    for (int64_t p = 0; p < s.npatches; ++p) {
      const NqType& T = types[ptype[p]];
      const size_t need = size_t(T.nv == 3 ? 1 : 2) * H * size_t(7 + T.np) * a.rule_nq[T.rule];
      if (need * sizeof(double) > budget) {
        levels = -1;
        break;
      }
      if ((used + need) * sizeof(double) > budget) {
        groups.emplace_back(g0, p);
        g0 = p;
        used = 0;
      }
      coff[p] = int64_t(used);
      used += need;
      cache_doubles = std::max(cache_doubles, used);
    }
    if (levels >= 0) groups.emplace_back(g0, s.npatches);
  }
  if (levels < 0) {
    groups.assign(1, {0, s.npatches});
    std::fill(coff.begin(), coff.end(), -1);
    cache_doubles = 0;
  }
  const int64_t want = (int64_t(items.size()) + wpb - 1) / wpb;
  const int blocks = int(std::max<int64_t>(1, std::min<int64_t>(int64_t(nsm) * bps, want)));
  const int64_t nwarps = int64_t(blocks) * wpb;

  DBuf<double> d_coefs, d_arena, d_targ, d_uvt, d_tol, d_scratch, d_cache;
  DBuf<NqType> d_types;
  DBuf<int> d_ptype;
  DBuf<int64_t> d_pstart, d_col, d_iq, d_coff;
  const int nlaunch = 1 + int(groups.size());
  DBuf<longlong2> d_items;
  DBuf<unsigned long long> d_cnt;
  const size_t per_warp = size_t(kNqSlots) * 2 * np_max + size_t(kNqSlots) * kNqStackDoubles;
  if ((e = upload(d_coefs, s.srccoefs, 9 * size_t(s.npts), st)) != cudaSuccess ||
      (e = upload(d_arena, arena.data(), arena.size(), st)) != cudaSuccess ||
      (e = upload(d_targ, targ3.data(), targ3.size(), st)) != cudaSuccess ||
      (e = upload(d_uvt, uvt.data(), uvt.size(), st)) != cudaSuccess ||
      (e = d_tol.alloc(s.npatches)) != cudaSuccess ||
      (e = d_scratch.alloc(per_warp * nwarps)) != cudaSuccess ||
      (e = upload(d_types, types.data(), types.size(), st)) != cudaSuccess ||
      (e = upload(d_ptype, ptype.data(), ptype.size(), st)) != cudaSuccess ||
      (e = upload(d_pstart, pstart.data(), pstart.size(), st)) != cudaSuccess ||
      (e = upload(d_col, col_ind, size_t(nnz), st)) != cudaSuccess ||
      (e = upload(d_iq, iquad, size_t(nnz) + 1, st)) != cudaSuccess ||
      (e = upload(d_items, items.data(), items.size(), st)) != cudaSuccess ||
      (e = upload(d_coff, coff.data(), coff.size(), st)) != cudaSuccess ||
      (e = d_cache.alloc(std::max<size_t>(cache_doubles, 1))) != cudaSuccess ||
      (e = d_cnt.alloc(nlaunch + 2)) != cudaSuccess ||
      (e = cudaMemsetAsync(d_cnt.p, 0, (nlaunch + 2) * sizeof(unsigned long long), st)) !=
          cudaSuccess) {
    set_last_error(std::string("getnearquad_gpu: device buffers: ") + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? kErrNoMem : kErrCuda;
  }
  fill_basis_constants(st);
  a.zr = zk.real();
  a.zi = zk.imag();
  a.ar = alpha.real();
  a.ai = kind == 1 ? alpha.imag() : 0.0;
  a.br = beta.real();
  a.bi = kind == 1 ? beta.imag() : 0.0;
  a.eps = eps;
  a.coefs = d_coefs.p;
  a.types = d_types.p;
  a.ptype = d_ptype.p;
  a.pstart = d_pstart.p;
  a.ptol = d_tol.p;
  a.arena = d_arena.p;
  a.targ = d_targ.p;
  a.uvt = d_uvt.p;
  a.items = d_items.p;
  a.nself_items = nself_items;
  a.cache = d_cache.p;
  a.coff = d_coff.p;
  a.cache_levels = levels;
  a.cache_h = H;
  a.npatches = s.npatches;
  a.col_ind = d_col.p;
  a.iquad = d_iq.p;
  a.wout = wnear_dev;
  a.scratch = d_scratch.p;
  a.scratch_per_warp = int64_t(per_warp);
  a.np_max = np_max;
  a.warp_doubles = warp_doubles;
  a.stat = d_cnt.p + nlaunch;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaEventCreate(&ev[0]);
  cudaEventCreate(&ev[1]);
  nq_tol_kernel<<<unsigned((s.npatches * 32 + 255) / 256), 256, 0, st>>>(a);
  cudaEventRecord(ev[0], st);
  int64_t launches = 1;
  // self pairs (no cache), then each patch group: its cache, its near pairs
  a.item_lo = 0;
  a.item_hi = nself_items;
  a.next = d_cnt.p;
  if (nself_items > 0) {
    kern<<<blocks, 32 * wpb, smem, st>>>(a);
    ++launches;
  }
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    const int64_t pa = groups[gi].first, pb = groups[gi].second;
    a.item_lo = nself_items + pfirst[pa];
    a.item_hi = nself_items + pfirst[pb];
    a.next = d_cnt.p + 1 + gi;
    if (a.item_hi == a.item_lo) continue;
    if (levels >= 0) {
      nq_cache_kernel<<<unsigned((pb - pa) * 2 * H), 128, 0, st>>>(a, pa);
      ++launches;
    }
    kern<<<blocks, 32 * wpb, smem, st>>>(a);
    ++launches;
  }
  cudaEventRecord(ev[1], st);
  dev::note_launches(launches);
  unsigned long long cnt[2] = {0, 0};
  cudaMemcpyAsync(cnt, d_cnt.p + nlaunch, sizeof cnt, cudaMemcpyDeviceToHost, st);
  e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();
  float ms = 0.f;
  if (e == cudaSuccess) cudaEventElapsedTime(&ms, ev[0], ev[1]);
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (e != cudaSuccess) {
    set_last_error(std::string("getnearquad_gpu: ") + cudaGetErrorString(e));
    return kErrCuda;
  }
  if (stats) {
    stats->device_ms = ms;
    stats->kernel_evals = int64_t(cnt[0]);
    stats->self_targets = nself_items;
    stats->near_targets = int64_t(items.size()) - nself_items;
  }
  if (cnt[1]) {
    set_last_error("getnearquad_gpu: " + std::to_string(cnt[1]) +
                   " warps hit the refinement-step cap");
    return kErrTimeout;
  }
  return kOk;
}

}  // namespace bie
