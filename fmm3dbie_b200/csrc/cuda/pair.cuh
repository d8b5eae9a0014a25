// Pair functions of the far field (one source's contribution to one target)
// and the vector types they use, shared by the kernels that must evaluate the
// kernel identically: the far-field kernels, the FP32 fold that cancels their
// near-pair values, and the tensor-core far field.
#pragma once
#include <cuda_runtime.h>

#include "trig_table.cuh"

namespace bie {
namespace dev {
namespace {

template <typename R>
struct Vec;
template <>
struct Vec<float> {
  using T2 = float2;
  using T4 = float4;
};
template <>
struct Vec<double> {
  using T2 = double2;
  using T4 = double4;
};

// Contribution of one source to one target: charge c = (s.x, s.y), dipole
// strength d = (s.z, s.w) along the source normal n,
//   e^{ikr}/r [ c + d (n.(t-s)) (1 - ikr) / r^2 ],   (1/(4 pi) is in c, d).
// The phase kr carries an absolute error of about kr 2^-24 in single
// precision already; __sincosf's scaled argument adds an error of the same
// order, so no separate range reduction is done.
// CHECK = false drops the r^2 >= thresh^2 test; callers use it only where no
// pair of the tile can fall below the threshold, so the result is the same.
template <bool CHECK = true>
__device__ __forceinline__ void pair_helm(float tx, float ty, float tz, const float4 g0,
                                          const float2 g1, const float4 s, float k, float kim,
                                          float thr2, bool ck, float& pr, float& pi,
                                          const double2* = nullptr) {
  const float dx = tx - g0.x, dy = ty - g0.y, dz = tz - g0.z;
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  const float rinv = (!CHECK || r2 >= thr2) ? rsqrtf(r2) : 0.0f;
  const float r = r2 * rinv;
  const float kr = k * r;
  float sn, cs;
  __sincosf(kr, &sn, &cs);
  float rs = rinv;
  if (ck) rs *= __expf(-kim * r);
  const float dn = fmaf(dx, g0.w, fmaf(dy, g1.x, dz * g1.y));
  const float u = dn * (rinv * rinv);
  float xr, xi;
  if (ck) {
    // x = c + d u ((1 + kim r) - i kr)  for complex k = kr + i kim
    const float ur = u * (1.0f + kim * r);
    const float p = u * kr;
    xr = fmaf(s.w, p, fmaf(s.z, ur, s.x));
    xi = fmaf(-s.z, p, fmaf(s.w, ur, s.y));
  } else {
    // x = c + d u (1 - i kr) = c + u (d_r + d_i kr, d_i - d_r kr)
    xr = fmaf(u, fmaf(s.w, kr, s.z), s.x);
    xi = fmaf(u, fmaf(-s.z, kr, s.w), s.y);
  }
  const float er = xr * rs, ei = xi * rs;
  pr = fmaf(cs, er, fmaf(-sn, ei, pr));
  pi = fmaf(cs, ei, fmaf(sn, er, pi));
}

// FP64: tab is the far-field sine/cosine table (sincos_far; kFarTrigN
// entries) or null for the library sincos; 1/r from rsqrt_far.
template <bool CHECK = true>
__device__ __forceinline__ void pair_helm(double tx, double ty, double tz, const double4 g0,
                                          const double2 g1, const double4 s, double k, double kim,
                                          double thr2, bool ck, double& pr, double& pi,
                                          const double2* tab = nullptr) {
  const double dx = tx - g0.x, dy = ty - g0.y, dz = tz - g0.z;
  const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
  const double rinv = (!CHECK || r2 >= thr2) ? rsqrt_far(r2) : 0.0;
  const double r = r2 * rinv;
  const double kr = k * r;
  double sn, cs;
  if (tab)
    sincos_far(kr, tab, sn, cs);
  else
    sincos(kr, &sn, &cs);
  double rs = rinv;
  if (ck) rs *= exp(-kim * r);
  const double dn = fma(dx, g0.w, fma(dy, g1.x, dz * g1.y));
  const double q = dn * (rinv * rinv);
  // x = c + d q (1 - ikr) (real k) or c + d q ((1 + kim r) - ikr)
  double xr, xi;
  if (ck) {
    const double qr = q * fma(kim, r, 1.0), p = q * kr;
    xr = fma(s.w, p, fma(s.z, qr, s.x));
    xi = fma(-s.z, p, fma(s.w, qr, s.y));
  } else {
    xr = fma(q, fma(s.w, kr, s.z), s.x);
    xi = fma(q, fma(-s.z, kr, s.w), s.y);
  }
  const double er = xr * rs, ei = xi * rs;
  pr = fma(cs, er, fma(-sn, ei, pr));
  pi = fma(cs, ei, fma(sn, er, pi));
}

template <typename R, bool CHECK = true>
__device__ __forceinline__ void pair_lap(R tx, R ty, R tz, const typename Vec<R>::T4 g0,
                                         const typename Vec<R>::T2 g1,
                                         const typename Vec<R>::T2 s, R thr2, R& p) {
  const R dx = tx - g0.x, dy = ty - g0.y, dz = tz - g0.z;
  const R r2 = fma(dx, dx, fma(dy, dy, dz * dz));
  R rinv;
  if constexpr (sizeof(R) == 4)
    rinv = (!CHECK || r2 >= thr2) ? rsqrtf(r2) : R(0);
  else
    rinv = (!CHECK || r2 >= thr2) ? rsqrt_far(r2) : R(0);
  const R dn = fma(dx, g0.w, fma(dy, g1.x, dz * g1.y));
  const R e = fma(s.y * dn, rinv * rinv, s.x);
  p = fma(e, rinv, p);
}

// Two targets against one source with the packed FP32 instructions of
// sm_100 (add/mul/fma .f32x2: two lanes per instruction, each lane rounded
// as the scalar instruction rounds it): lane .x is one target, lane .y the
// other.  Source values come as pairs of equal lanes: the coordinates
// negated (t - s is then one packed add), the normal, the charge c, the
// dipole strength d and -d_r (the imaginary part then needs no negation).
// The real part accumulates as pa - pb (pa = sum cos er, pb = sum sin ei),
// which avoids negating the sine.  Per lane the pair value is pair_helm's:
// the same operations on the same operands in the same order.
template <bool CHECK = true>
__device__ __forceinline__ void pair_helm_x2(const float2 tx, const float2 ty, const float2 tz,
                                             const float2 msx, const float2 msy, const float2 msz,
                                             const float2 nx, const float2 ny, const float2 nz,
                                             const float2 cr, const float2 ci, const float2 dr,
                                             const float2 di, const float2 mdr, const float2 k2,
                                             const float2 kim2, float thr2, bool ck, float2& pa,
                                             float2& pb, float2& pi) {
  const float2 dx = __fadd2_rn(tx, msx), dy = __fadd2_rn(ty, msy), dz = __fadd2_rn(tz, msz);
  const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
  float2 rinv;
  rinv.x = (!CHECK || r2.x >= thr2) ? rsqrtf(r2.x) : 0.0f;
  rinv.y = (!CHECK || r2.y >= thr2) ? rsqrtf(r2.y) : 0.0f;
  const float2 r = __fmul2_rn(r2, rinv);
  const float2 kr = __fmul2_rn(k2, r);
  float2 sn, cs;
  __sincosf(kr.x, &sn.x, &cs.x);
  __sincosf(kr.y, &sn.y, &cs.y);
  float2 rs = rinv;
  if (ck) {
    rs.x *= __expf(-kim2.x * r.x);
    rs.y *= __expf(-kim2.y * r.y);
  }
  const float2 dn = __ffma2_rn(dx, nx, __ffma2_rn(dy, ny, __fmul2_rn(dz, nz)));
  const float2 u = __fmul2_rn(dn, __fmul2_rn(rinv, rinv));
  float2 xr, xi;
  if (ck) {
    const float2 ur = __fmul2_rn(u, __ffma2_rn(kim2, r, make_float2(1.0f, 1.0f)));
    const float2 p = __fmul2_rn(u, kr);
    xr = __ffma2_rn(di, p, __ffma2_rn(dr, ur, cr));
    xi = __ffma2_rn(mdr, p, __ffma2_rn(di, ur, ci));
  } else {
    xr = __ffma2_rn(u, __ffma2_rn(di, kr, dr), cr);
    xi = __ffma2_rn(u, __ffma2_rn(mdr, kr, di), ci);
  }
  const float2 er = __fmul2_rn(xr, rs), ei = __fmul2_rn(xi, rs);
  pa = __ffma2_rn(cs, er, pa);
  pb = __ffma2_rn(sn, ei, pb);
  pi = __ffma2_rn(cs, ei, __ffma2_rn(sn, er, pi));
}

// Laplace counterpart of pair_helm_x2 (charge c, dipole strength d).
template <bool CHECK = true>
__device__ __forceinline__ void pair_lap_x2(const float2 tx, const float2 ty, const float2 tz,
                                            const float2 msx, const float2 msy, const float2 msz,
                                            const float2 nx, const float2 ny, const float2 nz,
                                            const float2 c, const float2 d, float thr2,
                                            float2& p) {
  const float2 dx = __fadd2_rn(tx, msx), dy = __fadd2_rn(ty, msy), dz = __fadd2_rn(tz, msz);
  const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
  float2 rinv;
  rinv.x = (!CHECK || r2.x >= thr2) ? rsqrtf(r2.x) : 0.0f;
  rinv.y = (!CHECK || r2.y >= thr2) ? rsqrtf(r2.y) : 0.0f;
  const float2 dn = __ffma2_rn(dx, nx, __ffma2_rn(dy, ny, __fmul2_rn(dz, nz)));
  const float2 e = __ffma2_rn(__fmul2_rn(d, dn), __fmul2_rn(rinv, rinv), c);
  p = __ffma2_rn(e, rinv, p);
}

// Unit responses of one source at one target, for evaluating several
// densities from one kernel evaluation: G = e^{ikr}/r and D = G u (1 - ikr)
// with u = n.(t-s)/r^2 (complex k = kr + i kim: 1 - ikr becomes
// (1 + kim r) - i kr r); a source with charge c and dipole strength d then
// contributes c G + d D, as pair_helm computes it.  Laplace: G = 1/r,
// D = u/r.  CHECK = false drops the threshold test (as in pair_helm).
template <bool CHECK = true>
__device__ __forceinline__ void pair_helm_unit(float tx, float ty, float tz, const float4 g0,
                                               const float2 g1, float k, float kim, float thr2,
                                               bool ck, float& gr, float& gi, float& dr,
                                               float& di, const double2* = nullptr) {
  const float dx = tx - g0.x, dy = ty - g0.y, dz = tz - g0.z;
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  const float rinv = (!CHECK || r2 >= thr2) ? rsqrtf(r2) : 0.0f;
  const float r = r2 * rinv;
  const float kr = k * r;
  float sn, cs;
  __sincosf(kr, &sn, &cs);
  float rs = rinv;
  if (ck) rs *= __expf(-kim * r);
  gr = cs * rs;
  gi = sn * rs;
  const float u = fmaf(dx, g0.w, fmaf(dy, g1.x, dz * g1.y)) * (rinv * rinv);
  const float fr = ck ? u * (1.0f + kim * r) : u, fi = -u * kr;
  dr = fmaf(gr, fr, -gi * fi);
  di = fmaf(gr, fi, gi * fr);
}

template <bool CHECK = true>
__device__ __forceinline__ void pair_helm_unit(double tx, double ty, double tz, const double4 g0,
                                               const double2 g1, double k, double kim,
                                               double thr2, bool ck, double& gr, double& gi,
                                               double& dr, double& di,
                                               const double2* tab = nullptr) {
  const double dx = tx - g0.x, dy = ty - g0.y, dz = tz - g0.z;
  const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
  const double rinv = (!CHECK || r2 >= thr2) ? rsqrt_far(r2) : 0.0;
  const double r = r2 * rinv;
  const double kr = k * r;
  double sn, cs;
  if (tab)
    sincos_far(kr, tab, sn, cs);
  else
    sincos(kr, &sn, &cs);
  double rs = rinv;
  if (ck) rs *= exp(-kim * r);
  gr = cs * rs;
  gi = sn * rs;
  const double u = fma(dx, g0.w, fma(dy, g1.x, dz * g1.y)) * (rinv * rinv);
  const double fr = ck ? u * (1.0 + kim * r) : u, fi = -u * kr;
  dr = fma(gr, fr, -gi * fi);
  di = fma(gr, fi, gi * fr);
}

template <typename R, bool CHECK = true>
__device__ __forceinline__ void pair_lap_unit(R tx, R ty, R tz, const typename Vec<R>::T4 g0,
                                              const typename Vec<R>::T2 g1, R thr2, R& g, R& dd) {
  const R dx = tx - g0.x, dy = ty - g0.y, dz = tz - g0.z;
  const R r2 = fma(dx, dx, fma(dy, dy, dz * dz));
  R rinv;
  if constexpr (sizeof(R) == 4)
    rinv = (!CHECK || r2 >= thr2) ? rsqrtf(r2) : R(0);
  else
    rinv = (!CHECK || r2 >= thr2) ? rsqrt_far(r2) : R(0);
  const R dn = fma(dx, g0.w, fma(dy, g1.x, dz * g1.y));
  g = rinv;
  dd = dn * rinv * rinv * rinv;
}

// Contribution of a charge q = (q.x, q.y) (complex for Helmholtz) at g0.xyz to
// a well-separated target: q e^{ikr}/r (Laplace: q.x / r).  Used for the
// proxy charges of the hierarchical far field, which carry no dipoles.
template <int KIND>
__device__ __forceinline__ void pair_charge(float tx, float ty, float tz, const float4 g0,
                                            const float4 q, float k, float kim, bool ck, float& pr,
                                            float& pi, const double2* = nullptr) {
  const float dx = tx - g0.x, dy = ty - g0.y, dz = tz - g0.z;
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  const float rinv = rsqrtf(r2);
  if constexpr (KIND == 1) {
    const float r = r2 * rinv;
    float sn, cs;
    __sincosf(k * r, &sn, &cs);
    float rs = rinv;
    if (ck) rs *= __expf(-kim * r);
    const float er = q.x * rs, ei = q.y * rs;
    pr = fmaf(cs, er, fmaf(-sn, ei, pr));
    pi = fmaf(cs, ei, fmaf(sn, er, pi));
  } else {
    pr = fmaf(q.x, rinv, pr);
  }
}

template <int KIND>
__device__ __forceinline__ void pair_charge(double tx, double ty, double tz, const double4 g0,
                                            const double4 q, double k, double kim, bool ck,
                                            double& pr, double& pi, const double2* tab = nullptr) {
  const double dx = tx - g0.x, dy = ty - g0.y, dz = tz - g0.z;
  const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
  const double rinv = rsqrt_far(r2);
  if constexpr (KIND == 1) {
    const double r = r2 * rinv;
    double sn, cs;
    if (tab)
      sincos_far(k * r, tab, sn, cs);
    else
      sincos(k * r, &sn, &cs);
    double rs = rinv;
    if (ck) rs *= exp(-kim * r);
    const double er = q.x * rs, ei = q.y * rs;
    pr = fma(cs, er, fma(-sn, ei, pr));
    pi = fma(cs, ei, fma(sn, er, pi));
  } else {
    pr = fma(q.x, rinv, pr);
  }
}

}  // namespace
}  // namespace dev
}  // namespace bie
