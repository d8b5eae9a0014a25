// Table-driven FP64 sine and cosine shared by the far-field and
// near-quadrature kernels.
#pragma once

namespace bie {
namespace dev {

// Table-driven sine and cosine (FP64) (the table-driven
// reduction of P. T. P. Tang, ACM TOMS 15 (1989) / 16 (1990)):
//   x = j (2 pi / N) + rho,  |rho| <= pi / N,
//   sin x = S_j cos rho + C_j sin rho,  cos x = C_j cos rho - S_j sin rho,
// with (C_j, S_j) = (cos, sin)(2 pi j / N) from a per-block table and the
// Taylor series of sin rho (to rho^5) and cos rho (to rho^6), whose first
// omitted terms are below 1e-17 for |rho| <= pi/256.  2 pi / N is split as
// C1 + C2 with C1 rounded to 24 bits, so j C1 is exact for |j| < 2^29.
constexpr int kTrigN = 256;
constexpr double kTrigStep = 0.02454369260617026;     // 2 pi / 256
constexpr double kTrigInvStep = 40.74366543152521;    // 256 / (2 pi)
constexpr double kTrigC1 = 0.02454369328916073;       // float(2 pi / 256)
constexpr double kTrigC2 = -6.829904687791004e-10;    // 2 pi / 256 - C1

// Fills tab[q] = (cos, sin)(2 pi q / N) with the block's threads.
__device__ __forceinline__ void fill_trig_table(double2* tab) {
  for (int q = threadIdx.x; q < kTrigN; q += blockDim.x) {
    double sq, cq;
    sincos(double(q) * kTrigStep, &sq, &cq);
    tab[q] = make_double2(cq, sq);
  }
}

__device__ __forceinline__ void sincos_tab(double x, const double2* tab, double& s, double& c) {
  const double jd = rint(x * kTrigInvStep);
  const int j = int(jd) & (kTrigN - 1);
  double rho = fma(-jd, kTrigC1, x);
  rho = fma(-jd, kTrigC2, rho);
  const double r2 = rho * rho;
  const double sp = fma(rho * r2, fma(r2, 1.0 / 120.0, -1.0 / 6.0), rho);
  const double cp = fma(r2, fma(r2, fma(r2, -1.0 / 720.0, 1.0 / 24.0), -0.5), 1.0);
  const double2 t = tab[j];
  s = fma(t.y, cp, t.x * sp);
  c = fma(t.x, cp, -(t.y * sp));
}

// The far-field variant of the same method, for the direct and hierarchical
// far-field kernels, whose phases stay below 100 and whose products only need
// ~1e-14: the same 256-entry table and series, with j found by the
// round-to-integer of adding 1.5 * 2^52 (no conversion instructions) and the
// reduction x - j (2 pi / N) in one fused multiply-add with 2 pi / N rounded
// to FP64: its error, j times the rounding of the step (at most 1.7e-18), is
// below 1e-14 for x < 100.
constexpr int kFarTrigN = kTrigN;
constexpr double kRoundMagic = 6755399441055744.0;  // 1.5 * 2^52

__device__ __forceinline__ void fill_far_trig_table(double2* tab) { fill_trig_table(tab); }

__device__ __forceinline__ void sincos_far(double x, const double2* tab, double& s, double& c) {
  const double u = fma(x, kTrigInvStep, kRoundMagic);  // 1.5 2^52 + rint(x / step)
  const int j = __double2loint(u) & (kFarTrigN - 1);
  const double jd = u - kRoundMagic;
  const double rho = fma(-jd, kTrigStep, x);
  const double r2 = rho * rho;
  const double sp = fma(rho * r2, fma(r2, 1.0 / 120.0, -1.0 / 6.0), rho);
  const double cp = fma(r2, fma(r2, fma(r2, -1.0 / 720.0, 1.0 / 24.0), -0.5), 1.0);
  const double2 t = tab[j];
  s = fma(t.y, cp, t.x * sp);
  c = fma(t.x, cp, -(t.y * sp));
}

// 1/sqrt(a) in FP64 for a > 0 in the FP32 normal range: the FP32 hardware
// approximation y0 (relative error e0 ~ 2^-22) refined by one third-order
// step of the binomial series of (1 - e)^(-1/2), e = 1 - a y0^2:
//   y = y0 (1 + e/2 + 3 e^2 / 8),
// whose truncation error 5 e^3 / 16 ~ 1e-20 is below the FP64 rounding.
__device__ __forceinline__ double rsqrt_far(double a) {
  const double y0 = double(rsqrtf(float(a)));
  const double e = fma(-(a * y0), y0, 1.0);
  return fma(y0 * e, fma(e, 0.375, 0.5), y0);
}

}  // namespace dev
}  // namespace bie
