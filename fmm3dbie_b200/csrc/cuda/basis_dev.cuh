// Patch bases and geometry on the device: the Koornwinder (triangles) and
// tensor Legendre / Chebyshev (quads) recurrences of host/basis.cpp with
// their constants in constant memory, and the geometry sum over a patch's
// coefficients.  Each translation unit that includes this header gets its
// own constant tables and fills them with fill_basis_constants() on the
// stream of its first launch.
#pragma once
#include <cmath>
#include <vector>

#include <cuda_runtime.h>

#include "../host/basis.h"

namespace bie {
namespace {

constexpr int kBdTriOrder = kMaxOrder;  // Koornwinder tables up to order 20
constexpr int kBdLeg = 41;              // tensor bases up to order 40
constexpr int kBdJac = kBdTriOrder + 1;

// npols of a patch type and order (get_npols).
__host__ __device__ __forceinline__ int npols_dev(int iptype, int n) {
  return iptype == 1 ? (n + 1) * (n + 2) / 2 : (n + 1) * (n + 1);
}

// Recurrence constants of the bases (uniform across a warp, so constant
// memory broadcasts them):
//   Koornwinder normalisation sqrt((2k+1)(2n+2)) at n(n+1)/2 + k;
//   Jacobi P_m^{(0,2k+1)}: P_{m+1} = (cJacP x - cJacQ) P_m - cJacR P_{m-1} at k*21+m;
//   Legendre: P_{k+1} = cLegA x P_k - cLegB P_{k-1}.
__constant__ double cKoornNorm[(kBdTriOrder + 1) * (kBdTriOrder + 2) / 2];
__constant__ double cJacP[kBdJac * kBdJac];
__constant__ double cJacQ[kBdJac * kBdJac];
__constant__ double cJacR[kBdJac * kBdJac];
__constant__ double cLegA[kBdLeg];
__constant__ double cLegB[kBdLeg];

// Basis values at (u, v) -> prow[l * ps], l < np (when STORE) and the geometry
// g = sum_l coefs_l P_l: xyz, d/du, d/dv.  Same bases as basis_pols.
// Coefficients: 9 per basis function in global memory, or (SHARED) the
// warp's copy in shared memory padded to 10 so that pairs load as one
// 16-byte access.
template <bool STORE, bool SHARED = false>
__device__ void basis_geom(int iptype, int n, double u, double v, const double* __restrict__ c,
                           double* prow, int ps, double* g) {
#pragma unroll
  for (int k = 0; k < 9; ++k) g[k] = 0.0;
  auto emit = [&](int idx, double p) {
    if (STORE) prow[idx * ps] = p;
    if (SHARED) {
      const double2* ci = reinterpret_cast<const double2*>(c + 10 * idx);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const double2 cc = ci[k];
        g[2 * k] = fma(cc.x, p, g[2 * k]);
        g[2 * k + 1] = fma(cc.y, p, g[2 * k + 1]);
      }
      g[8] = fma(ci[4].x, p, g[8]);
    } else {
      const double* ci = c + 9 * idx;
#pragma unroll
      for (int k = 0; k < 9; ++k) g[k] = fma(__ldg(ci + k), p, g[k]);
    }
  };
  if (iptype == 1) {
    double leg[kBdTriOrder + 1];
    const double z = 2.0 * u + v - 1.0, y = 1.0 - v, y2 = y * y, x = 1.0 - 2.0 * v;
    leg[0] = 1.0;
    if (n >= 1) leg[1] = z;
    for (int k = 1; k < n; ++k) leg[k + 1] = cLegA[k] * z * leg[k] - cLegB[k] * y2 * leg[k - 1];
    for (int k = 0; k <= n; ++k) {
      const double lk = leg[k];
      const double b = 2.0 * k + 1.0;
      int idx = k * (k + 1) / 2 + k;
      emit(idx, lk * cKoornNorm[idx]);
      if (n - k < 1) continue;
      double jp = 1.0, jc = 0.5 * ((b + 2.0) * x - b);
      idx = (k + 1) * (k + 2) / 2 + k;
      emit(idx, lk * jc * cKoornNorm[idx]);
      for (int m = 1; m < n - k; ++m) {
        const int t = k * kBdJac + m;
        const double jn = (cJacP[t] * x - cJacQ[t]) * jc - cJacR[t] * jp;
        jp = jc;
        jc = jn;
        const int nn = m + 1 + k;
        idx = nn * (nn + 1) / 2 + k;
        emit(idx, lk * jc * cKoornNorm[idx]);
      }
    }
  } else {
    const bool leg = iptype == 11;
    double pu[kBdLeg];
    pu[0] = 1.0;
    if (n >= 1) pu[1] = u;
    for (int k = 1; k < n; ++k)
      pu[k + 1] = leg ? cLegA[k] * u * pu[k] - cLegB[k] * pu[k - 1] : 2.0 * u * pu[k] - pu[k - 1];
    double pvm = 0.0, pvc = 1.0;
    for (int i = 0; i <= n; ++i) {
      for (int j = 0; j <= n; ++j) emit(j + (n + 1) * i, pu[j] * pvc);
      const double nx = i == 0 ? v : (leg ? cLegA[i] * v * pvc - cLegB[i] * pvm : 2.0 * v * pvc - pvm);
      pvm = pvc;
      pvc = nx;
    }
  }
}

void fill_basis_constants(cudaStream_t st) {
  static thread_local std::vector<double> host;
  if (host.empty()) {
    host.assign((kBdTriOrder + 1) * (kBdTriOrder + 2) / 2 + 3 * kBdJac * kBdJac + 2 * kBdLeg, 0.0);
    double* norm = host.data();
    double* jp = norm + (kBdTriOrder + 1) * (kBdTriOrder + 2) / 2;
    double* jq = jp + kBdJac * kBdJac;
    double* jr = jq + kBdJac * kBdJac;
    double* la = jr + kBdJac * kBdJac;
    double* lb = la + kBdLeg;
    for (int n = 0; n <= kBdTriOrder; ++n)
      for (int k = 0; k <= n; ++k) norm[n * (n + 1) / 2 + k] = std::sqrt((2.0 * k + 1.0) * (2.0 * n + 2.0));
    for (int k = 0; k < kBdJac; ++k) {
      const double b = 2.0 * k + 1.0;
      for (int m = 1; m < kBdJac; ++m) {
        const double c0 = 2.0 * (m + 1.0) * (m + b + 1.0) * (2.0 * m + b);
        jp[k * kBdJac + m] = (2.0 * m + b + 1.0) * (2.0 * m + b + 2.0) * (2.0 * m + b) / c0;
        jq[k * kBdJac + m] = (2.0 * m + b + 1.0) * b * b / c0;
        jr[k * kBdJac + m] = 2.0 * m * (m + b) * (2.0 * m + b + 2.0) / c0;
      }
    }
    for (int k = 0; k < kBdLeg; ++k) {
      la[k] = (2.0 * k + 1.0) / (k + 1.0);
      lb[k] = k / (k + 1.0);
    }
  }
  const double* h = host.data();
  size_t off = 0;
  auto put = [&](const void* sym, size_t n) {
    cudaMemcpyToSymbolAsync(sym, h + off, n * sizeof(double), 0, cudaMemcpyHostToDevice, st);
    off += n;
  };
  put(cKoornNorm, (kBdTriOrder + 1) * (kBdTriOrder + 2) / 2);
  put(cJacP, kBdJac * kBdJac);
  put(cJacQ, kBdJac * kBdJac);
  put(cJacR, kBdJac * kBdJac);
  put(cLegA, kBdLeg);
  put(cLegB, kBdLeg);
}

}  // namespace
}  // namespace bie
