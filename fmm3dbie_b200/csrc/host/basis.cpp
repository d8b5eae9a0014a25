// Patch bases and discretisation nodes; see basis.h for the conventions.
#include "basis.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

namespace bie {

namespace {
struct VRTable {
  bool loaded = false;
  std::vector<double> uvs[kMaxOrder + 1];
  std::vector<double> wts[kMaxOrder + 1];
};
VRTable g_vr;
std::mutex g_vr_mu;
}  // namespace

int npols_of(int iptype, int norder) {
  if (norder < 0) return 0;
  if (iptype == 1) return (norder + 1) * (norder + 2) / 2;
  if (iptype == 11 || iptype == 12) return (norder + 1) * (norder + 1);
  return 0;
}

bool valid_patch(int iptype, int norder) {
  if (iptype == 1) return norder >= 0 && norder <= kMaxOrder;
  if (iptype == 11 || iptype == 12) return norder >= 0 && norder <= 40;
  return false;
}

int load_vr_tables(const char* path) {
  std::lock_guard<std::mutex> lk(g_vr_mu);
  if (g_vr.loaded) return 0;
  FILE* f = std::fopen(path, "rb");
  if (!f) return 1;
  char magic[8];
  int nmax = 0;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "BIEVR001", 8) == 0 &&
            std::fread(&nmax, 4, 1, f) == 1 && nmax >= kMaxOrder;
  for (int n = 0; ok && n <= kMaxOrder; ++n) {
    int np = 0;
    ok = std::fread(&np, 4, 1, f) == 1 && np == npols_of(1, n);
    if (!ok) break;
    g_vr.uvs[n].resize(2 * np);
    g_vr.wts[n].resize(np);
    ok = std::fread(g_vr.uvs[n].data(), 8, 2 * np, f) == size_t(2 * np) &&
         std::fread(g_vr.wts[n].data(), 8, np, f) == size_t(np);
  }
  std::fclose(f);
  g_vr.loaded = ok;
  return ok ? 0 : 2;
}

bool vr_tables_loaded() { return g_vr.loaded; }

// Koornwinder polynomials on the simplex, written from the definition
//   K_{n,k}(u,v) = P_{n-k}^{(0,2k+1)}(1-2v) (1-v)^k P_k((2u+v-1)/(1-v))
// normalised to unit L2 norm on the simplex (koornexps.f90:206-330).
void koorn_pols(double u, double v, int nmax, double* pols) {
  double leg[kMaxOrder + 2];
  double jac[kMaxOrder + 2];
  const double z = 2.0 * u + v - 1.0;
  const double y = 1.0 - v;
  // Scaled Legendre: leg[k] = y^k P_k(z/y), via the homogenised recurrence.
  leg[0] = 1.0;
  if (nmax >= 1) leg[1] = z;
  for (int k = 1; k < nmax; ++k)
    leg[k + 1] = ((2.0 * k + 1.0) * z * leg[k] - k * y * y * leg[k - 1]) / (k + 1.0);
  const double x = 1.0 - 2.0 * v;
  // Reorder the output loop: for each k, generate Jacobi P_m^{(0,2k+1)}(x)
  // for m = 0..nmax-k, and scatter into (n = m + k, k).
  for (int k = 0; k <= nmax; ++k) {
    const double b = 2.0 * k + 1.0;  // beta, alpha = 0
    jac[0] = 1.0;
    if (nmax - k >= 1) jac[1] = 0.5 * ((b + 2.0) * x - b);
    for (int m = 1; m < nmax - k; ++m) {
      // 2(m+1)(m+b+1)(2m+b) P_{m+1} =
      //   (2m+b+1)[(2m+b+2)(2m+b) x - b^2] P_m - 2 m (m+b)(2m+b+2) P_{m-1}
      const double c0 = 2.0 * (m + 1.0) * (m + b + 1.0) * (2.0 * m + b);
      const double c1 = (2.0 * m + b + 1.0) * ((2.0 * m + b + 2.0) * (2.0 * m + b) * x - b * b);
      const double c2 = 2.0 * m * (m + b) * (2.0 * m + b + 2.0);
      jac[m + 1] = (c1 * jac[m] - c2 * jac[m - 1]) / c0;
    }
    for (int m = 0; m <= nmax - k; ++m) {
      const int n = m + k;
      const int idx = n * (n + 1) / 2 + k;
      // ||K_{n,k}||^2 on the simplex = 1 / ((2k+1)(2n+2))
      pols[idx] = leg[k] * jac[m] * std::sqrt((2.0 * k + 1.0) * (2.0 * n + 2.0));
    }
  }
}

void legendre_pols(double x, int n, double* p, double* dp) {
  p[0] = 1.0;
  if (dp) dp[0] = 0.0;
  if (n < 1) return;
  p[1] = x;
  if (dp) dp[1] = 1.0;
  for (int k = 1; k < n; ++k) {
    p[k + 1] = ((2.0 * k + 1.0) * x * p[k] - k * p[k - 1]) / (k + 1.0);
    if (dp) dp[k + 1] = dp[k - 1] + (2.0 * k + 1.0) * p[k];
  }
}

void chebyshev_pols(double x, int n, double* p, double* dp) {
  p[0] = 1.0;
  if (dp) dp[0] = 0.0;
  if (n < 1) return;
  p[1] = x;
  if (dp) dp[1] = 1.0;
  for (int k = 1; k < n; ++k) {
    p[k + 1] = 2.0 * x * p[k] - p[k - 1];
    if (dp) dp[k + 1] = 2.0 * p[k] + 2.0 * x * dp[k] - dp[k - 1];
  }
}

void gauss_legendre(int n, double* x, double* w) {
  std::vector<double> p(n + 1), dp(n + 1);
  for (int i = 0; i < n; ++i) {
    // Newton from the classical asymptotic guess; node i counted from +1.
    double t = std::cos(M_PI * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      legendre_pols(t, n, p.data(), dp.data());
      const double dt = p[n] / dp[n];
      t -= dt;
      if (std::fabs(dt) < 1e-16) break;
    }
    legendre_pols(t, n, p.data(), dp.data());
    x[n - 1 - i] = t;
    w[n - 1 - i] = 2.0 / ((1.0 - t * t) * dp[n] * dp[n]);
  }
  // Symmetrise to remove round-off asymmetry.
  for (int i = 0; i < n / 2; ++i) {
    const double a = 0.5 * (x[n - 1 - i] - x[i]);
    const double ww = 0.5 * (w[i] + w[n - 1 - i]);
    x[i] = -a;
    x[n - 1 - i] = a;
    w[i] = w[n - 1 - i] = ww;
  }
  if (n % 2 == 1) x[n / 2] = 0.0;
}

void chebyshev_nodes(int n, double* x, double* w) {
  for (int i = 1; i <= n; ++i) x[n - i] = std::cos((2.0 * i - 1.0) * M_PI / (2.0 * n));
  // Interpolatory weights: sum_j w_j T_k(x_j) = int_{-1}^1 T_k.
  std::vector<double> a(n * n), ainv(n * n), mom(n);
  std::vector<double> t(n);
  for (int j = 0; j < n; ++j) {
    chebyshev_pols(x[j], n - 1, t.data());
    for (int k = 0; k < n; ++k) a[k * n + j] = t[k];
  }
  for (int k = 0; k < n; ++k) mom[k] = (k % 2 == 1) ? 0.0 : 2.0 / (1.0 - double(k) * k);
  invert(n, a.data(), ainv.data());
  for (int j = 0; j < n; ++j) {
    double s = 0;
    for (int k = 0; k < n; ++k) s += ainv[j * n + k] * mom[k];
    w[j] = s;
  }
}

namespace {
void tensor_pols(int iptype, int norder, double u, double v, double* pols, double* ders) {
  const int n = norder + 1;
  double pu[64], pv[64], dpu[64], dpv[64];
  if (iptype == 11) {
    legendre_pols(u, norder, pu, dpu);
    legendre_pols(v, norder, pv, dpv);
  } else {
    chebyshev_pols(u, norder, pu, dpu);
    chebyshev_pols(v, norder, pv, dpv);
  }
  // "full" ordering: index = j + n*i, px(j)*py(i) (polytens.f:598-640)
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      pols[j + n * i] = pu[j] * pv[i];
      if (ders) {
        ders[2 * (j + n * i)] = dpu[j] * pv[i];
        ders[2 * (j + n * i) + 1] = pu[j] * dpv[i];
      }
    }
}
}  // namespace

void basis_pols(int iptype, int norder, double u, double v, double* pols) {
  if (iptype == 1)
    koorn_pols(u, v, norder, pols);
  else
    tensor_pols(iptype, norder, u, v, pols, nullptr);
}

int disc_nodes(int iptype, int norder, double* uvs) {
  if (!valid_patch(iptype, norder)) return 1;
  if (iptype == 1) {
    if (!g_vr.loaded) return 6;
    std::memcpy(uvs, g_vr.uvs[norder].data(), sizeof(double) * 2 * npols_of(1, norder));
    return 0;
  }
  const int n = norder + 1;
  std::vector<double> x(n), w(n);
  if (iptype == 11)
    gauss_legendre(n, x.data(), w.data());
  else
    chebyshev_nodes(n, x.data(), w.data());
  // x(1,ipt) = x1d(j), x(2,ipt) = x1d(i), j fastest (polytens.f:322-360)
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      uvs[2 * (j + n * i)] = x[j];
      uvs[2 * (j + n * i) + 1] = x[i];
    }
  return 0;
}

int disc_wts(int iptype, int norder, double* wts) {
  if (!valid_patch(iptype, norder)) return 1;
  if (iptype == 1) {
    if (!g_vr.loaded) return 6;
    std::memcpy(wts, g_vr.wts[norder].data(), sizeof(double) * npols_of(1, norder));
    return 0;
  }
  const int n = norder + 1;
  std::vector<double> x(n), w(n);
  if (iptype == 11)
    gauss_legendre(n, x.data(), w.data());
  else
    chebyshev_nodes(n, x.data(), w.data());
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) wts[j + n * i] = w[i] * w[j];
  return 0;
}

int disc_exps(int iptype, int norder, double* uvs, double* umat, double* vmat, double* wts) {
  int ier = disc_nodes(iptype, norder, uvs);
  if (ier) return ier;
  ier = disc_wts(iptype, norder, wts);
  if (ier) return ier;
  const int np = npols_of(iptype, norder);
  std::vector<double> p(np);
  for (int i = 0; i < np; ++i) {
    basis_pols(iptype, norder, uvs[2 * i], uvs[2 * i + 1], p.data());
    for (int j = 0; j < np; ++j) vmat[i * np + j] = p[j];
  }
  return invert(np, vmat, umat) ? 7 : 0;
}

int boundary_vertices(int iptype, double* uv) {
  if (iptype == 1) {
    const double c[6] = {0, 0, 1, 0, 0, 1};
    std::memcpy(uv, c, sizeof c);
    return 3;
  }
  const double c[8] = {-1, -1, 1, -1, 1, 1, -1, 1};
  std::memcpy(uv, c, sizeof c);
  return 4;
}

int clashing_indices(int iptype, int norder, int nfar, int* iclash, int* iclashfar) {
  // A node of order norder coincides with a node of order nfar when both
  // sets contain the centroid (VR orders divisible by 3) or, for tensor
  // grids, when 1-D nodes coincide (patch_basis_routs.f90:518-572).
  if (iptype == 1) {
    // Only the centroid is shared, and only when both orders are
    // multiples of 3; it is node 76 (1-based) at order 15, 106 at order 18
    // and node 1 otherwise.
    if (norder % 3 != 0 || nfar % 3 != 0) return 0;
    auto centroid = [](int n) { return n == 15 ? 75 : (n == 18 ? 105 : 0); };
    iclash[0] = centroid(norder);
    iclashfar[0] = centroid(nfar);
    return 1;
  }
  const int np = npols_of(iptype, norder), nf = npols_of(iptype, nfar);
  std::vector<double> a(2 * np), b(2 * nf);
  if (disc_nodes(iptype, norder, a.data()) || disc_nodes(iptype, nfar, b.data())) return 0;
  int nclash = 0;
  const double tol2 = 1e-24;
  for (int i = 0; i < np; ++i)
    for (int j = 0; j < nf; ++j) {
      const double du = a[2 * i] - b[2 * j], dv = a[2 * i + 1] - b[2 * j + 1];
      if (du * du + dv * dv <= tol2) {
        iclash[nclash] = i;
        iclashfar[nclash] = j;
        ++nclash;
      }
    }
  return nclash;
}

int invert(int n, const double* a, double* ainv) {
  std::vector<double> m(a, a + size_t(n) * n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) ainv[i * n + j] = (i == j) ? 1.0 : 0.0;
  for (int c = 0; c < n; ++c) {
    int piv = c;
    double best = std::fabs(m[c * n + c]);
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(m[r * n + c]) > best) {
        best = std::fabs(m[r * n + c]);
        piv = r;
      }
    if (best == 0.0) return 1;
    if (piv != c)
      for (int j = 0; j < n; ++j) {
        std::swap(m[c * n + j], m[piv * n + j]);
        std::swap(ainv[c * n + j], ainv[piv * n + j]);
      }
    const double inv = 1.0 / m[c * n + c];
    for (int j = 0; j < n; ++j) {
      m[c * n + j] *= inv;
      ainv[c * n + j] *= inv;
    }
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const double f = m[r * n + c];
      if (f == 0.0) continue;
      for (int j = 0; j < n; ++j) {
        m[r * n + j] -= f * m[c * n + j];
        ainv[r * n + j] -= f * ainv[c * n + j];
      }
    }
  }
  return 0;
}

int interp_matrix(int iptype, int norder, int nfar, std::vector<double>& imat) {
  const int np = npols_of(iptype, norder), nf = npols_of(iptype, nfar);
  std::vector<double> uvs(2 * np), umat(np * np), vmat(np * np), wts(np), uvf(2 * nf), p(np);
  int ier = disc_exps(iptype, norder, uvs.data(), umat.data(), vmat.data(), wts.data());
  if (ier) return ier;
  ier = disc_nodes(iptype, nfar, uvf.data());
  if (ier) return ier;
  imat.assign(size_t(nf) * np, 0.0);
  for (int i = 0; i < nf; ++i) {
    basis_pols(iptype, norder, uvf[2 * i], uvf[2 * i + 1], p.data());
    for (int j = 0; j < np; ++j) {
      double s = 0;
      for (int l = 0; l < np; ++l) s += p[l] * umat[l * np + j];
      imat[i * np + j] = s;
    }
  }
  return 0;
}

}  // namespace bie
