/*
 * Shared helpers of the FP64 CPU oracle (test infrastructure only; see
 * oracle.c): node tables, patch bases and small dense linear algebra.
 *
 *   koorn_pols           src/tria_routs/koornexps.f90:206-330
 *   legepols, GL nodes   src/common/polytens.f:598-640, legeexps
 *   get_disc_nodes(_wts) src/surface_routs/patch_basis_routs.f90:234
 */
#pragma once
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OVER4PI 0.07957747154594767

/* oracle_far.c */
int64_t oracle_get_far_method(void);
int oracle_farfield(int64_t ns, const double* srcover, const double* chg, const double* dip,
                    const double* zk, double thresh, int64_t ndt, int64_t nt, const double* targs,
                    double* pot);

/* Vioreanu-Rokhlin nodes (u0, v0, u1, v1, ...) and weights per order, set by
 * oracle_set_vr_table from the build's table file. */
extern double* g_vr_uvs[21];
extern double* g_vr_wts[21];
extern int64_t g_vr_np[21];

static inline int64_t npols_of(int64_t iptype, int64_t norder) {
  if (iptype == 1) return (norder + 1) * (norder + 2) / 2;
  return (norder + 1) * (norder + 1);
}

/* koorn_pols, koornexps.f90:206-330 (same recurrences and scaling).  The
 * Jacobi recurrence coefficients an, bn, cn and the normalisations are
 * tabulated once (koorn_init, called when the node tables are set, before
 * any parallel region). */
#define KOORN_NMAX 24
extern double g_koorn_abc[KOORN_NMAX + 1][KOORN_NMAX + 1][3]; /* [k][n] */
extern double g_koorn_sc[KOORN_NMAX + 1][KOORN_NMAX + 1];     /* [n][k] = 1/sc */
extern int g_koorn_ready;

static inline void koorn_init(void) {
  if (g_koorn_ready) return;
  for (int64_t k = 0; k <= KOORN_NMAX; ++k) {
    const double beta = 2 * k + 1;
    for (int64_t n = 1; n <= KOORN_NMAX; ++n) {
      g_koorn_abc[k][n][0] = (2 * n + beta + 1) * (2 * n + beta + 2) / 2 / (n + 1) / (n + beta + 1);
      g_koorn_abc[k][n][1] =
          (-beta * beta) * (2 * n + beta + 1) / 2 / (n + 1) / (n + beta + 1) / (2 * n + beta);
      g_koorn_abc[k][n][2] =
          n * (n + beta) * (2 * n + beta + 2) / (n + 1) / (n + beta + 1) / (2 * n + beta);
    }
  }
  for (int64_t n = 0; n <= KOORN_NMAX; ++n)
    for (int64_t k = 0; k <= n; ++k) g_koorn_sc[n][k] = 1.0 / sqrt(1.0 / (2 * k + 1) / (2 * n + 2));
  g_koorn_ready = 1;
}

static inline void koorn_pols(const double* uv, int64_t nmax, double* pols) {
  double legpols[KOORN_NMAX + 2], jacpols[KOORN_NMAX + 2][KOORN_NMAX + 2];
  const double u = uv[0], v = uv[1];
  const double z = 2 * u + v - 1, y = 1 - v;
  legpols[0] = 1;
  legpols[1] = z;
  for (int64_t k = 1; k <= nmax; ++k)
    legpols[k + 1] = ((2 * k + 1) * z * legpols[k] - k * legpols[k - 1] * y * y) / (k + 1);
  const double x = 1 - 2 * v;
  for (int64_t k = 0; k <= nmax; ++k) {
    const double beta = 2 * k + 1;
    jacpols[0][k] = 1;
    jacpols[1][k] = (-beta + (2 + beta) * x) / 2;
    for (int64_t n = 1; n <= nmax - k - 1; ++n) {
      const double* c = g_koorn_abc[k][n];
      jacpols[n + 1][k] = (c[0] * x + c[1]) * jacpols[n][k] - c[2] * jacpols[n - 1][k];
    }
  }
  int64_t iii = 0;
  for (int64_t n = 0; n <= nmax; ++n)
    for (int64_t k = 0; k <= n; ++k) pols[iii++] = legpols[k] * jacpols[n - k][k] * g_koorn_sc[n][k];
}

/* legepols: P_0..P_n */
static inline void legepols(double x, int64_t n, double* p) {
  p[0] = 1;
  if (n >= 1) p[1] = x;
  for (int64_t k = 1; k < n; ++k) p[k + 1] = ((2 * k + 1) * x * p[k] - k * p[k - 1]) / (k + 1);
}

/* Gauss-Legendre nodes (ascending), Newton on P_n */
static inline void legendre_nodes(int64_t n, double* x) {
  double p[128];
  for (int64_t i = 0; i < n; ++i) {
    double t = cos(M_PI * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      legepols(t, n, p);
      /* derivative from (1-t^2) P_n' = n (P_{n-1} - t P_n) */
      const double dp = n * (p[n - 1] - t * p[n]) / (1 - t * t);
      const double d = p[n] / dp;
      t -= d;
      if (fabs(d) < 1e-16) break;
    }
    x[n - 1 - i] = t;
  }
}

static inline void basis_pols(int64_t iptype, int64_t norder, const double* uv, double* pols) {
  if (iptype == 1) {
    koorn_pols(uv, norder, pols);
    return;
  }
  double px[64], py[64];
  legepols(uv[0], norder, px);
  legepols(uv[1], norder, py);
  const int64_t n = norder + 1;
  for (int64_t i = 0; i < n; ++i)
    for (int64_t j = 0; j < n; ++j) pols[j + n * i] = px[j] * py[i];
}

static inline int disc_nodes(int64_t iptype, int64_t norder, double* uvs) {
  if (iptype == 1) {
    if (!g_vr_uvs[norder]) return 6;
    memcpy(uvs, g_vr_uvs[norder], sizeof(double) * 2 * g_vr_np[norder]);
    return 0;
  }
  if (iptype != 11) return 1;
  const int64_t n = norder + 1;
  double x[64];
  legendre_nodes(n, x);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t j = 0; j < n; ++j) {
      uvs[2 * (j + n * i)] = x[j];
      uvs[2 * (j + n * i) + 1] = x[i];
    }
  return 0;
}

/* dinverse via Gauss-Jordan with partial pivoting; a is overwritten */
static inline int inverse(int64_t n, double* a, double* b) {
  for (int64_t i = 0; i < n * n; ++i) b[i] = 0;
  for (int64_t i = 0; i < n; ++i) b[i * n + i] = 1;
  for (int64_t c = 0; c < n; ++c) {
    int64_t piv = c;
    for (int64_t r = c + 1; r < n; ++r)
      if (fabs(a[r * n + c]) > fabs(a[piv * n + c])) piv = r;
    if (a[piv * n + c] == 0) return 7;
    for (int64_t j = 0; j < n; ++j) {
      double t = a[c * n + j];
      a[c * n + j] = a[piv * n + j];
      a[piv * n + j] = t;
      t = b[c * n + j];
      b[c * n + j] = b[piv * n + j];
      b[piv * n + j] = t;
    }
    const double inv = 1 / a[c * n + c];
    for (int64_t j = 0; j < n; ++j) {
      a[c * n + j] *= inv;
      b[c * n + j] *= inv;
    }
    for (int64_t r = 0; r < n; ++r) {
      if (r == c) continue;
      const double f = a[r * n + c];
      for (int64_t j = 0; j < n; ++j) {
        a[r * n + j] -= f * a[c * n + j];
        b[r * n + j] -= f * b[c * n + j];
      }
    }
  }
  return 0;
}


/* Gauss-Legendre weights at the nodes x (ascending) of order n:
 * w = 2 / ((1 - x^2) P_n'(x)^2). */
static inline void legendre_weights(int64_t n, const double* x, double* w) {
  double p[128];
  for (int64_t i = 0; i < n; ++i) {
    legepols(x[i], n, p);
    const double dp = n * (p[n - 1] - x[i] * p[n]) / (1 - x[i] * x[i]);
    w[i] = 2.0 / ((1 - x[i] * x[i]) * dp * dp);
  }
}

/* Weights of the discretisation nodes (get_disc_nodes_wts): Vioreanu-Rokhlin
 * weights on the simplex (sum 1/2), tensor Gauss-Legendre on [-1,1]^2. */
static inline int disc_wts(int64_t iptype, int64_t norder, double* w) {
  if (iptype == 1) {
    if (!g_vr_wts[norder]) return 6;
    memcpy(w, g_vr_wts[norder], sizeof(double) * g_vr_np[norder]);
    return 0;
  }
  if (iptype != 11) return 1;
  const int64_t n = norder + 1;
  double x[64], wx[64];
  legendre_nodes(n, x);
  legendre_weights(n, x, wx);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t j = 0; j < n; ++j) w[j + n * i] = wx[j] * wx[i];
  return 0;
}

/* umat of get_disc_exps: the inverse of vmat(i, m) = P_m(node i); coefs =
 * umat vals (row-major np x np, umat[m * np + i]). */
static inline int disc_umat(int64_t iptype, int64_t norder, double* umat) {
  const int64_t np = npols_of(iptype, norder);
  double* uvs = (double*)malloc(sizeof(double) * 2 * np);
  double* vmat = (double*)malloc(sizeof(double) * np * np);
  int ier = disc_nodes(iptype, norder, uvs);
  if (!ier) {
    for (int64_t i = 0; i < np; ++i) basis_pols(iptype, norder, uvs + 2 * i, vmat + i * np);
    ier = inverse(np, vmat, umat);
  }
  free(uvs);
  free(vmat);
  return ier;
}
