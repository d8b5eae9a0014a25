/*
 * FP64 CPU far field of the oracle's timed solves (test infrastructure
 * only, like oracle.c): the role of the FMM calls lfmm3d / hfmm3d in
 * lap_comb_dir_eval_addsub (src/lap_wrappers/lap_comb_dir.f90:1094) and
 * helm_comb_dir_eval_addsub (src/helm_wrappers/helm_comb_dir.f:1117),
 *   u(t) = sum_s [ c_s G(t,s) + d_s n_s . grad_s G(t,s) ],  G = e^{ikr}/(4 pi r),
 * over every oversampled source, pairs closer than the self-interaction
 * threshold skipped.  FMM3D (an un-vendored submodule of the reference) is
 * not available; its contract is this sum to a relative accuracy eps.
 *
 * Two methods, chosen with oracle_set_far_method:
 *   1  direct sum, every pair, vectorised (OpenMP SIMD lanes, libmvec sine
 *      and cosine); exact up to rounding;
 *   2  barycentric Lagrange treecode (the cluster-particle method of Wang,
 *      Krasny and Tlupova, restated from the published description): a k-d
 *      tree of the sources split at the median of the longest side; for
 *      every node with more sources than proxies, proxy charges at the
 *      Chebyshev points (second kind) of its bounding box, n + |k| side/2
 *      per side (at most 16; larger nodes get none and are descended),
 *        q_k = sum_s c_s L_k(s) + d_s n_s . grad L_k(s)
 *      (L_k the tensor Lagrange basis in barycentric form), so the cluster
 *      acts on a target as sum_k q_k G(t, s_k); a target takes a node's
 *      proxies when r_node < theta |t - c_node|, otherwise descends, and
 *      leaves are summed directly.  O(N log N) work for fixed (theta, n).
 * oracle.c's scalar direct sum (method 0) stays the parity oracle.
 */
#define _GNU_SOURCE
#include <omp.h>

#include "oracle_common.h"

static int64_t g_far_method = 0;
static double g_theta = 0.5;
static int64_t g_ncheb = 9;
static int64_t g_leaf = 256;

/* 0: oracle.c's scalar direct sum; 1: vectorised direct sum; 2: treecode
 * (theta, Chebyshev points per side, sources per leaf; <= 0 keeps the
 * current value). */
int oracle_set_far_method(int64_t method, double theta, int64_t ncheb, int64_t leaf) {
  if (method < 0 || method > 2) return 1;
  g_far_method = method;
  if (theta > 0) g_theta = theta;
  if (ncheb > 1) g_ncheb = ncheb > 16 ? 16 : ncheb;
  if (leaf > 0) g_leaf = leaf;
  return 0;
}

int64_t oracle_get_far_method(void) { return g_far_method; }

/* sources in SoA, tree order */
typedef struct {
  double *x, *y, *z, *nx, *ny, *nz, *cr, *ci, *dr, *di;
} Src;

/* sum over sources [b, e) at one target; Laplace when kr == ki == 0 */
static inline void leaf_sum(const Src* S, int64_t b, int64_t e, double tx, double ty, double tz,
                            double kr, double ki, double th2, double* ur, double* ui) {
  double ar = 0, ai = 0;
  if (ki == 0) {
#pragma omp simd reduction(+ : ar, ai)
    for (int64_t s = b; s < e; ++s) {
      const double dx = tx - S->x[s], dy = ty - S->y[s], dz = tz - S->z[s];
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double m = r2 < th2 ? 0.0 : 1.0;
      const double r2s = r2 < th2 ? 1.0 : r2;
      const double rinv = 1.0 / sqrt(r2s);
      const double r = r2s * rinv;
      const double dn = (dx * S->nx[s] + dy * S->ny[s] + dz * S->nz[s]) * rinv * rinv;
      const double cs = cos(kr * r), sn = sin(kr * r);
      /* c + d dn (1 - i k r) */
      const double xr = S->cr[s] + dn * (S->dr[s] + S->di[s] * kr * r);
      const double xi = S->ci[s] + dn * (S->di[s] - S->dr[s] * kr * r);
      ar += m * rinv * (xr * cs - xi * sn);
      ai += m * rinv * (xi * cs + xr * sn);
    }
  } else {
#pragma omp simd reduction(+ : ar, ai)
    for (int64_t s = b; s < e; ++s) {
      const double dx = tx - S->x[s], dy = ty - S->y[s], dz = tz - S->z[s];
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double m = r2 < th2 ? 0.0 : 1.0;
      const double r2s = r2 < th2 ? 1.0 : r2;
      const double rinv = 1.0 / sqrt(r2s);
      const double r = r2s * rinv;
      const double dn = (dx * S->nx[s] + dy * S->ny[s] + dz * S->nz[s]) * rinv * rinv;
      const double ea = exp(-ki * r) * rinv * m;
      const double cs = cos(kr * r), sn = sin(kr * r);
      /* c + d dn (1 - i k r) with k = kr + i ki: 1 - ikr = (1 + ki r) - i kr r */
      const double wr = dn * (1.0 + ki * r), wi = -dn * kr * r;
      const double xr = S->cr[s] + S->dr[s] * wr - S->di[s] * wi;
      const double xi = S->ci[s] + S->dr[s] * wi + S->di[s] * wr;
      ar += ea * (xr * cs - xi * sn);
      ai += ea * (xi * cs + xr * sn);
    }
  }
  *ur += ar;
  *ui += ai;
}

/* charge-only sum over the proxies of a node */
static inline void proxy_sum(const double* px, const double* py, const double* pz, const double* qr,
                             const double* qi, int64_t n, double tx, double ty, double tz,
                             double kr, double ki, double* ur, double* ui) {
  double ar = 0, ai = 0;
#pragma omp simd reduction(+ : ar, ai)
  for (int64_t k = 0; k < n; ++k) {
    const double dx = tx - px[k], dy = ty - py[k], dz = tz - pz[k];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double rinv = 1.0 / sqrt(r2);
    const double r = r2 * rinv;
    const double ea = (ki == 0 ? 1.0 : exp(-ki * r)) * rinv;
    const double cs = cos(kr * r), sn = sin(kr * r);
    ar += ea * (qr[k] * cs - qi[k] * sn);
    ai += ea * (qi[k] * cs + qr[k] * sn);
  }
  *ur += ar;
  *ui += ai;
}

typedef struct {
  int64_t b, e, c0, c1, prox; /* source range, children (-1: leaf), proxy offset (-1: none) */
  double c[3], r, lo[3], hi[3];
  int64_t n; /* Chebyshev points per side of the proxy grid */
} Node;

static void node_box(Node* nd, const double* xyz, const int64_t* idx) {
  for (int k = 0; k < 3; ++k) {
    nd->lo[k] = 1e300;
    nd->hi[k] = -1e300;
  }
  for (int64_t i = nd->b; i < nd->e; ++i)
    for (int k = 0; k < 3; ++k) {
      const double v = xyz[12 * idx[i] + k];
      if (v < nd->lo[k]) nd->lo[k] = v;
      if (v > nd->hi[k]) nd->hi[k] = v;
    }
  /* centre and half-diagonal of the box: the proxy grid fills the box, so
   * the acceptance test measures the box, not only its sources */
  double r2 = 0;
  for (int k = 0; k < 3; ++k) {
    nd->c[k] = 0.5 * (nd->lo[k] + nd->hi[k]);
    r2 += 0.25 * (nd->hi[k] - nd->lo[k]) * (nd->hi[k] - nd->lo[k]);
  }
  nd->r = sqrt(r2);
}

/* reorder idx[b, e) so that the m-th smallest coordinate is at b + m
 * (quickselect) */
static void select_k(int64_t* idx, int64_t b, int64_t e, int64_t m, const double* xyz, int dim) {
  int64_t lo = b, hi = e - 1, k = b + m;
  while (lo < hi) {
    const double piv = xyz[12 * idx[(lo + hi) / 2] + dim];
    int64_t i = lo, j = hi;
    while (i <= j) {
      while (xyz[12 * idx[i] + dim] < piv) ++i;
      while (xyz[12 * idx[j] + dim] > piv) --j;
      if (i <= j) {
        const int64_t t = idx[i];
        idx[i] = idx[j];
        idx[j] = t;
        ++i;
        --j;
      }
    }
    if (k <= j)
      hi = j;
    else if (k >= i)
      lo = i;
    else
      break;
  }
}

/* barycentric Lagrange values and derivatives at x for Chebyshev points
 * xs[0..n) with weights w.  Off the nodes, l_i' = l_i (s2/s - 1/(x - x_i))
 * (s = sum w_i/(x - x_i), s2 = sum w_i/(x - x_i)^2) loses every digit for
 * the node nearest x when x is within rounding of it (a box's extreme
 * sources sit on its end nodes), so that one is taken as minus the sum of
 * the others (the l_i sum to one). */
static void lagrange1(int64_t n, const double* xs, const double* w, double x, double* l,
                      double* dl) {
  int64_t jn = 0;
  for (int64_t j = 1; j < n; ++j)
    if (fabs(x - xs[j]) < fabs(x - xs[jn])) jn = j;
  if (x == xs[jn]) {
    for (int64_t i = 0; i < n; ++i) l[i] = i == jn ? 1.0 : 0.0;
    double djj = 0;
    for (int64_t i = 0; i < n; ++i) {
      if (i == jn) continue;
      dl[i] = (w[i] / w[jn]) / (xs[jn] - xs[i]);
      djj -= dl[i];
    }
    dl[jn] = djj;
    return;
  }
  double s = 0, s2 = 0;
  for (int64_t i = 0; i < n; ++i) {
    const double t = w[i] / (x - xs[i]);
    s += t;
    s2 += t / (x - xs[i]);
  }
  double dsum = 0;
  for (int64_t i = 0; i < n; ++i) {
    const double t = w[i] / (x - xs[i]);
    l[i] = t / s;
    if (i == jn) continue;
    dl[i] = l[i] * (s2 / s - 1.0 / (x - xs[i]));
    dsum += dl[i];
  }
  dl[jn] = -dsum;
}

/* the sum at nt targets (ndt values each, xyz first): pot complex
 * interleaved.  c, d: complex interleaved source strengths (1/(4 pi)
 * included by the caller); srcover 12 x ns; zk = (re, im). */
int oracle_farfield(int64_t ns, const double* srcover, const double* chg, const double* dip,
                    const double* zk, double thresh, int64_t ndt, int64_t nt, const double* targs,
                    double* pot) {
  const double kr = zk[0], ki = zk[1], th2 = thresh * thresh;
  const int tree = g_far_method == 2;
  int64_t* idx = malloc(sizeof(int64_t) * (ns > 0 ? ns : 1));
  for (int64_t i = 0; i < ns; ++i) idx[i] = i;
  /* tree (a single leaf for the direct method) */
  int64_t cap = 64, nn = 1;
  Node* nodes = malloc(sizeof(Node) * cap);
  nodes[0].b = 0;
  nodes[0].e = ns;
  nodes[0].c0 = nodes[0].c1 = -1;
  nodes[0].prox = -1;
  const int64_t n = g_ncheb;
  if (tree) {
    for (int64_t q = 0; q < nn; ++q) {
      node_box(&nodes[q], srcover, idx);
      const int64_t cnt = nodes[q].e - nodes[q].b;
      if (cnt <= g_leaf) continue;
      int dim = 0;
      for (int k = 1; k < 3; ++k)
        if (nodes[q].hi[k] - nodes[q].lo[k] > nodes[q].hi[dim] - nodes[q].lo[dim]) dim = k;
      const int64_t half = cnt / 2;
      select_k(idx, nodes[q].b, nodes[q].e, half, srcover, dim);
      if (nn + 2 > cap) {
        cap *= 2;
        nodes = realloc(nodes, sizeof(Node) * cap);
      }
      const int64_t b = nodes[q].b, e = nodes[q].e;
      nodes[q].c0 = nn;
      nodes[q].c1 = nn + 1;
      nodes[nn] = (Node){b, b + half, -1, -1, -1, {0, 0, 0}, 0, {0, 0, 0}, {0, 0, 0}, 0};
      nodes[nn + 1] = (Node){b + half, e, -1, -1, -1, {0, 0, 0}, 0, {0, 0, 0}, {0, 0, 0}, 0};
      nn += 2;
    }
  }
  Src S;
  double* buf = malloc(sizeof(double) * 10 * (ns > 0 ? ns : 1));
  double** f[10] = {&S.x, &S.y, &S.z, &S.nx, &S.ny, &S.nz, &S.cr, &S.ci, &S.dr, &S.di};
  for (int k = 0; k < 10; ++k) *f[k] = buf + k * ns;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < ns; ++i) {
    const double* s = srcover + 12 * idx[i];
    S.x[i] = s[0];
    S.y[i] = s[1];
    S.z[i] = s[2];
    S.nx[i] = s[9];
    S.ny[i] = s[10];
    S.nz[i] = s[11];
    S.cr[i] = chg[2 * idx[i]];
    S.ci[i] = chg[2 * idx[i] + 1];
    S.dr[i] = dip[2 * idx[i]];
    S.di[i] = dip[2 * idx[i] + 1];
  }
  /* proxies: n + |k| side / 2 points per side (e^{ikr} resolved across the
   * box as well as 1/r), for nodes with more sources than proxies and at
   * most 16 points per side */
  int64_t nprox = 0;
  if (tree)
    for (int64_t q = 0; q < nn; ++q) {
      double side = 0;
      for (int k = 0; k < 3; ++k)
        if (nodes[q].hi[k] - nodes[q].lo[k] > side) side = nodes[q].hi[k] - nodes[q].lo[k];
      const int64_t nq = n + (int64_t)ceil(sqrt(kr * kr + ki * ki) * side / 2);
      if (nq <= 16 && nodes[q].e - nodes[q].b > nq * nq * nq) {
        nodes[q].n = nq;
        nodes[q].prox = nprox;
        nprox += nq * nq * nq;
      }
    }
  double* P = malloc(sizeof(double) * 5 * (nprox > 0 ? nprox : 1)); /* x y z qr qi */
  if (nprox) {
    const double pi = 4 * atan(1.0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t q = 0; q < nn; ++q) {
      if (nodes[q].prox < 0) continue;
      Node* nd = &nodes[q];
      const int64_t n = nd->n;
      double cx[16], cw[16];
      for (int64_t j = 0; j < n; ++j) {
        cx[j] = cos(pi * j / (n - 1));
        cw[j] = (j % 2 ? -1.0 : 1.0) * ((j == 0 || j == n - 1) ? 0.5 : 1.0);
      }
      double xs[3][16];
      for (int k = 0; k < 3; ++k) {
        double h = 0.5 * (nd->hi[k] - nd->lo[k]);
        const double mid = 0.5 * (nd->hi[k] + nd->lo[k]);
        if (h < 1e-12 * (nd->r + 1e-300)) h = 1e-12 * (nd->r + 1e-300);
        for (int64_t j = 0; j < n; ++j) xs[k][j] = mid + h * cx[j];
      }
      double* px = P + nd->prox;
      double* py = P + nprox + nd->prox;
      double* pz = P + 2 * nprox + nd->prox;
      double* qr = P + 3 * nprox + nd->prox;
      double* qi = P + 4 * nprox + nd->prox;
      for (int64_t l = 0; l < n; ++l)
        for (int64_t j = 0; j < n; ++j)
          for (int64_t i = 0; i < n; ++i) {
            const int64_t k = i + n * (j + n * l);
            px[k] = xs[0][i];
            py[k] = xs[1][j];
            pz[k] = xs[2][l];
            qr[k] = 0;
            qi[k] = 0;
          }
      double L[3][16], D[3][16];
      const int64_t n3 = n * n * n;
      (void)n3;
      for (int64_t s = nd->b; s < nd->e; ++s) {
        lagrange1(n, xs[0], cw, S.x[s], L[0], D[0]);
        lagrange1(n, xs[1], cw, S.y[s], L[1], D[1]);
        lagrange1(n, xs[2], cw, S.z[s], L[2], D[2]);
        const double cr = S.cr[s], ci = S.ci[s], dr = S.dr[s], di = S.di[s];
        const double nx = S.nx[s], ny = S.ny[s], nz = S.nz[s];
        for (int64_t l = 0; l < n; ++l)
          for (int64_t j = 0; j < n; ++j) {
            const double a = L[1][j] * L[2][l];
            const double bx = nx * a;
            const double byz = ny * D[1][j] * L[2][l] + nz * L[1][j] * D[2][l];
            double* qrr = qr + n * (j + n * l);
            double* qii = qi + n * (j + n * l);
#pragma omp simd
            for (int64_t i = 0; i < n; ++i) {
              const double v = L[0][i] * a;                   /* L_k(s) */
              const double g = D[0][i] * bx + L[0][i] * byz;  /* n . grad L_k(s) */
              qrr[i] += cr * v + dr * g;
              qii[i] += ci * v + di * g;
            }
          }
      }
    }
  }
  const double theta = g_theta;
#pragma omp parallel
  {
    int64_t* stk = malloc(sizeof(int64_t) * (nn + 8));
#pragma omp for schedule(dynamic, 16)
    for (int64_t t = 0; t < nt; ++t) {
      const double tx = targs[ndt * t], ty = targs[ndt * t + 1], tz = targs[ndt * t + 2];
      double ur = 0, ui = 0;
      if (!tree) {
        leaf_sum(&S, 0, ns, tx, ty, tz, kr, ki, th2, &ur, &ui);
      } else {
        int64_t top = 0;
        stk[top++] = 0;
        while (top > 0) {
          const Node* nd = &nodes[stk[--top]];
          const double dx = tx - nd->c[0], dy = ty - nd->c[1], dz = tz - nd->c[2];
          const double dist = sqrt(dx * dx + dy * dy + dz * dz);
          if (nd->prox >= 0 && nd->r < theta * dist) {
            proxy_sum(P + nd->prox, P + nprox + nd->prox, P + 2 * nprox + nd->prox,
                      P + 3 * nprox + nd->prox, P + 4 * nprox + nd->prox, nd->n * nd->n * nd->n,
                      tx, ty, tz, kr, ki, &ur, &ui);
          } else if (nd->c0 < 0) {
            leaf_sum(&S, nd->b, nd->e, tx, ty, tz, kr, ki, th2, &ur, &ui);
          } else {
            stk[top++] = nd->c0;
            stk[top++] = nd->c1;
          }
        }
      }
      pot[2 * t] = ur;
      pot[2 * t + 1] = ui;
    }
    free(stk);
  }
  free(idx);
  free(nodes);
  free(buf);
  free(P);
  return 0;
}
