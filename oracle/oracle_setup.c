/*
 * FP64 CPU oracle: surfaces and the setup of the combined-field solvers.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, like oracle.c): tests/, smoke() and
 * bench.py's CPU legs load it; the product never links or calls it.  It
 * shares no code with the product: everything the oracle's matvec and GMRES
 * consume (surface, near list, far orders, oversampled geometry, weights and
 * near quadrature) can be made here, so a parity test compares two
 * independent pipelines.
 *
 * Restated reference routines (fmm3dbie):
 *   xtri_rsolid (icosahedron)   src/surface_routs/xtri_parameterizations.f90:1419-1830
 *   xtri_platonic, refine4_flat src/surface_routs/xtri_parameterizations.f90:1335-1413,1864-1949
 *   xtri_ellipsoid_eval         src/surface_routs/xtri_parameterizations.f90:247-334
 *   getgeominfo                 src/surface_routs/surf_routs.f90:3200-3277
 *   get_qwts                    src/surface_routs/surf_routs.f90:1598
 *   get_centroid_rads(_guru)    src/surface_routs/surf_routs.f90:195-300
 *   oversample_geom             src/surface_routs/surf_routs.f90:304-450
 *   get_clashing_indices        src/surface_routs/patch_basis_routs.f90:518-575
 *   get_rfacs                   src/quadratures/near_field_routs.f:826-872
 *   findnearslow                src/quadratures/near_field_routs.f:30-80 (brute force)
 *   get_iquad_rsc               src/quadratures/near_field_routs.f:765-820
 *   get_far_order(_guru)        src/quadratures/far_field_routs.f90:10-425
 *   hkrand / LAPACK dlaran      src/common/hkrand.f:3-19 (48-bit LCG, published
 *                               LAPACK definition)
 *   h3d_slp, h3d_dlp            src/kernels/helm_kernels.f90:8-62
 *
 * Near quadrature (getnearquad_{lap,helm}_comb_dir[_eval]): the reference's
 * generalized Gaussian self rules cannot be rebuilt (their data file is
 * missing from the checkout), so the oracle computes the same integrals,
 *   wnear(l) = sum_m umat(m,l) int_patch K(t, X(y)) P_m(y) |J(y)| dy,
 * with rules of its own, unlike the product's (collapsed Gauss rules, Duffy
 * and sinh maps):
 *   * target on the patch (ipatch_id): the parameter domain is split at the
 *     target into triangles; each is integrated in polar coordinates about
 *     the target (the rho Jacobian cancels the 1/r singularity), 20-point
 *     Gauss-Legendre in rho on [0, R(theta)] and adaptive 20-point
 *     Gauss-Legendre panels in theta (halving until a panel agrees with its
 *     halves);
 *   * other targets: 4-way adaptive subdivision of the parameter triangle
 *     (the reference's adaptive scheme, adap-quads.f:935-1253) with the
 *     degree-22 Vioreanu-Rokhlin rule of order 12 on every triangle.
 * Both stop at an absolute tolerance of 1e-9 (|alpha| + |beta|/R) A/(4 pi R)
 * (A, R: area and radius of the patch; oracle_set_nq_tol changes the 1e-9):
 * the accepted sums are those of the finer level, about 1e-11 of the largest
 * weight on the test surfaces (1e-12 gives the same weights to 1e-11), far
 * below the eps of any configuration, so the oracle's weights serve as the
 * exact values.
 */
#define _GNU_SOURCE /* sincos */
#include <stdio.h>

#include "oracle_common.h"

/* ---------------- surfaces ------------------------------------------------ */

/* xtri_rsolid itype 4: a pentagon ring at height x, the apex (0,0,d+x), and
 * their point reflections; scaled to unit circumradius. */
static void icosahedron(double v[12][3], int f[20][3]) {
  const double pi = 4 * atan(1.0);
  for (int i = 1; i <= 5; ++i) {
    v[i - 1][0] = cos(2 * pi * i / 5.0);
    v[i - 1][1] = sin(2 * pi * i / 5.0);
    v[i - 1][2] = 0;
  }
  const double s = sqrt((v[1][0] - v[0][0]) * (v[1][0] - v[0][0]) +
                        (v[1][1] - v[0][1]) * (v[1][1] - v[0][1]));
  const double d = sqrt(s * s - 1);
  v[5][0] = 0;
  v[5][1] = 0;
  v[5][2] = d;
  const double x = (1 - d * d) / (2 * d);
  for (int i = 0; i < 6; ++i) v[i][2] += x;
  for (int i = 0; i < 6; ++i)
    for (int k = 0; k < 3; ++k) v[i + 6][k] = -v[i][k];
  static const int F[20][3] = {{1, 2, 6},  {2, 3, 6},   {3, 4, 6},  {4, 5, 6},   {5, 1, 6},
                               {8, 7, 12}, {9, 8, 12},  {10, 9, 12}, {11, 10, 12}, {7, 11, 12},
                               {2, 1, 10}, {3, 2, 11},  {4, 3, 7},  {5, 4, 8},   {1, 5, 9},
                               {8, 9, 5},  {9, 10, 1},  {10, 11, 2}, {11, 7, 3},  {7, 8, 4}};
  for (int i = 0; i < 20; ++i)
    for (int k = 0; k < 3; ++k) f[i][k] = F[i][k] - 1;
  const double r = sqrt(v[0][0] * v[0][0] + v[0][1] * v[0][1] + v[0][2] * v[0][2]);
  for (int i = 0; i < 12; ++i)
    for (int k = 0; k < 3; ++k) v[i][k] /= r;
}

int64_t oracle_icosa_npatches(int64_t nref) {
  int64_t n = 20;
  for (int64_t i = 0; i < nref; ++i) n *= 4;
  return n;
}

/* srccoefs = umat * srcvals(1:9) per patch (getgeominfo) */
static int vals_to_coefs(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                         const int64_t* iptype, const double* srcvals, double* srccoefs) {
  int err = 0;
#pragma omp parallel for schedule(dynamic, 8)
  for (int64_t p = 0; p < npatches; ++p) {
    const int64_t np = ixyzs[p + 1] - ixyzs[p], i0 = ixyzs[p] - 1;
    double* um = (double*)malloc(sizeof(double) * np * np);
    const int ier = disc_umat(iptype[p], norders[p], um);
    if (ier) {
      err = ier;
    } else {
      for (int64_t m = 0; m < np; ++m)
        for (int c = 0; c < 9; ++c) {
          double s = 0;
          for (int64_t l = 0; l < np; ++l) s += um[m * np + l] * srcvals[12 * (i0 + l) + c];
          srccoefs[9 * (i0 + m) + c] = s;
        }
    }
    free(um);
  }
  return err;
}

static void unit_normal(double* sv) {
  const double n0 = sv[4] * sv[8] - sv[5] * sv[7];
  const double n1 = sv[5] * sv[6] - sv[3] * sv[8];
  const double n2 = sv[3] * sv[7] - sv[4] * sv[6];
  const double r = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
  sv[9] = n0 / r;
  sv[10] = n1 / r;
  sv[11] = n2 / r;
}

/* The icosahedron refined nref times by xtri_platonic (child 1 of a triangle
 * replaces it, children 2-4 are appended), each flat triangle projected
 * radially onto the ellipsoid center + axes * x/|x| (xtri_ellipsoid_eval),
 * order-norder Vioreanu-Rokhlin nodes. */
int oracle_surf_icosa_ellipsoid(int64_t nref, int64_t norder, const double* axes,
                                const double* center, int64_t* norders, int64_t* ixyzs,
                                int64_t* iptype, double* srcvals, double* srccoefs) {
  if (nref < 0 || nref > 8 || norder < 0 || norder > 20 || !g_vr_uvs[norder]) return 1;
  const int64_t ntri = oracle_icosa_npatches(nref);
  double(*tri)[3][3] = malloc(sizeof(double) * 9 * ntri);
  double v[12][3];
  int f[20][3];
  icosahedron(v, f);
  for (int i = 0; i < 20; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) tri[i][j][k] = v[f[i][j]][k];
  int64_t n = 20;
  for (int64_t lev = 0; lev < nref; ++lev) {
    const int64_t nn = n;
    for (int64_t i = 0; i < nn; ++i) {
      double a[3], b[3], c[3], m12[3], m23[3], m13[3];
      for (int k = 0; k < 3; ++k) {
        a[k] = tri[i][0][k];
        b[k] = tri[i][1][k];
        c[k] = tri[i][2][k];
        m12[k] = (a[k] + b[k]) / 2;
        m23[k] = (b[k] + c[k]) / 2;
        m13[k] = (a[k] + c[k]) / 2;
      }
      for (int k = 0; k < 3; ++k) {
        tri[i][0][k] = a[k];
        tri[i][1][k] = m12[k];
        tri[i][2][k] = m13[k];
        tri[n][0][k] = m23[k];
        tri[n][1][k] = m13[k];
        tri[n][2][k] = m12[k];
        tri[n + 1][0][k] = m12[k];
        tri[n + 1][1][k] = b[k];
        tri[n + 1][2][k] = m23[k];
        tri[n + 2][0][k] = m13[k];
        tri[n + 2][1][k] = m23[k];
        tri[n + 2][2][k] = c[k];
      }
      n += 3;
    }
  }
  const int64_t np = npols_of(1, norder);
  const double* uvs = g_vr_uvs[norder];
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < ntri; ++p) {
    norders[p] = norder;
    iptype[p] = 1;
    ixyzs[p] = 1 + p * np;
    const double* x0 = tri[p][0];
    const double* x1 = tri[p][1];
    const double* x2 = tri[p][2];
    for (int64_t i = 0; i < np; ++i) {
      const double u = uvs[2 * i], w = uvs[2 * i + 1];
      double x[3], du[3], dv[3];
      for (int k = 0; k < 3; ++k) {
        du[k] = x1[k] - x0[k];
        dv[k] = x2[k] - x0[k];
        x[k] = x0[k] + u * du[k] + w * dv[k];
      }
      const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
      const double drdu = (x[0] * du[0] + x[1] * du[1] + x[2] * du[2]) / r;
      const double drdv = (x[0] * dv[0] + x[1] * dv[1] + x[2] * dv[2]) / r;
      double* sv = srcvals + 12 * (p * np + i);
      for (int k = 0; k < 3; ++k) {
        sv[k] = axes[k] * x[k] / r + center[k];
        sv[3 + k] = axes[k] * (r * du[k] - x[k] * drdu) / r / r;
        sv[6 + k] = axes[k] * (r * dv[k] - x[k] * drdv) / r / r;
      }
      unit_normal(sv);
    }
  }
  ixyzs[ntri] = 1 + ntri * np;
  free(tri);
  return vals_to_coefs(ntri, norders, ixyzs, iptype, srcvals, srccoefs);
}

/* The quad torus of the warm-start workload: x = (R + r(p) cos t) cos p,
 * y = (R + r(p) cos t) sin p, z = r(p) sin t, r(p) = r0 + r1 cos(m p); nu x nv
 * patches (p outer), tensor Gauss-Legendre nodes of order norder (iptype 11).
 * The surface is this repository's workload definition, not a reference
 * routine. */
int oracle_surf_torus_quad(int64_t nu, int64_t nv, int64_t norder, double R, double r0, double r1,
                           int64_t m, int64_t* norders, int64_t* ixyzs, int64_t* iptype,
                           double* srcvals, double* srccoefs) {
  if (nu < 1 || nv < 1 || norder < 0 || norder > 30) return 1;
  const int64_t np = npols_of(11, norder);
  double* uvs = malloc(sizeof(double) * 2 * np);
  disc_nodes(11, norder, uvs);
  const double pi = 4 * atan(1.0);
  const double dpu = pi / nu, dtv = pi / nv;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < nu * nv; ++p) {
    const int64_t iu = p / nv, iv = p % nv;
    norders[p] = norder;
    iptype[p] = 11;
    ixyzs[p] = 1 + p * np;
    for (int64_t i = 0; i < np; ++i) {
      const double pp = 2 * pi * (iu + 0.5 * (uvs[2 * i] + 1)) / nu;
      const double tt = 2 * pi * (iv + 0.5 * (uvs[2 * i + 1] + 1)) / nv;
      const double rp = r0 + r1 * cos(m * pp), drp = -r1 * m * sin(m * pp);
      const double rho = R + rp * cos(tt);
      double* sv = srcvals + 12 * (p * np + i);
      sv[0] = rho * cos(pp);
      sv[1] = rho * sin(pp);
      sv[2] = rp * sin(tt);
      sv[3] = (drp * cos(tt) * cos(pp) - rho * sin(pp)) * dpu;
      sv[4] = (drp * cos(tt) * sin(pp) + rho * cos(pp)) * dpu;
      sv[5] = drp * sin(tt) * dpu;
      sv[6] = -rp * sin(tt) * cos(pp) * dtv;
      sv[7] = -rp * sin(tt) * sin(pp) * dtv;
      sv[8] = rp * cos(tt) * dtv;
      unit_normal(sv);
    }
  }
  ixyzs[nu * nv] = 1 + nu * nv * np;
  free(uvs);
  return vals_to_coefs(nu * nv, norders, ixyzs, iptype, srcvals, srccoefs);
}

/* get_qwts: w = w_ref(node) |du x dv| */
int oracle_get_qwts(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                    const int64_t* iptype, int64_t npts, const double* srcvals, double* qwts) {
  (void)npts;
  int err = 0;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t p = 0; p < npatches; ++p) {
    const int64_t np = ixyzs[p + 1] - ixyzs[p];
    double* w = malloc(sizeof(double) * np);
    const int ier = disc_wts(iptype[p], norders[p], w);
    if (ier) err = ier;
    for (int64_t i = 0; i < np && !ier; ++i) {
      const double* sv = srcvals + 12 * (ixyzs[p] - 1 + i);
      const double n0 = sv[4] * sv[8] - sv[5] * sv[7];
      const double n1 = sv[5] * sv[6] - sv[3] * sv[8];
      const double n2 = sv[3] * sv[7] - sv[4] * sv[6];
      qwts[ixyzs[p] - 1 + i] = w[i] * sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    }
    free(w);
  }
  return err;
}

/* ---------------- setup --------------------------------------------------- */

void oracle_get_rfacs(int64_t norder, int64_t iptype, double* rfac, double* rfac0) {
  (void)iptype;
  *rfac = 1.25;
  if (norder <= 2) *rfac = 2.75;
  if (norder <= 6 && norder > 2) *rfac = 2.0;
  if (norder > 6) *rfac = 1.25;
  *rfac0 = 1.25;
}

/* evaluate the 9 geometry values of a patch at uv from its coefficients */
static void patch_geom(int64_t iptype, int64_t norder, int64_t np, const double* coefs,
                       const double* uv, double* pols, double* g9) {
  basis_pols(iptype, norder, uv, pols);
  for (int c = 0; c < 9; ++c) g9[c] = 0;
  for (int64_t m = 0; m < np; ++m)
    for (int c = 0; c < 9; ++c) g9[c] += coefs[9 * m + c] * pols[m];
}

/* get_centroid_rads: mean of the images of the parameter domain's corners,
 * radius = largest distance from it to a corner image */
int oracle_get_centroid_rads(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                             const int64_t* iptype, int64_t npts, const double* srccoefs,
                             double* cms, double* rads) {
  (void)npts;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < npatches; ++p) {
    const int64_t np = ixyzs[p + 1] - ixyzs[p];
    static const double tv[3][2] = {{0, 0}, {1, 0}, {0, 1}};
    static const double qv[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
    const int nv = iptype[p] == 1 ? 3 : 4;
    double* pols = malloc(sizeof(double) * np);
    double x[4][9], c[3] = {0, 0, 0};
    for (int v = 0; v < nv; ++v) {
      patch_geom(iptype[p], norders[p], np, srccoefs + 9 * (ixyzs[p] - 1),
                 iptype[p] == 1 ? tv[v] : qv[v], pols, x[v]);
      for (int k = 0; k < 3; ++k) c[k] += x[v][k];
    }
    double r2 = 0;
    for (int k = 0; k < 3; ++k) c[k] /= nv;
    for (int v = 0; v < nv; ++v) {
      const double d = (c[0] - x[v][0]) * (c[0] - x[v][0]) + (c[1] - x[v][1]) * (c[1] - x[v][1]) +
                       (c[2] - x[v][2]) * (c[2] - x[v][2]);
      if (d >= r2) r2 = d;
    }
    for (int k = 0; k < 3; ++k) cms[3 * p + k] = c[k];
    rads[p] = sqrt(r2);
    free(pols);
  }
  return 0;
}

/* findnearslow: every (target, patch) pair with |t - c_j|^2 <= rad_j^2,
 * patches in increasing order within a row.  col_ind == NULL: only row_ptr
 * (1-based) is filled, so the caller can size col_ind from row_ptr[nt] - 1. */
int oracle_findnear(const double* cms, int64_t ns, const double* rads, int64_t ndt,
                    const double* targs, int64_t nt, int64_t* row_ptr, int64_t* col_ind) {
  int64_t* cnt = calloc(nt + 1, sizeof(int64_t));
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < nt; ++i) {
    const double* t = targs + ndt * i;
    int64_t c = 0;
    for (int64_t j = 0; j < ns; ++j) {
      const double rr = (cms[3 * j] - t[0]) * (cms[3 * j] - t[0]) +
                        (cms[3 * j + 1] - t[1]) * (cms[3 * j + 1] - t[1]) +
                        (cms[3 * j + 2] - t[2]) * (cms[3 * j + 2] - t[2]);
      if (rr <= rads[j] * rads[j]) {
        if (col_ind) col_ind[row_ptr[i] - 1 + c] = j + 1;
        ++c;
      }
    }
    cnt[i] = c;
  }
  if (!col_ind) {
    row_ptr[0] = 1;
    for (int64_t i = 0; i < nt; ++i) row_ptr[i + 1] = row_ptr[i] + cnt[i];
  }
  free(cnt);
  return 0;
}

/* hkrand(iseed): LAPACK dlaran after reseeding with (0, 0, 0, (2 iseed + 1)
 * mod 4096): one step of the 48-bit multiplicative generator with multiplier
 * 494*2^36 + 322*2^24 + 2508*2^12 + 2549, returned as seed / 2^48. */
double oracle_hkrand(int64_t iseed) {
  const unsigned __int128 mult = ((unsigned __int128)494 << 36) + ((unsigned __int128)322 << 24) +
                                 ((unsigned __int128)2508 << 12) + 2549;
  int64_t s0 = (2 * iseed + 1) % 4096;
  if (s0 < 0) s0 += 4096;
  const uint64_t s = (uint64_t)(((unsigned __int128)s0 * mult) & (((unsigned __int128)1 << 48) - 1));
  return ldexp((double)s, -48);
}

/* h3d_slp (ikerorder -1) or h3d_dlp (0) at complex zk, with 1/(4 pi) */
static double complex far_order_kernel(int ikerorder, double complex zk, const double* src,
                                       const double* t) {
  const double dx = t[0] - src[0], dy = t[1] - src[1], dz = t[2] - src[2];
  const double r = sqrt(dx * dx + dy * dy + dz * dz);
  const double complex e = cexp(I * zk * r);
  if (ikerorder == -1) return e / r * OVER4PI;
  const double d = dx * src[9] + dy * src[10] + dz * src[11];
  return d * (1.0 - I * zk * r) * e / (r * r * r) * OVER4PI;
}

/* geometry (12 values) and |du x dv| of a patch at the nodes of order nf */
static int far_nodes(int64_t iptype, int64_t norder, int64_t np, const double* coefs, int64_t nf,
                     double* src12, double* qw, double* pmat) {
  const int64_t nfp = npols_of(iptype, nf);
  double* uvs = malloc(sizeof(double) * 2 * nfp);
  double* w = malloc(sizeof(double) * nfp);
  int ier = disc_nodes(iptype, nf, uvs);
  if (!ier) ier = disc_wts(iptype, nf, w);
  for (int64_t j = 0; j < nfp && !ier; ++j) {
    double* s = src12 + 12 * j;
    patch_geom(iptype, norder, np, coefs, uvs + 2 * j, pmat + np * j, s);
    unit_normal(s);
    const double n0 = s[4] * s[8] - s[5] * s[7];
    const double n1 = s[5] * s[6] - s[3] * s[8];
    const double n2 = s[3] * s[7] - s[4] * s[6];
    qw[j] = w[j] * sqrt(n0 * n0 + n1 * n1 + n2 * n2);
  }
  free(uvs);
  free(w);
  return ier;
}

/* get_far_order_guru for one patch: probes = the min(10, ntarg/2) farthest of
 * the patch's near targets and hkrand points on the sphere of radius rad0
 * about the centroid (25 in all); the basis integrals against the probes at
 * successive orders of {1,2,3,4,6,8,10,12,14,16}; the first order whose
 * successor changes them by less than eps (min |du x dv|^2)^(1/4) (largest
 * l2 change over probes) is kept, 16 when none does. */
static int far_order_patch(double eps, int64_t norder, int64_t np, int64_t iptype,
                           const double* cm, double rad0, const double* coefs, int ikerorder,
                           double complex zk, int64_t ndtarg, int64_t nnear, const double* targs,
                           const int64_t* near_t, int64_t* nfar_out) {
  static const int64_t orders[10] = {1, 2, 3, 4, 6, 8, 10, 12, 14, 16};
  const int nmax = 25;
  const double pi = 4 * atan(1.0);
  double tt[25][3];
  /* the farthest near targets, ties by target index */
  int64_t* ord = malloc(sizeof(int64_t) * (nnear > 0 ? nnear : 1));
  double* dd = malloc(sizeof(double) * (nnear > 0 ? nnear : 1));
  for (int64_t i = 0; i < nnear; ++i) {
    const double* t = targs + ndtarg * near_t[i];
    dd[i] = (t[0] - cm[0]) * (t[0] - cm[0]) + (t[1] - cm[1]) * (t[1] - cm[1]) +
            (t[2] - cm[2]) * (t[2] - cm[2]);
    ord[i] = i;
  }
  const int64_t i0 = nnear / 2 < 10 ? nnear / 2 : 10;
  for (int64_t a = 0; a < i0; ++a) { /* partial selection sort: largest first */
    int64_t b = a;
    for (int64_t c = a + 1; c < nnear; ++c)
      if (dd[ord[c]] > dd[ord[b]] || (dd[ord[c]] == dd[ord[b]] && ord[c] > ord[b])) b = c;
    const int64_t t = ord[a];
    ord[a] = ord[b];
    ord[b] = t;
  }
  for (int64_t i = 0; i < i0; ++i)
    for (int k = 0; k < 3; ++k) tt[i][k] = targs[ndtarg * near_t[ord[i]] + k];
  for (int64_t i = i0 + 1; i <= nmax; ++i) { /* 1-based probe index as in the reference */
    const double phi = oracle_hkrand(1001 + i) * 2 * pi;
    const double thet = oracle_hkrand(3042 + i) * pi;
    tt[i - 1][0] = cm[0] + rad0 * sin(thet) * cos(phi);
    tt[i - 1][1] = cm[1] + rad0 * sin(thet) * sin(phi);
    tt[i - 1][2] = cm[2] + rad0 * cos(thet);
  }
  free(ord);
  free(dd);

  const int64_t npmax = 17 * 17;
  double* src = malloc(sizeof(double) * 12 * npmax);
  double* qw = malloc(sizeof(double) * npmax);
  double* pmat = malloc(sizeof(double) * np * npmax);
  double complex* vcomp = malloc(sizeof(double complex) * np * nmax);
  double complex* vref = malloc(sizeof(double complex) * np * nmax);
  /* epsp from the patch's own nodes */
  int ier = far_nodes(iptype, norder, np, coefs, norder, src, qw, pmat);
  double rsc = 0;
  for (int64_t j = 0; j < np && !ier; ++j) {
    const double* s = src + 12 * j;
    const double n0 = s[4] * s[8] - s[5] * s[7];
    const double n1 = s[5] * s[6] - s[3] * s[8];
    const double n2 = s[3] * s[7] - s[4] * s[6];
    const double r2 = n0 * n0 + n1 * n1 + n2 * n2;
    if (j == 0 || r2 < rsc) rsc = r2;
  }
  const double epsp = pow(rsc, 0.25) * eps;
  int64_t kept = 9;
  for (int64_t o = 0; o < 10 && !ier; ++o) {
    const int64_t nf = orders[o], nfp = npols_of(iptype, nf);
    ier = far_nodes(iptype, norder, np, coefs, nf, src, qw, pmat);
    if (ier) break;
    double complex* v = o == 0 ? vcomp : vref;
    for (int it = 0; it < nmax; ++it) {
      for (int64_t l = 0; l < np; ++l) v[it * np + l] = 0;
      for (int64_t j = 0; j < nfp; ++j) {
        const double complex val = far_order_kernel(ikerorder, zk, src + 12 * j, tt[it]) * qw[j];
        for (int64_t l = 0; l < np; ++l) v[it * np + l] += val * pmat[np * j + l];
      }
    }
    if (o == 0) continue;
    double errmax = 0;
    for (int it = 0; it < nmax; ++it) {
      double e2 = 0;
      for (int64_t l = 0; l < np; ++l) {
        const double e = cabs(vref[it * np + l] - vcomp[it * np + l]);
        e2 += e * e;
      }
      if (sqrt(e2) > errmax) errmax = sqrt(e2);
    }
    if (errmax < epsp) {
      kept = o - 1;
      break;
    }
    memcpy(vcomp, vref, sizeof(double complex) * np * nmax);
  }
  *nfar_out = orders[kept];
  free(src);
  free(qw);
  free(pmat);
  free(vcomp);
  free(vref);
  return ier;
}

/* get_far_order: nfars per patch and ixyzso.  zk = (re, im). */
int oracle_get_far_order(double eps, int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                         const int64_t* iptype, const double* cms, const double* rads, int64_t npts,
                         const double* srccoefs, int64_t ndtarg, int64_t ntarg, const double* targs,
                         int64_t ikerorder, const double* zk, int64_t nnz, const int64_t* row_ptr,
                         const int64_t* col_ind, double rfac, int64_t* nfars, int64_t* ixyzso) {
  (void)npts;
  /* transpose of the near list: the targets near each patch, in target order */
  int64_t* cp = calloc(npatches + 1, sizeof(int64_t));
  int64_t* rows = malloc(sizeof(int64_t) * (nnz > 0 ? nnz : 1));
  for (int64_t k = 0; k < nnz; ++k) cp[col_ind[k]]++;
  for (int64_t p = 0; p < npatches; ++p) cp[p + 1] += cp[p];
  int64_t* fill = calloc(npatches, sizeof(int64_t));
  for (int64_t i = 0; i < ntarg; ++i)
    for (int64_t k = row_ptr[i] - 1; k < row_ptr[i + 1] - 1; ++k) {
      const int64_t p = col_ind[k] - 1;
      rows[cp[p] + fill[p]++] = i;
    }
  free(fill);
  const double complex z = zk[0] + I * zk[1];
  int err = 0;
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t p = 0; p < npatches; ++p) {
    const int64_t np = ixyzs[p + 1] - ixyzs[p];
    const int ier = far_order_patch(eps, norders[p], np, iptype[p], cms + 3 * p, rfac * rads[p],
                                    srccoefs + 9 * (ixyzs[p] - 1), (int)ikerorder, z, ndtarg,
                                    cp[p + 1] - cp[p], targs, rows + cp[p], &nfars[p]);
    if (ier) err = ier;
  }
  ixyzso[0] = 1;
  for (int64_t p = 0; p < npatches; ++p) ixyzso[p + 1] = ixyzso[p] + npols_of(iptype[p], nfars[p]);
  free(cp);
  free(rows);
  return err;
}

/* oversample_geom: geometry at the nodes of order nfar from the patch
 * expansion; nodes shared by the two node sets (distance^2 <= 1e-24 in the
 * parameter domain, the rule get_clashing_indices states) copy srcvals. */
int oracle_oversample_geom(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                           const int64_t* iptype, int64_t npts, const double* srccoefs,
                           const double* srcvals, const int64_t* nfars, const int64_t* ixyzso,
                           int64_t nptso, double* srcover) {
  (void)npts;
  (void)nptso;
  int err = 0;
#pragma omp parallel for schedule(dynamic, 8)
  for (int64_t p = 0; p < npatches; ++p) {
    const int64_t np = ixyzs[p + 1] - ixyzs[p], nfp = ixyzso[p + 1] - ixyzso[p];
    double* out = srcover + 12 * (ixyzso[p] - 1);
    const double* vals = srcvals + 12 * (ixyzs[p] - 1);
    if (nfars[p] == norders[p]) {
      memcpy(out, vals, sizeof(double) * 12 * np);
      continue;
    }
    double* uv0 = malloc(sizeof(double) * 2 * np);
    double* uvf = malloc(sizeof(double) * 2 * nfp);
    double* pols = malloc(sizeof(double) * np);
    int ier = disc_nodes(iptype[p], norders[p], uv0);
    if (!ier) ier = disc_nodes(iptype[p], nfars[p], uvf);
    for (int64_t j = 0; j < nfp && !ier; ++j) {
      patch_geom(iptype[p], norders[p], np, srccoefs + 9 * (ixyzs[p] - 1), uvf + 2 * j, pols,
                 out + 12 * j);
      unit_normal(out + 12 * j);
      for (int64_t i = 0; i < np; ++i) {
        const double du = uv0[2 * i] - uvf[2 * j], dv = uv0[2 * i + 1] - uvf[2 * j + 1];
        if (du * du + dv * dv <= 1e-24) memcpy(out + 12 * j, vals + 12 * i, sizeof(double) * 12);
      }
    }
    if (ier) err = ier;
    free(uv0);
    free(uvf);
    free(pols);
  }
  return err;
}

/* ---------------- near quadrature ------------------------------------------ */

/* relative tolerance of the adaptive rules (absolute tolerance = this times
 * (|alpha| + |beta|/R) A/(4 pi R)) */
static double g_nq_tol = 1e-9;
void oracle_set_nq_tol(double tol) { g_nq_tol = tol; }

typedef struct {
  int64_t iptype, norder, np;
  const double* coefs; /* 9 x np */
  const double* t;     /* target xyz */
  double complex zk, alpha, beta;
  double complex* acc; /* np integrals */
  double* pols;
  int64_t evals;
} NqCtx;

/* K(t, X(uv)) |J| P_m(uv) * wgt added to out[m] */
static void nq_point(NqCtx* c, const double* uv, double wgt, double complex* out) {
  double g[9];
  patch_geom(c->iptype, c->norder, c->np, c->coefs, uv, c->pols, g);
  const double n0 = g[4] * g[8] - g[5] * g[7];
  const double n1 = g[5] * g[6] - g[3] * g[8];
  const double n2 = g[3] * g[7] - g[4] * g[6];
  const double J = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
  const double dx = c->t[0] - g[0], dy = c->t[1] - g[1], dz = c->t[2] - g[2];
  const double r2 = dx * dx + dy * dy + dz * dz;
  const double r = sqrt(r2);
  const double dn = (dx * n0 + dy * n1 + dz * n2) / J;
  const double kr = creal(c->zk) * r, ki = cimag(c->zk) * r;
  const double ea = ki != 0 ? exp(-ki) : 1.0;
  double sn, cs;
  sincos(kr, &sn, &cs);
  const double complex e = ea * cs + I * (ea * sn);
  const double rinv = 1.0 / r;
  const double complex k =
      (c->alpha + c->beta * dn * (1.0 - I * c->zk * r) * rinv * rinv) * e * (OVER4PI * rinv);
  const double complex f = k * J * wgt;
  for (int64_t m = 0; m < c->np; ++m) out[m] += f * c->pols[m];
  c->evals++;
}

/* Vioreanu-Rokhlin order-12 rule on the triangle (a, b, c) of the parameter
 * domain */
#define NQ_RULE 12
static void nq_tri(NqCtx* c, const double* a, const double* b, const double* d,
                   double complex* out) {
  const int64_t nr = g_vr_np[NQ_RULE];
  const double* ru = g_vr_uvs[NQ_RULE];
  const double* rw = g_vr_wts[NQ_RULE];
  const double e1[2] = {b[0] - a[0], b[1] - a[1]}, e2[2] = {d[0] - a[0], d[1] - a[1]};
  const double jac = fabs(e1[0] * e2[1] - e1[1] * e2[0]);
  for (int64_t m = 0; m < c->np; ++m) out[m] = 0;
  for (int64_t q = 0; q < nr; ++q) {
    const double uv[2] = {a[0] + ru[2 * q] * e1[0] + ru[2 * q + 1] * e2[0],
                          a[1] + ru[2 * q] * e1[1] + ru[2 * q + 1] * e2[1]};
    nq_point(c, uv, rw[q] * jac, out);
  }
}

static double maxdiff(int64_t n, const double complex* a, const double complex* b) {
  double m = 0;
  for (int64_t i = 0; i < n; ++i) {
    const double d = cabs(a[i] - b[i]);
    if (d > m) m = d;
  }
  return m;
}

typedef struct {
  double v[3][2];
  int lev;
} NqTri;

/* adaptive 4-way subdivision from the root triangles of the domain */
static void nq_adaptive(NqCtx* c, double tol) {
  const int64_t np = c->np;
  int cap = 256, top = 0;
  NqTri* st = malloc(sizeof(NqTri) * cap);
  double complex* sv = malloc(sizeof(double complex) * np * cap); /* integral of each entry */
  double complex* ch = malloc(sizeof(double complex) * np * 4);
  double complex* sum = malloc(sizeof(double complex) * np);
  if (c->iptype == 1) {
    st[0] = (NqTri){{{0, 0}, {1, 0}, {0, 1}}, 0};
    top = 1;
  } else {
    st[0] = (NqTri){{{-1, -1}, {1, -1}, {1, 1}}, 0};
    st[1] = (NqTri){{{-1, -1}, {1, 1}, {-1, 1}}, 0};
    top = 2;
  }
  for (int i = 0; i < top; ++i) nq_tri(c, st[i].v[0], st[i].v[1], st[i].v[2], sv + np * i);
  while (top > 0) {
    --top;
    const NqTri T = st[top];
    double complex* parent = sv + np * top;
    double m01[2], m12[2], m02[2];
    for (int k = 0; k < 2; ++k) {
      m01[k] = 0.5 * (T.v[0][k] + T.v[1][k]);
      m12[k] = 0.5 * (T.v[1][k] + T.v[2][k]);
      m02[k] = 0.5 * (T.v[0][k] + T.v[2][k]);
    }
    NqTri kids[4] = {{{{T.v[0][0], T.v[0][1]}, {m01[0], m01[1]}, {m02[0], m02[1]}}, T.lev + 1},
                     {{{m01[0], m01[1]}, {T.v[1][0], T.v[1][1]}, {m12[0], m12[1]}}, T.lev + 1},
                     {{{m02[0], m02[1]}, {m12[0], m12[1]}, {T.v[2][0], T.v[2][1]}}, T.lev + 1},
                     {{{m12[0], m12[1]}, {m02[0], m02[1]}, {m01[0], m01[1]}}, T.lev + 1}};
    for (int q = 0; q < 4; ++q) nq_tri(c, kids[q].v[0], kids[q].v[1], kids[q].v[2], ch + np * q);
    for (int64_t m = 0; m < np; ++m) sum[m] = ch[m] + ch[np + m] + ch[2 * np + m] + ch[3 * np + m];
    if (maxdiff(np, parent, sum) <= tol || T.lev >= 30) {
      for (int64_t m = 0; m < np; ++m) c->acc[m] += sum[m];
      continue;
    }
    if (top + 4 > cap) {
      cap *= 2;
      st = realloc(st, sizeof(NqTri) * cap);
      sv = realloc(sv, sizeof(double complex) * np * cap);
    }
    for (int q = 0; q < 4; ++q) {
      st[top] = kids[q];
      memcpy(sv + np * top, ch + np * q, sizeof(double complex) * np);
      ++top;
    }
  }
  free(st);
  free(sv);
  free(ch);
  free(sum);
}

#define NQ_GL 20
static double g_gl_x[NQ_GL], g_gl_w[NQ_GL]; /* on [0, 1] */

/* polar integral over theta in [th0, th1] of the triangle (uv0, va, vb):
 * int_th int_0^R(th) f(uv0 + rho e(th)) rho drho dth with 20-point rules */
static void nq_polar_panel(NqCtx* c, const double* uv0, const double* va, const double* vb,
                           double th0, double th1, double complex* out) {
  const double ex = vb[0] - va[0], ey = vb[1] - va[1];
  const double num = (va[0] - uv0[0]) * ey - (va[1] - uv0[1]) * ex;
  for (int64_t m = 0; m < c->np; ++m) out[m] = 0;
  for (int i = 0; i < NQ_GL; ++i) {
    const double th = th0 + (th1 - th0) * g_gl_x[i];
    const double ct = cos(th), st = sin(th);
    const double R = num / (ct * ey - st * ex);
    const double wt = (th1 - th0) * g_gl_w[i];
    for (int j = 0; j < NQ_GL; ++j) {
      const double rho = R * g_gl_x[j];
      const double uv[2] = {uv0[0] + rho * ct, uv0[1] + rho * st};
      nq_point(c, uv, wt * R * g_gl_w[j] * rho, out);
    }
  }
}

static void nq_self(NqCtx* c, const double* uv0, double tol) {
  static const double tv[3][2] = {{0, 0}, {1, 0}, {0, 1}};
  static const double qv[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
  const int nv = c->iptype == 1 ? 3 : 4;
  const int64_t np = c->np;
  double complex* a = malloc(sizeof(double complex) * np);
  double complex* l = malloc(sizeof(double complex) * np);
  double complex* r = malloc(sizeof(double complex) * np);
  int cap = 128;
  double (*stk)[3] = malloc(sizeof(double) * 3 * cap); /* th0, th1, level */
  double complex* sv = malloc(sizeof(double complex) * np * cap);
  for (int e = 0; e < nv; ++e) {
    const double* va = c->iptype == 1 ? tv[e] : qv[e];
    const double* vb = c->iptype == 1 ? tv[(e + 1) % nv] : qv[(e + 1) % nv];
    const double tha = atan2(va[1] - uv0[1], va[0] - uv0[0]);
    double thb = atan2(vb[1] - uv0[1], vb[0] - uv0[0]);
    while (thb <= tha) thb += 8 * atan(1.0);
    int top = 0;
    stk[0][0] = tha;
    stk[0][1] = thb;
    stk[0][2] = 0;
    nq_polar_panel(c, uv0, va, vb, tha, thb, sv);
    top = 1;
    while (top > 0) {
      --top;
      const double t0 = stk[top][0], t1 = stk[top][1], lev = stk[top][2];
      memcpy(a, sv + np * top, sizeof(double complex) * np);
      const double tm = 0.5 * (t0 + t1);
      nq_polar_panel(c, uv0, va, vb, t0, tm, l);
      nq_polar_panel(c, uv0, va, vb, tm, t1, r);
      double dmax = 0;
      for (int64_t m = 0; m < np; ++m) {
        const double d = cabs(a[m] - l[m] - r[m]);
        if (d > dmax) dmax = d;
      }
      if (dmax <= tol || lev >= 40) {
        for (int64_t m = 0; m < np; ++m) c->acc[m] += l[m] + r[m];
        continue;
      }
      if (top + 2 > cap) {
        cap *= 2;
        stk = realloc(stk, sizeof(double) * 3 * cap);
        sv = realloc(sv, sizeof(double complex) * np * cap);
      }
      memcpy(sv + np * top, l, sizeof(double complex) * np);
      stk[top][0] = t0;
      stk[top][1] = tm;
      stk[top][2] = lev + 1;
      ++top;
      memcpy(sv + np * top, r, sizeof(double complex) * np);
      stk[top][0] = tm;
      stk[top][1] = t1;
      stk[top][2] = lev + 1;
      ++top;
    }
  }
  free(a);
  free(l);
  free(r);
  free(stk);
  free(sv);
}

/* getnearquad_{lap,helm}_comb_dir_eval: wnear for every (target, patch)
 * pair of the near list.  kind 0: params = (alpha, beta) real, wnear real;
 * kind 1: params = (zk, alpha, beta) complex interleaved, wnear complex
 * interleaved.  ipatch_id (1-based, <= 0 for none) and uvs_targ mark targets
 * on a patch.  stats[0] += kernel evaluations (may be NULL). */
int oracle_getnearquad(int64_t kind, int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                       const int64_t* iptype, int64_t npts, const double* srccoefs,
                       const double* srcvals, int64_t ndtarg, int64_t ntarg, const double* targs,
                       const int64_t* ipatch_id, const double* uvs_targ, double eps,
                       const double* params, int64_t nnz, const int64_t* row_ptr,
                       const int64_t* col_ind, const int64_t* iquad, int64_t nquad, double* wnear,
                       int64_t* stats) {
  (void)npts;
  (void)srcvals;
  (void)eps;
  (void)nnz;
  (void)nquad;
  if (!g_vr_uvs[NQ_RULE] || !g_vr_wts[NQ_RULE]) return 6;
  legendre_nodes(NQ_GL, g_gl_x);
  legendre_weights(NQ_GL, g_gl_x, g_gl_w);
  for (int i = 0; i < NQ_GL; ++i) {
    g_gl_x[i] = 0.5 * (g_gl_x[i] + 1);
    g_gl_w[i] *= 0.5;
  }
  double complex zk = 0, alpha, beta;
  if (kind == 0) {
    alpha = params[0];
    beta = params[1];
  } else {
    zk = params[0] + I * params[1];
    alpha = params[2] + I * params[3];
    beta = params[4] + I * params[5];
  }
  /* per-patch area, radius, umat */
  double* area = calloc(npatches, sizeof(double));
  double* rad = calloc(npatches, sizeof(double));
  double* cms = calloc(3 * npatches, sizeof(double));
  oracle_get_centroid_rads(npatches, norders, ixyzs, iptype, 0, srccoefs, cms, rad);
  int64_t umax = 0;
  for (int64_t p = 0; p < npatches; ++p)
    if (ixyzs[p + 1] - ixyzs[p] > umax) umax = ixyzs[p + 1] - ixyzs[p];
  double** umats = calloc(npatches, sizeof(double*));
  int err = 0;
#pragma omp parallel for schedule(dynamic, 8)
  for (int64_t p = 0; p < npatches; ++p) {
    const int64_t np = ixyzs[p + 1] - ixyzs[p];
    umats[p] = malloc(sizeof(double) * np * np);
    if (disc_umat(iptype[p], norders[p], umats[p])) err = 7;
    double* uvs = malloc(sizeof(double) * 2 * np);
    double* w = malloc(sizeof(double) * np);
    double* pols = malloc(sizeof(double) * np);
    disc_nodes(iptype[p], norders[p], uvs);
    disc_wts(iptype[p], norders[p], w);
    double a = 0;
    for (int64_t i = 0; i < np; ++i) {
      double g[9];
      patch_geom(iptype[p], norders[p], np, srccoefs + 9 * (ixyzs[p] - 1), uvs + 2 * i, pols, g);
      const double n0 = g[4] * g[8] - g[5] * g[7];
      const double n1 = g[5] * g[6] - g[3] * g[8];
      const double n2 = g[3] * g[7] - g[4] * g[6];
      a += w[i] * sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    }
    area[p] = a;
    free(uvs);
    free(w);
    free(pols);
  }
  int64_t nev = 0;
#pragma omp parallel reduction(+ : nev)
  {
    NqCtx c;
    c.zk = zk;
    c.alpha = alpha;
    c.beta = beta;
    c.acc = malloc(sizeof(double complex) * umax);
    c.pols = malloc(sizeof(double) * umax);
    c.evals = 0;
#pragma omp for schedule(dynamic, 4)
    for (int64_t i = 0; i < ntarg; ++i) {
      for (int64_t k = row_ptr[i] - 1; k < row_ptr[i + 1] - 1; ++k) {
        const int64_t p = col_ind[k] - 1;
        c.iptype = iptype[p];
        c.norder = norders[p];
        c.np = ixyzs[p + 1] - ixyzs[p];
        c.coefs = srccoefs + 9 * (ixyzs[p] - 1);
        c.t = targs + ndtarg * i;
        for (int64_t m = 0; m < c.np; ++m) c.acc[m] = 0;
        const double R = rad[p];
        const double tol = g_nq_tol * (cabs(alpha) + cabs(beta) / R) * area[p] * OVER4PI / R;
        if (ipatch_id && ipatch_id[i] == p + 1)
          nq_self(&c, uvs_targ + 2 * i, tol);
        else
          nq_adaptive(&c, tol);
        const double* um = umats[p];
        const int64_t q0 = iquad[k] - 1;
        for (int64_t l = 0; l < c.np; ++l) {
          double complex s = 0;
          for (int64_t m = 0; m < c.np; ++m) s += c.acc[m] * um[m * c.np + l];
          if (kind == 0) {
            wnear[q0 + l] = creal(s);
          } else {
            wnear[2 * (q0 + l)] = creal(s);
            wnear[2 * (q0 + l) + 1] = cimag(s);
          }
        }
      }
    }
    nev += c.evals;
    free(c.acc);
    free(c.pols);
  }
  if (stats) stats[0] += nev;
  for (int64_t p = 0; p < npatches; ++p) free(umats[p]);
  free(umats);
  free(area);
  free(rad);
  free(cms);
  return err;
}
