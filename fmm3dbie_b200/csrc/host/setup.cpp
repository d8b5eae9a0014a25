// Host-side setup for the layer-potential path (see setup.h).
#include "setup.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <numeric>
#include <unordered_map>

#include "basis.h"

namespace bie {

namespace {
inline void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
inline double norm3(const double* a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

using V3 = std::array<double, 3>;
using Tri = std::array<V3, 3>;

// The icosahedron of xtri_rsolid (itype 4, xtri_parameterizations.f90:1674-1829):
// a ring of five vertices at angles 2 pi i / 5 lifted to the height that
// makes the apex (0, 0, d) equidistant, the apex, and the point reflections
// of those six; faces in the reference's order and orientation, so that
// (v1-v0)x(v2-v0) points outward; vertices scaled to the unit sphere.
std::vector<Tri> icosahedron() {
  const double pi = 4.0 * std::atan(1.0);
  std::array<V3, 12> v{};
  for (int i = 0; i < 5; ++i) v[i] = {std::cos(2 * pi * (i + 1) / 5.0), std::sin(2 * pi * (i + 1) / 5.0), 0.0};
  const double edge = std::hypot(v[1][0] - v[0][0], v[1][1] - v[0][1]);
  const double apex = std::sqrt(edge * edge - 1.0);
  v[5] = {0.0, 0.0, apex};
  const double lift = (1.0 - apex * apex) / (2.0 * apex);
  for (int i = 0; i < 6; ++i) {
    v[i][2] += lift;
    v[i + 6] = {-v[i][0], -v[i][1], -v[i][2]};
  }
  const double scale = 1.0 / norm3(v[0].data());
  for (auto& p : v)
    for (auto& c : p) c *= scale;
  static const int faces[20][3] = {{0, 1, 5},  {1, 2, 5}, {2, 3, 5},  {3, 4, 5},  {4, 0, 5},
                                   {7, 6, 11}, {8, 7, 11}, {9, 8, 11}, {10, 9, 11}, {6, 10, 11},
                                   {1, 0, 9},  {2, 1, 10}, {3, 2, 6},  {4, 3, 7},  {0, 4, 8},
                                   {7, 8, 4},  {8, 9, 0},  {9, 10, 1}, {10, 6, 2}, {6, 7, 3}};
  std::vector<Tri> out;
  for (const auto& f : faces) out.push_back({v[f[0]], v[f[1]], v[f[2]]});
  return out;
}

// Flat 4-way refinement in xtri_platonic's order (xtri_parameterizations.f90:
// 1335-1413, xtri_refine4_flat :1864-1949): triangle i becomes its corner
// child (v0, m01, m02) in place and the other three children
// (m12, m02, m01), (m01, v1, m12), (m02, m12, v2) are appended, so patch
// numbering matches the reference's at every level.
std::vector<Tri> refine4(const std::vector<Tri>& in) {
  std::vector<Tri> out(in);
  out.reserve(in.size() * 4);
  for (size_t i = 0; i < in.size(); ++i) {
    const Tri& t = in[i];
    V3 m01, m12, m02;
    for (int k = 0; k < 3; ++k) {
      m01[k] = 0.5 * (t[0][k] + t[1][k]);
      m12[k] = 0.5 * (t[1][k] + t[2][k]);
      m02[k] = 0.5 * (t[0][k] + t[2][k]);
    }
    out[i] = {t[0], m01, m02};
    out.push_back({m12, m02, m01});
    out.push_back({m01, t[1], m12});
    out.push_back({m02, m12, t[2]});
  }
  return out;
}

// Radial projection of the flat triangle onto an ellipsoid, with
// derivatives (xtri_ellipsoid_eval, xtri_parameterizations.f90:247-334).
void ellipsoid_chart(const Tri& t, double u, double v, const double* ax, const double* c,
                     double* out12) {
  double x[3], du[3], dv[3];
  for (int k = 0; k < 3; ++k) {
    du[k] = t[1][k] - t[0][k];
    dv[k] = t[2][k] - t[0][k];
    x[k] = t[0][k] + u * du[k] + v * dv[k];
  }
  const double r = norm3(x);
  const double xdu = x[0] * du[0] + x[1] * du[1] + x[2] * du[2];
  const double xdv = x[0] * dv[0] + x[1] * dv[1] + x[2] * dv[2];
  for (int k = 0; k < 3; ++k) {
    out12[k] = ax[k] * x[k] / r + c[k];
    out12[3 + k] = ax[k] * (du[k] / r - x[k] * xdu / (r * r * r));
    out12[6 + k] = ax[k] * (dv[k] / r - x[k] * xdv / (r * r * r));
  }
}

void finish_normal(double* sv) {
  double n[3];
  cross3(sv + 3, sv + 6, n);
  const double r = norm3(n);
  for (int k = 0; k < 3; ++k) sv[9 + k] = n[k] / r;
}
}  // namespace

int64_t icosa_npatches(int nref) {
  int64_t n = 20;
  for (int i = 0; i < nref; ++i) n *= 4;
  return n;
}

int vals_to_coefs(const Surf& s, const double* srcvals, double* srccoefs) {
  std::map<std::pair<int, int>, std::vector<double>> umats;
  for (int64_t p = 0; p < s.npatches; ++p) {
    const int ip = int(s.iptype[p]), no = int(s.norders[p]);
    const int np = npols_of(ip, no);
    if (np != s.npols(p)) return 1;
    auto key = std::make_pair(ip, no);
    if (!umats.count(key)) {
      std::vector<double> uvs(2 * np), um(np * np), vm(np * np), w(np);
      const int ier = disc_exps(ip, no, uvs.data(), um.data(), vm.data(), w.data());
      if (ier) return ier;
      umats[key] = um;
    }
    const auto& um = umats[key];
    const int64_t st = s.start(p);
    for (int i = 0; i < np; ++i)
      for (int j = 0; j < 9; ++j) {
        double acc = 0;
        for (int l = 0; l < np; ++l) acc += um[i * np + l] * srcvals[12 * (st + l) + j];
        srccoefs[9 * (st + i) + j] = acc;
      }
  }
  return 0;
}

int surf_icosa_ellipsoid(int nref, int norder, const double axes[3], const double center[3],
                         int64_t* norders, int64_t* ixyzs, int64_t* iptype, double* srcvals,
                         double* srccoefs) {
  if (!valid_patch(1, norder) || nref < 0 || nref > 8) return 1;
  std::vector<Tri> tris = icosahedron();
  for (int i = 0; i < nref; ++i) tris = refine4(tris);
  const int np = npols_of(1, norder);
  std::vector<double> uvs(2 * np);
  const int ier = disc_nodes(1, norder, uvs.data());
  if (ier) return ier;
  const int64_t npatches = int64_t(tris.size());
  for (int64_t p = 0; p < npatches; ++p) {
    norders[p] = norder;
    iptype[p] = 1;
    ixyzs[p] = 1 + p * np;
    for (int i = 0; i < np; ++i) {
      double* sv = srcvals + 12 * (p * np + i);
      ellipsoid_chart(tris[p], uvs[2 * i], uvs[2 * i + 1], axes, center, sv);
      finish_normal(sv);
    }
  }
  ixyzs[npatches] = 1 + npatches * np;
  Surf s;
  s.npatches = npatches;
  s.npts = npatches * np;
  s.norders = norders;
  s.ixyzs = ixyzs;
  s.iptype = iptype;
  return vals_to_coefs(s, srcvals, srccoefs);
}

int surf_torus_quad(int nu, int nv, int norder, double R, double r0, double r1, int m,
                    int64_t* norders, int64_t* ixyzs, int64_t* iptype, double* srcvals,
                    double* srccoefs) {
  if (!valid_patch(11, norder) || nu < 1 || nv < 1) return 1;
  const int np = npols_of(11, norder);
  std::vector<double> uvs(2 * np);
  disc_nodes(11, norder, uvs.data());
  const int64_t npatches = int64_t(nu) * nv;
  const double dpu = M_PI / nu, dtv = M_PI / nv;  // d(p)/du, d(t)/dv
  for (int iu = 0; iu < nu; ++iu)
    for (int iv = 0; iv < nv; ++iv) {
      const int64_t p = int64_t(iu) * nv + iv;
      norders[p] = norder;
      iptype[p] = 11;
      ixyzs[p] = 1 + p * np;
      for (int i = 0; i < np; ++i) {
        const double pp = 2.0 * M_PI * (iu + 0.5 * (uvs[2 * i] + 1.0)) / nu;
        const double tt = 2.0 * M_PI * (iv + 0.5 * (uvs[2 * i + 1] + 1.0)) / nv;
        const double rp = r0 + r1 * std::cos(m * pp), drp = -r1 * m * std::sin(m * pp);
        const double cp = std::cos(pp), sp = std::sin(pp), ct = std::cos(tt), st = std::sin(tt);
        double* sv = srcvals + 12 * (p * np + i);
        const double rho = R + rp * ct;
        sv[0] = rho * cp;
        sv[1] = rho * sp;
        sv[2] = rp * st;
        sv[3] = (drp * ct * cp - rho * sp) * dpu;
        sv[4] = (drp * ct * sp + rho * cp) * dpu;
        sv[5] = drp * st * dpu;
        sv[6] = -rp * st * cp * dtv;
        sv[7] = -rp * st * sp * dtv;
        sv[8] = rp * ct * dtv;
        finish_normal(sv);
      }
    }
  ixyzs[npatches] = 1 + npatches * np;
  Surf s;
  s.npatches = npatches;
  s.npts = npatches * np;
  s.norders = norders;
  s.ixyzs = ixyzs;
  s.iptype = iptype;
  return vals_to_coefs(s, srcvals, srccoefs);
}

void centroid_rads(const Surf& s, double* cms, double* rads) {
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < s.npatches; ++p) {
    const int ip = int(s.iptype[p]), no = int(s.norders[p]);
    const int np = int(s.npols(p));
    double uv[8];
    const int nv = boundary_vertices(ip, uv);
    std::vector<double> pols(np);
    double xyz[4][3] = {};
    const double* sc = s.srccoefs + 9 * s.start(p);
    for (int j = 0; j < nv; ++j) {
      basis_pols(ip, no, uv[2 * j], uv[2 * j + 1], pols.data());
      for (int l = 0; l < np; ++l)
        for (int k = 0; k < 3; ++k) xyz[j][k] += sc[9 * l + k] * pols[l];
    }
    double c[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k) {
      for (int j = 0; j < nv; ++j) c[k] += xyz[j][k];
      c[k] /= nv;
    }
    double rmax = 0;
    for (int j = 0; j < nv; ++j) {
      const double r2 = (c[0] - xyz[j][0]) * (c[0] - xyz[j][0]) + (c[1] - xyz[j][1]) * (c[1] - xyz[j][1]) +
                        (c[2] - xyz[j][2]) * (c[2] - xyz[j][2]);
      rmax = std::max(rmax, r2);
    }
    for (int k = 0; k < 3; ++k) cms[3 * p + k] = c[k];
    rads[p] = std::sqrt(rmax);
  }
}

void rfacs(int norder, int /*iptype*/, double* rfac, double* rfac0) {
  // near_field_routs.f:826-846
  double r = 1.25;
  if (norder <= 2) r = 2.75;
  if (norder <= 6 && norder > 2) r = 2.0;
  if (norder > 6) r = 1.25;
  *rfac = r;
  *rfac0 = 1.25;
}

void qwts(const Surf& s, double* wts) {
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < s.npatches; ++p) {
    const int np = int(s.npols(p));
    std::vector<double> w0(np);
    disc_wts(int(s.iptype[p]), int(s.norders[p]), w0.data());
    for (int j = 0; j < np; ++j) {
      const double* sv = s.srcvals + 12 * (s.start(p) + j);
      double n[3];
      cross3(sv + 3, sv + 6, n);
      wts[s.start(p) + j] = norm3(n) * w0[j];
    }
  }
}

double fmm_thresh(int64_t ns, const double* src, int nds, int64_t nt, const double* trg, int ndt) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  auto upd = [&](const double* x) {
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], x[k]);
      hi[k] = std::max(hi[k], x[k]);
    }
  };
  for (int64_t i = 0; i < ns; ++i) upd(src + size_t(nds) * i);
  for (int64_t i = 0; i < nt; ++i) upd(trg + size_t(ndt) * i);
  const double b = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]});
  return std::ldexp(b, -51);  // get_fmm_thresh.f:81
}

void patch_id_uvs(const Surf& s, int64_t* ipatch_id, double* uvs) {
  for (int64_t p = 0; p < s.npatches; ++p) {
    const int64_t st = s.start(p);
    for (int64_t j = 0; j < s.npols(p); ++j) ipatch_id[st + j] = p + 1;
    disc_nodes(int(s.iptype[p]), int(s.norders[p]), uvs + 2 * st);
  }
}

namespace {
// |c - t|^2 <= r^2 with every product and sum rounded separately (no fused
// multiply-add), the same decision as the device near list makes.
bool within_radius(const double* c, const double* t, double r) {
  const double a = c[0] - t[0], b = c[1] - t[1], e = c[2] - t[2];
  volatile double a2 = a * a, b2 = b * b, e2 = e * e;
  volatile double s = a2 + b2;
  volatile double s2 = s + e2;
  volatile double r2 = r * r;
  return s2 <= r2;
}
}  // namespace

void findnear(int64_t npatches, const double* cms, const double* rads, int ndt, int64_t nt,
              const double* targs, std::vector<int64_t>& row_ptr, std::vector<int64_t>& col_ind) {
  // Bin patch centroids on a uniform grid of cell size >= max radius; a
  // target then only needs the 27 cells around its own.
  double rmax = 0, lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t j = 0; j < npatches; ++j) {
    rmax = std::max(rmax, rads[j]);
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], cms[3 * j + k]);
      hi[k] = std::max(hi[k], cms[3 * j + k]);
    }
  }
  double h = std::max(rmax, 1e-300);
  int64_t dims[3];
  for (int k = 0; k < 3; ++k) {
    dims[k] = std::max<int64_t>(1, int64_t((hi[k] - lo[k]) / h) + 1);
  }
  while (dims[0] * dims[1] * dims[2] > 8 * npatches + 64) {
    h *= 1.5;
    for (int k = 0; k < 3; ++k) dims[k] = std::max<int64_t>(1, int64_t((hi[k] - lo[k]) / h) + 1);
  }
  auto cell_of = [&](const double* x, int64_t* c) {
    for (int k = 0; k < 3; ++k) c[k] = int64_t(std::floor((x[k] - lo[k]) / h));
  };
  const int64_t ncell = dims[0] * dims[1] * dims[2];
  std::vector<int64_t> cstart(ncell + 1, 0), cidx(npatches);
  std::vector<int64_t> cellid(npatches);
  for (int64_t j = 0; j < npatches; ++j) {
    int64_t c[3];
    cell_of(cms + 3 * j, c);
    for (int k = 0; k < 3; ++k) c[k] = std::min(std::max<int64_t>(c[k], 0), dims[k] - 1);
    cellid[j] = (c[2] * dims[1] + c[1]) * dims[0] + c[0];
    cstart[cellid[j] + 1]++;
  }
  for (int64_t i = 0; i < ncell; ++i) cstart[i + 1] += cstart[i];
  {
    std::vector<int64_t> fill(cstart.begin(), cstart.end() - 1);
    for (int64_t j = 0; j < npatches; ++j) cidx[fill[cellid[j]]++] = j;
  }
  std::vector<std::vector<int64_t>> rows(nt);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < nt; ++i) {
    const double* t = targs + size_t(ndt) * i;
    int64_t c[3];
    cell_of(t, c);
    auto& row = rows[i];
    for (int64_t dz = -1; dz <= 1; ++dz)
      for (int64_t dy = -1; dy <= 1; ++dy)
        for (int64_t dx = -1; dx <= 1; ++dx) {
          const int64_t x = c[0] + dx, y = c[1] + dy, z = c[2] + dz;
          if (x < 0 || y < 0 || z < 0 || x >= dims[0] || y >= dims[1] || z >= dims[2]) continue;
          const int64_t cell = (z * dims[1] + y) * dims[0] + x;
          for (int64_t q = cstart[cell]; q < cstart[cell + 1]; ++q) {
            const int64_t j = cidx[q];
            if (within_radius(cms + 3 * j, t, rads[j])) row.push_back(j);
          }
        }
    std::sort(row.begin(), row.end());
  }
  row_ptr.assign(nt + 1, 1);
  for (int64_t i = 0; i < nt; ++i) row_ptr[i + 1] = row_ptr[i] + int64_t(rows[i].size());
  col_ind.resize(row_ptr[nt] - 1);
  for (int64_t i = 0; i < nt; ++i)
    for (size_t k = 0; k < rows[i].size(); ++k) col_ind[row_ptr[i] - 1 + k] = rows[i][k] + 1;
}

void iquad_rsc(const Surf& s, int64_t /*nt*/, int64_t nnz, const int64_t* /*row_ptr*/,
               const int64_t* col_ind, int64_t* iquad) {
  iquad[0] = 1;
  for (int64_t k = 0; k < nnz; ++k) iquad[k + 1] = iquad[k] + s.npols(col_ind[k] - 1);
}

void rsc_to_csc(int64_t ncol, int64_t nrow, int64_t nnz, const int64_t* row_ptr,
                const int64_t* col_ind, int64_t* col_ptr, int64_t* row_ind, int64_t* iper) {
  std::vector<int64_t> cnt(ncol + 1, 0);
  for (int64_t k = 0; k < nnz; ++k) cnt[col_ind[k]]++;
  col_ptr[0] = 1;
  for (int64_t j = 0; j < ncol; ++j) col_ptr[j + 1] = col_ptr[j] + cnt[j + 1];
  std::vector<int64_t> fill(col_ptr, col_ptr + ncol);
  for (int64_t i = 0; i < nrow; ++i)
    for (int64_t k = row_ptr[i] - 1; k < row_ptr[i + 1] - 1; ++k) {
      const int64_t j = col_ind[k] - 1;
      const int64_t pos = fill[j]++ - 1;
      row_ind[pos] = i + 1;
      iper[pos] = k + 1;
    }
}

double hkrand(int64_t iseed) {
  // LAPACK DLARAN: x <- a x mod 2^48 with a = 33952834046453, output
  // x/2^48 accumulated from the four base-4096 digits, most significant
  // first, exactly as the Fortran forms it.
  const uint64_t a = 33952834046453ull;
  const uint64_t mask = (1ull << 48) - 1;
  uint64_t x = uint64_t(((2 * iseed + 1) % 4096 + 4096) % 4096);
  double out;
  do {
    x = uint64_t(((unsigned __int128)x * a) & mask);
    const double r = 1.0 / 4096.0;
    const double d1 = double((x >> 36) & 4095), d2 = double((x >> 24) & 4095),
                 d3 = double((x >> 12) & 4095), d4 = double(x & 4095);
    out = r * (d1 + r * (d2 + r * (d3 + r * d4)));
  } while (out == 1.0);
  return out;
}

namespace {
inline cdouble kern_slp(const double* s, const double* t, cdouble zk) {
  const double dx = t[0] - s[0], dy = t[1] - s[1], dz = t[2] - s[2];
  const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
  return std::exp(cdouble(0, 1) * zk * r) / r * (0.25 / M_PI);
}
inline cdouble kern_dlp(const double* s, const double* t, cdouble zk) {
  const double dx = t[0] - s[0], dy = t[1] - s[1], dz = t[2] - s[2];
  const double d = dx * s[9] + dy * s[10] + dz * s[11];
  const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
  const cdouble ikr = cdouble(0, 1) * zk * r;
  return d * (1.0 - ikr) * std::exp(ikr) / (r * r * r) * (0.25 / M_PI);
}
}  // namespace

int far_order(double eps, const Surf& s, const double* cms, const double* rads, int ndt,
              int64_t nt, const double* targs, int ikerorder, cdouble zk, int64_t nnz,
              const int64_t* row_ptr, const int64_t* col_ind, double rfac, int64_t* nfars,
              int64_t* ixyzso) {
  std::vector<int64_t> col_ptr(s.npatches + 1), row_ind(nnz), iper(nnz);
  rsc_to_csc(s.npatches, nt, nnz, row_ptr, col_ind, col_ptr.data(), row_ind.data(), iper.data());
  static const int kOrders[10] = {1, 2, 3, 4, 6, 8, 10, 12, 14, 16};
  int err = 0;
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t p = 0; p < s.npatches; ++p) {
    const int ip = int(s.iptype[p]), no = int(s.norders[p]);
    const int np = int(s.npols(p));
    const double* sc = s.srccoefs + 9 * s.start(p);
    const double* cm = cms + 3 * p;
    const double rad0 = rfac * rads[p];
    // probe targets: the 10 farthest near targets, then points on the
    // sphere of radius rad0 from hkrand (far_field_routs.f90:300-330)
    const int64_t ntp = col_ptr[p + 1] - col_ptr[p];
    std::vector<std::pair<double, int64_t>> dd(ntp);
    for (int64_t q = 0; q < ntp; ++q) {
      const double* t = targs + size_t(ndt) * (row_ind[col_ptr[p] - 1 + q] - 1);
      dd[q] = {(t[0] - cm[0]) * (t[0] - cm[0]) + (t[1] - cm[1]) * (t[1] - cm[1]) +
                   (t[2] - cm[2]) * (t[2] - cm[2]),
               q};
    }
    std::stable_sort(dd.begin(), dd.end(),
                     [](const auto& a, const auto& b) { return a.first < b.first; });
    const int nmax = 25;
    const int i0 = int(std::min<int64_t>(10, ntp / 2));
    double tt[25][3];
    for (int i = 0; i < i0; ++i) {
      const double* t = targs + size_t(ndt) * (row_ind[col_ptr[p] - 1 + dd[ntp - 1 - i].second] - 1);
      for (int k = 0; k < 3; ++k) tt[i][k] = t[k];
    }
    for (int i = i0; i < nmax; ++i) {
      const double ph = hkrand(1001 + i + 1) * 2 * M_PI;
      const double th = hkrand(3042 + i + 1) * M_PI;
      tt[i][0] = cm[0] + rad0 * std::sin(th) * std::cos(ph);
      tt[i][1] = cm[1] + rad0 * std::sin(th) * std::sin(ph);
      tt[i][2] = cm[2] + rad0 * std::cos(th);
    }
    // epsp = eps * (min |du x dv|^2)^(1/4) over the discretisation nodes
    std::vector<double> uvs(2 * 289), w(289), pm(size_t(np) * 289), pl(np);
    disc_nodes(ip, no, uvs.data());
    double rsc = 1e300;
    for (int j = 0; j < np; ++j) {
      basis_pols(ip, no, uvs[2 * j], uvs[2 * j + 1], pl.data());
      double g[9] = {0};
      for (int l = 0; l < np; ++l)
        for (int k = 0; k < 9; ++k) g[k] += sc[9 * l + k] * pl[l];
      double n[3];
      cross3(g + 3, g + 6, n);
      rsc = std::min(rsc, n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    }
    const double epsp = std::pow(rsc, 0.25) * eps;
    auto integrals = [&](int nfar, std::vector<cdouble>& v) {
      const int nf = npols_of(ip, nfar);
      disc_nodes(ip, nfar, uvs.data());
      disc_wts(ip, nfar, w.data());
      v.assign(size_t(np) * nmax, 0.0);
      for (int j = 0; j < nf; ++j) {
        basis_pols(ip, no, uvs[2 * j], uvs[2 * j + 1], pl.data());
        double src[12] = {0};
        for (int l = 0; l < np; ++l)
          for (int k = 0; k < 9; ++k) src[k] += sc[9 * l + k] * pl[l];
        double n[3];
        cross3(src + 3, src + 6, n);
        const double rr = norm3(n);
        for (int k = 0; k < 3; ++k) src[9 + k] = n[k] / rr;
        const double qw = w[j] * rr;
        for (int it = 0; it < nmax; ++it) {
          const cdouble val =
              (ikerorder == -1 ? kern_slp(src, tt[it], zk) : kern_dlp(src, tt[it], zk)) * qw;
          for (int l = 0; l < np; ++l) v[size_t(it) * np + l] += val * pl[l];
        }
      }
    };
    std::vector<cdouble> vcomp, vref;
    integrals(kOrders[0], vcomp);
    int nnn = 1;
    for (; nnn < 10; ++nnn) {
      integrals(kOrders[nnn], vref);
      double errmax = 0;
      for (int it = 0; it < nmax; ++it) {
        double e2 = 0;
        for (int l = 0; l < np; ++l) e2 += std::norm(vref[size_t(it) * np + l] - vcomp[size_t(it) * np + l]);
        errmax = std::max(errmax, std::sqrt(e2));
      }
      if (errmax < epsp) break;
      vcomp.swap(vref);
    }
    // The loop stops at the first order whose successor agrees to epsp;
    // if none does, the largest order is used.
    nfars[p] = kOrders[nnn - 1 < 0 ? 0 : nnn - 1];
    if (nnn == 10) nfars[p] = kOrders[9];
    if (npols_of(ip, int(nfars[p])) > 289) err = 1;
  }
  ixyzso[0] = 1;
  for (int64_t p = 0; p < s.npatches; ++p)
    ixyzso[p + 1] = ixyzso[p] + npols_of(int(s.iptype[p]), int(nfars[p]));
  return err;
}

int oversample_geom(const Surf& s, const int64_t* nfars, const int64_t* ixyzso, int64_t /*nptso*/,
                    double* srcover) {
  int err = 0;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t p = 0; p < s.npatches; ++p) {
    const int ip = int(s.iptype[p]), no = int(s.norders[p]), nfar = int(nfars[p]);
    const int np = int(s.npols(p));
    const int nf = npols_of(ip, nfar);
    if (nf != ixyzso[p + 1] - ixyzso[p]) {
      err = 1;
      continue;
    }
    const int64_t st = s.start(p), so = ixyzso[p] - 1;
    if (nfar == no) {
      for (int j = 0; j < np; ++j)
        for (int k = 0; k < 12; ++k) srcover[12 * (so + j) + k] = s.srcvals[12 * (st + j) + k];
      continue;
    }
    std::vector<double> uvs(2 * nf), pl(np);
    disc_nodes(ip, nfar, uvs.data());
    const double* sc = s.srccoefs + 9 * st;
    for (int j = 0; j < nf; ++j) {
      basis_pols(ip, no, uvs[2 * j], uvs[2 * j + 1], pl.data());
      double* o = srcover + 12 * (so + j);
      for (int k = 0; k < 9; ++k) {
        double acc = 0;
        for (int l = 0; l < np; ++l) acc += sc[9 * l + k] * pl[l];
        o[k] = acc;
      }
      finish_normal(o);
    }
    std::vector<int> ic(std::max(np, nf)), icf(ic.size());
    const int nclash = clashing_indices(ip, no, nfar, ic.data(), icf.data());
    for (int c = 0; c < nclash; ++c)
      for (int k = 0; k < 12; ++k) srcover[12 * (so + icf[c]) + k] = s.srcvals[12 * (st + ic[c]) + k];
  }
  return err;
}

int oversample_fun(const Surf& s, int nd, const double* u, const int64_t* nfars,
                   const int64_t* ixyzso, int64_t /*nptso*/, double* uover) {
  std::map<std::array<int, 3>, std::vector<double>> mats;
  for (int64_t p = 0; p < s.npatches; ++p) {
    std::array<int, 3> key{int(s.iptype[p]), int(s.norders[p]), int(nfars[p])};
    if (!mats.count(key)) {
      std::vector<double> m;
      const int ier = interp_matrix(key[0], key[1], key[2], m);
      if (ier) return ier;
      mats[key] = m;
    }
  }
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < s.npatches; ++p) {
    const auto& m = mats.at({int(s.iptype[p]), int(s.norders[p]), int(nfars[p])});
    const int np = int(s.npols(p));
    const int nf = int(ixyzso[p + 1] - ixyzso[p]);
    const int64_t st = s.start(p), so = ixyzso[p] - 1;
    for (int i = 0; i < nf; ++i)
      for (int d = 0; d < nd; ++d) {
        double acc = 0;
        for (int j = 0; j < np; ++j) acc += m[size_t(i) * np + j] * u[nd * (st + j) + d];
        uover[nd * (so + i) + d] = acc;
      }
  }
  return 0;
}

}  // namespace bie
