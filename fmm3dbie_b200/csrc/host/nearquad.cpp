// Near-field quadrature generator (see nearquad.h).
#include "nearquad.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "basis.h"

namespace bie {

namespace {

constexpr double kOver4Pi = 0.07957747154594767;

// Combined-field kernels (lap_kernels.f90:123-165 l3d_comb,
// helm_kernels.f90:120-162 h3d_comb): y = source point, n = source normal,
// x = target.
struct LapComb {
  using T = double;
  double alpha, beta;
  T operator()(const double* y, const double* n, const double* x) const {
    const double dx = x[0] - y[0], dy = x[1] - y[1], dz = x[2] - y[2];
    const double d = dx * n[0] + dy * n[1] + dz * n[2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double r = std::sqrt(r2);
    return (beta * d / (r2 * r) + alpha / r) * kOver4Pi;
  }
};

struct HelmComb {
  using T = cdouble;
  cdouble zk, alpha, beta;
  T operator()(const double* y, const double* n, const double* x) const {
    const double dx = x[0] - y[0], dy = x[1] - y[1], dz = x[2] - y[2];
    const double d = dx * n[0] + dy * n[1] + dz * n[2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double r = std::sqrt(r2);
    const cdouble ikr = cdouble(-zk.imag() * r, zk.real() * r);
    const cdouble e = std::exp(ikr);
    return (beta * d * (1.0 - ikr) / (r2 * r) + alpha / r) * e * kOver4Pi;
  }
};

inline double absval(double v) { return std::fabs(v); }
inline double absval(const cdouble& v) { return std::abs(v); }

struct PatchGeom {
  int ip = 1, no = 0, np = 0;
  const double* sc = nullptr;
  // pols[np]; g: xyz(3), du(3), dv(3); returns |du x dv|, writes normal.
  double eval(double u, double v, double* pols, double* xyz, double* nrm, double* du = nullptr,
              double* dv = nullptr) const {
    basis_pols(ip, no, u, v, pols);
    double g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int l = 0; l < np; ++l) {
      const double p = pols[l];
      const double* c = sc + 9 * l;
      for (int k = 0; k < 9; ++k) g[k] += c[k] * p;
    }
    for (int k = 0; k < 3; ++k) xyz[k] = g[k];
    if (du)
      for (int k = 0; k < 3; ++k) du[k] = g[3 + k];
    if (dv)
      for (int k = 0; k < 3; ++k) dv[k] = g[6 + k];
    const double n0 = g[4] * g[8] - g[5] * g[7];
    const double n1 = g[5] * g[6] - g[3] * g[8];
    const double n2 = g[3] * g[7] - g[4] * g[6];
    const double jn = std::sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    nrm[0] = n0 / jn;
    nrm[1] = n1 / jn;
    nrm[2] = n2 / jn;
    return jn;
  }
};

// Collapsed Gauss-Legendre rule on the simplex (0,0),(1,0),(0,1); weights
// sum to 1/2.
struct TriRule {
  int nq = 0;
  std::vector<double> xi, eta, w;
};

TriRule make_tri_rule(int ng) {
  TriRule r;
  r.nq = ng * ng;
  nearquad_tri_rule(ng, r.xi, r.eta, r.w);
  return r;
}

// Lazily refined tree of sub-triangles of one patch's parameter domain,
// caching geometry and basis values at the rule's nodes so every target
// of the patch reuses them.
class PatchTree {
 public:
  struct Node {
    double v[6];
    int child = -1;
    int64_t off = 0;  // node index into cache arrays (times nq)
  };
  PatchTree(const PatchGeom& g, const TriRule& rule) : g_(g), rule_(rule) {
    double uv[8];
    const int nv = boundary_vertices(g.ip, uv);
    if (nv == 3) {
      roots_.push_back(add(uv));
    } else {
      const double t1[6] = {uv[0], uv[1], uv[2], uv[3], uv[4], uv[5]};
      const double t2[6] = {uv[0], uv[1], uv[4], uv[5], uv[6], uv[7]};
      roots_.push_back(add(t1));
      roots_.push_back(add(t2));
    }
  }
  const std::vector<int>& roots() const { return roots_; }
  int children(int idx) {
    if (nodes_[idx].child < 0) {
      const double* v = nodes_[idx].v;
      const double m01[2] = {0.5 * (v[0] + v[2]), 0.5 * (v[1] + v[3])};
      const double m12[2] = {0.5 * (v[2] + v[4]), 0.5 * (v[3] + v[5])};
      const double m20[2] = {0.5 * (v[4] + v[0]), 0.5 * (v[5] + v[1])};
      const double c0[6] = {v[0], v[1], m01[0], m01[1], m20[0], m20[1]};
      const double c1[6] = {m01[0], m01[1], v[2], v[3], m12[0], m12[1]};
      const double c2[6] = {m20[0], m20[1], m12[0], m12[1], v[4], v[5]};
      const double c3[6] = {m01[0], m01[1], m12[0], m12[1], m20[0], m20[1]};
      const int first = add(c0);
      add(c1);
      add(c2);
      add(c3);
      nodes_[idx].child = first;
    }
    return nodes_[idx].child;
  }
  // integral over node idx of ker(y, n, x) * basis_l
  template <class K, class T>
  void integrate(int idx, const K& ker, const double* x, T* res) const {
    const int np = g_.np, nq = rule_.nq;
    for (int l = 0; l < np; ++l) res[l] = T(0);
    const int64_t off = nodes_[idx].off;
    for (int q = 0; q < nq; ++q) {
      const double* ge = geo_.data() + 7 * (off + q);
      const T kv = ker(ge, ge + 3, x) * ge[6];
      const double* b = bas_.data() + size_t(off + q) * np;
      for (int l = 0; l < np; ++l) res[l] += kv * b[l];
    }
  }
  size_t size() const { return nodes_.size(); }

 private:
  int add(const double* v6) {
    Node nd;
    std::memcpy(nd.v, v6, sizeof nd.v);
    nd.off = int64_t(nodes_.size()) * rule_.nq;
    const int np = g_.np, nq = rule_.nq;
    geo_.resize(geo_.size() + 7 * size_t(nq));
    bas_.resize(bas_.size() + size_t(nq) * np);
    const double ax = v6[2] - v6[0], ay = v6[3] - v6[1];
    const double bx = v6[4] - v6[0], by = v6[5] - v6[1];
    const double area2 = std::fabs(ax * by - ay * bx);  // 2 x area = jacobian vs simplex
    for (int q = 0; q < nq; ++q) {
      const double u = v6[0] + rule_.xi[q] * ax + rule_.eta[q] * bx;
      const double v = v6[1] + rule_.xi[q] * ay + rule_.eta[q] * by;
      double* ge = geo_.data() + 7 * (nd.off + q);
      double* b = bas_.data() + size_t(nd.off + q) * np;
      const double jn = g_.eval(u, v, b, ge, ge + 3);
      ge[6] = jn * rule_.w[q] * area2;
    }
    nodes_.push_back(nd);
    return int(nodes_.size()) - 1;
  }
  const PatchGeom& g_;
  const TriRule& rule_;
  std::vector<Node> nodes_;
  std::vector<int> roots_;
  std::vector<double> geo_;  // per rule node: xyz(3), normal(3), weight
  std::vector<double> bas_;  // per rule node: basis values
};

template <class K, class T>
int64_t adaptive_integral(PatchTree& tree, const K& ker, const double* x, double tol, int np,
                          T* out, std::vector<T>& work) {
  constexpr int kMaxLevel = 18;
  struct Item {
    int idx, lev;
    int64_t slot;
  };
  std::vector<Item> stack;
  int64_t nslots = 0;
  auto slot = [&](int64_t s) { return work.data() + size_t(s) * np; };
  auto alloc = [&]() {
    if (size_t(nslots + 1) * np > work.size()) work.resize(size_t(nslots + 1) * np * 2);
    return nslots++;
  };
  for (int l = 0; l < np; ++l) out[l] = T(0);
  int64_t nev = 0;
  std::vector<int64_t> free_slots;
  auto get = [&]() -> int64_t {
    if (!free_slots.empty()) {
      const int64_t s = free_slots.back();
      free_slots.pop_back();
      return s;
    }
    return alloc();
  };
  for (int r : tree.roots()) {
    const int64_t s = get();
    tree.integrate(r, ker, x, slot(s));
    stack.push_back({r, 0, s});
    nev++;
  }
  std::vector<T> sum(np);
  while (!stack.empty()) {
    const Item it = stack.back();
    stack.pop_back();
    const int c0 = tree.children(it.idx);
    int64_t cs[4];
    for (int c = 0; c < 4; ++c) {
      cs[c] = get();
      tree.integrate(c0 + c, ker, x, slot(cs[c]));
    }
    nev += 4;
    double err = 0;
    const T* par = slot(it.slot);
    for (int l = 0; l < np; ++l) {
      sum[l] = slot(cs[0])[l] + slot(cs[1])[l] + slot(cs[2])[l] + slot(cs[3])[l];
      err = std::max(err, absval(sum[l] - par[l]));
    }
    free_slots.push_back(it.slot);
    if (err <= tol || it.lev >= kMaxLevel) {
      for (int l = 0; l < np; ++l) out[l] += sum[l];
      for (int c = 0; c < 4; ++c) free_slots.push_back(cs[c]);
    } else {
      for (int c = 0; c < 4; ++c) stack.push_back({c0 + c, it.lev + 1, cs[c]});
    }
  }
  return nev;
}

// Singular integral for a target at parameter point (u0,v0) of the patch.
template <class K, class T>
int64_t self_integral(const PatchGeom& g, const K& ker, double u0, double v0, int ns, int nw,
                      const std::vector<double>& xs, const std::vector<double>& ws,
                      const std::vector<double>& xw, const std::vector<double>& www, T* out) {
  const int np = g.np;
  std::vector<double> pols(np);
  double x0[3], n0[3], du[3], dv[3];
  g.eval(u0, v0, pols.data(), x0, n0, du, dv);
  const double g11 = du[0] * du[0] + du[1] * du[1] + du[2] * du[2];
  const double g12 = du[0] * dv[0] + du[1] * dv[1] + du[2] * dv[2];
  const double g22 = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
  auto gdot = [&](double ax, double ay, double bx, double by) {
    return ax * (g11 * bx + g12 * by) + ay * (g12 * bx + g22 * by);
  };
  double V[8];
  const int nv = boundary_vertices(g.ip, V);
  for (int l = 0; l < np; ++l) out[l] = T(0);
  int64_t nev = 0;
  for (int e = 0; e < nv; ++e) {
    const double ax = V[2 * e], ay = V[2 * e + 1];
    const double bx = V[2 * ((e + 1) % nv)], by = V[2 * ((e + 1) % nv) + 1];
    const double dx = bx - ax, dy = by - ay;
    const double tau = gdot(u0 - ax, v0 - ay, dx, dy) / gdot(dx, dy, dx, dy);
    double P[2][2], Q[2][2];
    int nsub = 0;
    if (tau <= 0.0) {
      P[0][0] = ax, P[0][1] = ay, Q[0][0] = bx, Q[0][1] = by, nsub = 1;
    } else if (tau >= 1.0) {
      P[0][0] = bx, P[0][1] = by, Q[0][0] = ax, Q[0][1] = ay, nsub = 1;
    } else {
      const double fx = ax + tau * dx, fy = ay + tau * dy;
      P[0][0] = fx, P[0][1] = fy, Q[0][0] = ax, Q[0][1] = ay;
      P[1][0] = fx, P[1][1] = fy, Q[1][0] = bx, Q[1][1] = by;
      nsub = 2;
    }
    for (int sbt = 0; sbt < nsub; ++sbt) {
      const double a0 = P[sbt][0] - u0, a1 = P[sbt][1] - v0;
      const double b0 = Q[sbt][0] - P[sbt][0], b1 = Q[sbt][1] - P[sbt][1];
      const double det = std::fabs(a0 * b1 - a1 * b0);
      if (det <= 1e-300) continue;
      const double h = std::sqrt(gdot(a0, a1, a0, a1));
      const double L = std::sqrt(gdot(b0, b1, b0, b1));
      const double W = std::asinh(L / h);
      for (int iw = 0; iw < nw; ++iw) {
        const double w = 0.5 * W * (xw[iw] + 1.0);
        const double t = (h / L) * std::sinh(w);
        const double dtw = (h / L) * std::cosh(w) * 0.5 * W * www[iw];
        const double ex = a0 + t * b0, ey = a1 + t * b1;
        for (int is = 0; is < ns; ++is) {
          const double s = 0.5 * (xs[is] + 1.0);
          const double jac = s * det * dtw * 0.5 * ws[is];
          double y[3], ny[3];
          const double jn = g.eval(u0 + s * ex, v0 + s * ey, pols.data(), y, ny);
          const T kv = ker(y, ny, x0) * (jn * jac);
          for (int l = 0; l < np; ++l) out[l] += kv * pols[l];
          ++nev;
        }
      }
    }
  }
  return nev;
}

template <class K>
int run(const K& ker, const Surf& s, int ndt, int64_t nt, const double* targs,
        const int64_t* ipatch_id, const double* uvs_targ, double eps, int64_t nnz,
        const int64_t* row_ptr, const int64_t* col_ind, const int64_t* iquad, double* wre,
        double* wim, NearQuadStats* stats) {
  using T = typename K::T;
  std::vector<int64_t> col_ptr(s.npatches + 1), row_ind(nnz), iper(nnz);
  rsc_to_csc(s.npatches, nt, nnz, row_ptr, col_ind, col_ptr.data(), row_ind.data(), iper.data());
  // rule sizes from the requested tolerance
  const int nself = nearquad_self_order(eps);
  std::vector<double> xs(nself), ws(nself);
  gauss_legendre(nself, xs.data(), ws.data());
  std::map<int, TriRule> rules;
  for (int64_t p = 0; p < s.npatches; ++p) {
    const int no = int(s.norders[p]);
    const int ng = nearquad_tri_ng(no);
    if (!rules.count(ng)) rules[ng] = make_tri_rule(ng);
  }
  std::atomic<int64_t> nev_total{0}, nself_total{0}, nnear_total{0};
  std::atomic<int> err{0};
#pragma omp parallel
  {
    std::vector<T> work, sints, row;
#pragma omp for schedule(dynamic, 1)
    for (int64_t p = 0; p < s.npatches; ++p) {
      PatchGeom g;
      g.ip = int(s.iptype[p]);
      g.no = int(s.norders[p]);
      g.np = int(s.npols(p));
      g.sc = s.srccoefs + 9 * s.start(p);
      const int np = g.np;
      if (npols_of(g.ip, g.no) != np) {
        err = 1;
        continue;
      }
      std::vector<double> uvs(2 * np), umat(np * np), vmat(np * np), w(np);
      if (disc_exps(g.ip, g.no, uvs.data(), umat.data(), vmat.data(), w.data())) {
        err = 6;
        continue;
      }
      // tolerance scaled by the patch size: eps * 0.1 * sqrt(min |J| w)
      double jwmin = 1e300;
      {
        std::vector<double> pl(np);
        for (int j = 0; j < np; ++j) {
          double xyz[3], n[3];
          const double jn = g.eval(uvs[2 * j], uvs[2 * j + 1], pl.data(), xyz, n);
          jwmin = std::min(jwmin, jn * w[j]);
        }
      }
      const double tol = 0.1 * eps * std::sqrt(jwmin);
      const int ng = nearquad_tri_ng(g.no);
      PatchTree tree(g, rules.at(ng));
      sints.resize(np);
      row.resize(np);
      int64_t nev = 0, nsf = 0, nnr = 0;
      for (int64_t q = col_ptr[p] - 1; q < col_ptr[p + 1] - 1; ++q) {
        const int64_t it = row_ind[q] - 1;
        const int64_t k = iper[q] - 1;
        const double* x = targs + size_t(ndt) * it;
        if (ipatch_id && ipatch_id[it] == p + 1) {
          nev += self_integral(g, ker, uvs_targ[2 * it], uvs_targ[2 * it + 1], nself, nself, xs, ws,
                               xs, ws, sints.data());
          ++nsf;
        } else {
          nev += adaptive_integral(tree, ker, x, tol, np, sints.data(), work) * rules.at(ng).nq;
          ++nnr;
        }
        for (int j = 0; j < np; ++j) {
          T acc = T(0);
          for (int l = 0; l < np; ++l) acc += sints[l] * umat[l * np + j];
          row[j] = acc;
        }
        const int64_t base = iquad[k] - 1;
        for (int j = 0; j < np; ++j) {
          if constexpr (std::is_same_v<T, double>) {
            wre[base + j] = row[j];
            if (wim) wim[base + j] = 0.0;
          } else {
            wre[base + j] = row[j].real();
            if (wim) wim[base + j] = row[j].imag();
          }
        }
      }
      nev_total += nev;
      nself_total += nsf;
      nnear_total += nnr;
    }
  }
  if (stats) {
    stats->kernel_evals = nev_total;
    stats->self_targets = nself_total;
    stats->near_targets = nnear_total;
  }
  return err;
}

}  // namespace

int nearquad_tri_ng(int norder) { return norder <= 6 ? 8 : (norder <= 10 ? 10 : 12); }

int nearquad_self_order(double eps) {
  const double digits = std::max(1.0, -std::log10(std::max(eps, 1e-15)));
  return std::min(40, std::max(12, int(std::ceil(2.2 * digits)) + 4));
}

void nearquad_tri_rule(int ng, std::vector<double>& xi, std::vector<double>& eta,
                       std::vector<double>& w) {
  std::vector<double> x(ng), wg(ng);
  gauss_legendre(ng, x.data(), wg.data());
  xi.clear();
  eta.clear();
  w.clear();
  for (int i = 0; i < ng; ++i)
    for (int j = 0; j < ng; ++j) {
      const double a = 0.5 * (x[i] + 1.0), wa = 0.5 * wg[i];
      const double b = 0.5 * (x[j] + 1.0), wb = 0.5 * wg[j];
      xi.push_back(a);
      eta.push_back(b * (1.0 - a));
      w.push_back(wa * wb * (1.0 - a));
    }
}

int getnearquad(const Surf& s, int ndt, int64_t nt, const double* targs, const int64_t* ipatch_id,
                const double* uvs_targ, double eps, int kind, cdouble zk, cdouble alpha,
                cdouble beta, int64_t nnz, const int64_t* row_ptr, const int64_t* col_ind,
                const int64_t* iquad, double /*rfac0*/, int64_t nquad, double* wnear_re,
                double* wnear_im, NearQuadStats* stats) {
  if (nnz > 0 && iquad[nnz] - 1 != nquad) return 1;
  if (kind == 0) {
    LapComb k{alpha.real(), beta.real()};
    return run(k, s, ndt, nt, targs, ipatch_id, uvs_targ, eps, nnz, row_ptr, col_ind, iquad,
               wnear_re, wnear_im, stats);
  }
  HelmComb k{zk, alpha, beta};
  return run(k, s, ndt, nt, targs, ipatch_id, uvs_targ, eps, nnz, row_ptr, col_ind, iquad,
             wnear_re, wnear_im, stats);
}

}  // namespace bie
