// Cluster trees, proxy grids, dual traversal and the flattened interaction
// lists of the hierarchical far field (see tree.h).
#include "tree.h"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace bie {
namespace tree {

void cheb_nodes(int p, double* x, double* w) {
  if (p <= 1) {
    x[0] = 0.0;
    w[0] = 1.0;
    return;
  }
  for (int j = 0; j < p; ++j) x[j] = std::cos(M_PI * j / (p - 1));
  for (int j = 0; j < p; ++j) {
    double d = 1.0;
    for (int i = 0; i < p; ++i)
      if (i != j) d *= x[j] - x[i];
    w[j] = 1.0 / d;
  }
}

void build_tree(int64_t n, const double* x, const double* y, const double* z, int leaf, Tree& t) {
  // points with their original index, kept contiguous per node while the
  // nodes of one level are split in parallel
  struct Pt {
    double v[3];
    int64_t id;
  };
  std::vector<Pt> pts(static_cast<size_t>(n));
  for (int64_t q = 0; q < n; ++q) pts[q] = {{x[q], y[q], z[q]}, q};
  t.nodes.clear();
  Node root;
  root.b = 0;
  root.e = n;
  t.nodes.push_back(root);
  size_t lev0 = 0, lev1 = 1;  // nodes of the current level
  std::vector<int64_t> split;
  while (lev0 < lev1) {
    const int64_t cnt = int64_t(lev1 - lev0);
    split.assign(static_cast<size_t>(cnt), 0);
#pragma omp parallel for schedule(dynamic, 1) if (cnt > 1)
    for (int64_t i = 0; i < cnt; ++i) {
      Node& nd = t.nodes[lev0 + i];
      const int64_t m = nd.n();
      for (int d = 0; d < 3; ++d) {
        nd.lo[d] = m > 0 ? 1e300 : 0.0;
        nd.hi[d] = m > 0 ? -1e300 : 0.0;
      }
      for (int64_t q = nd.b; q < nd.e; ++q)
        for (int d = 0; d < 3; ++d) {
          nd.lo[d] = std::min(nd.lo[d], pts[q].v[d]);
          nd.hi[d] = std::max(nd.hi[d], pts[q].v[d]);
        }
      double r2 = 0.0, ext[3];
      for (int d = 0; d < 3; ++d) {
        nd.c[d] = 0.5 * (nd.lo[d] + nd.hi[d]);
        ext[d] = nd.hi[d] - nd.lo[d];
        r2 += 0.25 * ext[d] * ext[d];
      }
      nd.r = std::sqrt(r2);
      const int d = ext[0] >= ext[1] ? (ext[0] >= ext[2] ? 0 : 2) : (ext[1] >= ext[2] ? 1 : 2);
      if (m > leaf && ext[d] > 0.0) {
        // two children split at a multiple of 32 points near the median
        // along the longest side, so that leaves hold leaf/2 .. leaf points
        // and fill whole warps
        int64_t k = ((m / 2 + 16) / 32) * 32;
        k = std::min<int64_t>(std::max<int64_t>(k, std::min<int64_t>(32, m - 1)), m - 1);
        auto first = pts.begin() + nd.b;
        std::nth_element(first, first + k, first + m,
                         [d](const Pt& a, const Pt& b) { return a.v[d] < b.v[d]; });
        split[i] = k;
      }
    }
    // children of this level, appended in order (siblings contiguous)
    const size_t next0 = t.nodes.size();
    for (int64_t i = 0; i < cnt; ++i) {
      if (split[i] == 0) continue;
      const size_t pi = lev0 + i;
      t.nodes[pi].child0 = int(t.nodes.size());
      t.nodes[pi].nchild = 2;
      for (int cc = 0; cc < 2; ++cc) {
        Node ch;
        ch.b = cc == 0 ? t.nodes[pi].b : t.nodes[pi].b + split[i];
        ch.e = cc == 0 ? t.nodes[pi].b + split[i] : t.nodes[pi].e;
        ch.parent = int(pi);
        ch.level = t.nodes[pi].level + 1;
        t.nodes.push_back(ch);
      }
    }
    lev0 = next0;
    lev1 = t.nodes.size();
  }
  t.perm.resize(static_cast<size_t>(n));
  for (int64_t q = 0; q < n; ++q) t.perm[q] = pts[q].id;
}

void set_proxies(Tree& t, const Params& prm) {
  for (Node& nd : t.nodes) {
    nd.np[0] = nd.np[1] = nd.np[2] = 0;
    nd.capped = false;
    if (nd.n() <= 1) continue;
    double ext[3], emax = 0.0;
    for (int d = 0; d < 3; ++d) {
      ext[d] = nd.hi[d] - nd.lo[d];
      emax = std::max(emax, ext[d]);
    }
    int np[3];
    if (emax <= 0.0) {
      np[0] = np[1] = np[2] = 1;  // coincident points: one proxy is exact
    } else {
      // Bernstein-ellipse parameter of a side for a singularity at distance
      // r / theta from the centre: rho = a + sqrt(a^2 - 1), a = 2 D / side
      const double D = nd.r / prm.theta;
      auto rho = [&](double side) {
        const double a = std::max(2.0 * D / side, 1.0 + 1e-12);
        return a + std::sqrt(a * a - 1.0);
      };
      const double lmax = std::log(rho(emax));
      for (int d = 0; d < 3; ++d) {
        int pd = 1;
        if (ext[d] > 1e-12 * emax) {
          pd = int(std::ceil(prm.p * lmax / std::log(rho(ext[d])) - 1e-9));
          pd += int(std::ceil(prm.kscale * prm.k * 0.5 * ext[d] - 1e-9));
        }
        np[d] = std::max(pd, 1);
      }
      // a grid the caps cannot hold would miss the accuracy: no proxies,
      // and the traversal splits the node instead of accepting its pairs
      if (np[0] > kMaxP || np[1] > kMaxP || np[2] > kMaxP ||
          int64_t(np[0]) * np[1] * np[2] > kMaxProxies) {
        nd.capped = true;
        continue;
      }
    }
    if (int64_t(np[0]) * np[1] * np[2] >= nd.n()) continue;
    for (int d = 0; d < 3; ++d) nd.np[d] = np[d];
  }
}

void traverse(const Tree& T, const Tree& S, const Params& prm, double sep_min,
              std::vector<Interaction>& out) {
  out.clear();
  if (T.nodes.empty() || S.nodes.empty() || T.nodes[0].n() == 0 || S.nodes[0].n() == 0) return;
  std::vector<std::pair<int, int>> stack{{0, 0}};
  while (!stack.empty()) {
    const auto [a, b] = stack.back();
    stack.pop_back();
    const Node& t = T.nodes[a];
    const Node& s = S.nodes[b];
    double d2 = 0.0;
    for (int d = 0; d < 3; ++d) d2 += (t.c[d] - s.c[d]) * (t.c[d] - s.c[d]);
    const double D = std::sqrt(d2);
    const bool tleaf = t.nchild == 0, sleaf = s.nchild == 0;
    // a pair with a node too large for an accurate grid is split further
    const bool split_capped = (t.capped && !tleaf) || (s.capped && !sleaf);
    if (t.r + s.r < prm.theta * D && !split_capped) {
      const double nt = double(t.n()), ns = double(s.n());
      const double pt = t.nprox(), ps = s.nprox();
      double best = nt * ns;
      int kind = D - t.r - s.r > sep_min ? kPP : kPPCheck;
      if (ps > 0 && nt * ps < best) {
        best = nt * ps;
        kind = kPC;
      }
      if (pt > 0 && pt * ns < best) {
        best = pt * ns;
        kind = kCP;
      }
      if (pt > 0 && ps > 0 && pt * ps < best) {
        best = pt * ps;
        kind = kCC;
      }
      out.push_back({a, b, kind});
      continue;
    }
    if (tleaf && sleaf) {
      out.push_back({a, b, kPPCheck});
    } else if (split_capped) {
      if (t.capped && !tleaf && (!s.capped || sleaf || t.r >= s.r)) {
        for (int c = 0; c < t.nchild; ++c) stack.push_back({t.child0 + c, b});
      } else {
        for (int c = 0; c < s.nchild; ++c) stack.push_back({a, s.child0 + c});
      }
    } else if (sleaf || (!tleaf && t.r >= s.r)) {
      for (int c = 0; c < t.nchild; ++c) stack.push_back({t.child0 + c, b});
    } else {
      for (int c = 0; c < s.nchild; ++c) stack.push_back({a, s.child0 + c});
    }
  }
}

namespace {
void leaves_under(const Tree& t, int a, std::vector<int>& out) {
  const Node& nd = t.nodes[a];
  if (nd.nchild == 0) {
    out.push_back(a);
    return;
  }
  for (int c = 0; c < nd.nchild; ++c) leaves_under(t, nd.child0 + c, out);
}
}  // namespace

int check_coverage(const Tree& T, const Tree& S, const std::vector<Interaction>& ia) {
  std::vector<int> tl, sl;
  leaves_under(T, 0, tl);
  leaves_under(S, 0, sl);
  std::vector<int> tid(T.nodes.size(), -1), sid(S.nodes.size(), -1);
  for (size_t i = 0; i < tl.size(); ++i) tid[tl[i]] = int(i);
  for (size_t i = 0; i < sl.size(); ++i) sid[sl[i]] = int(i);
  std::vector<int> cnt(tl.size() * sl.size(), 0);
  std::vector<int> a, b;
  for (const auto& x : ia) {
    a.clear();
    b.clear();
    leaves_under(T, x.t, a);
    leaves_under(S, x.s, b);
    for (int u : a)
      for (int v : b) ++cnt[size_t(tid[u]) * sl.size() + sid[v]];
  }
  int bad = 0;
  for (size_t i = 0; i < tl.size(); ++i)
    for (size_t j = 0; j < sl.size(); ++j) {
      const bool empty = T.nodes[tl[i]].n() == 0 || S.nodes[sl[j]].n() == 0;
      if (!empty && cnt[i * sl.size() + j] != 1) ++bad;
    }
  return bad;
}

}  // namespace tree
}  // namespace bie
