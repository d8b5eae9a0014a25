// Hierarchical far field on the device: the dual-tree barycentric Lagrange
// method of host/tree.h with its lists in HBM and four launches per matvec
// (upward pass, its chunk reduction, proxy-target lists, leaf lists with the
// downward pass).  It replaces the O(ntarg * nptso) direct far kernels for
// large surfaces; its result feeds the same combine kernel (one chunk of
// partial potentials in the original target order).
#pragma once
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "../host/tree.h"
#include "device.cuh"
#include "plan.h"

namespace bie {

struct TreeStats {
  int64_t tnodes = 0, snodes = 0, leaves = 0, proxy_items = 0, up_items = 0;
  int64_t interactions[5] = {0, 0, 0, 0, 0};  // by tree::Kind
  double pair_evals = 0;                        // kernel evaluations per density
  double up_evals = 0, down_evals = 0;          // basis-weighted terms per density
  int64_t source_proxies = 0, target_proxies = 0;
  double build_ms = 0;
};

class TreeFar {
 public:
  // Builds the trees and lists for the plan's targets and oversampled
  // sources (read back from the device geometry).  Accepted particle pairs
  // closer than thresh plus 2^-12 of the coordinates' extent (a margin far
  // above the FP32 rounding of centred coordinates) keep the
  // self-interaction test r >= thresh.
  // kp and precision (optional, with g.sw set): also keep the per-source
  // constants (alpha w_s/(4 pi), beta w_s/(4 pi)) in tree order and that
  // precision, for several densities at once.
  int build(const dev::Geometry& g, const tree::Params& prm, double thresh, cudaStream_t st,
            const dev::KParams* kp = nullptr, int precision = 0);
  // Far field into partial[(i * nd + m) * C] at original target index i.
  // nd = 1: from per-source (charge, dipole) strengths in tree order
  // (str_sorted[(s * nd + m) * SW], SW = 4 Helmholtz / 2 Laplace, far
  // precision).  nd >= 2: from the oversampled densities in tree order
  // (sig_sorted[(s * nd + m) * C], C = 2 / 1) and the constants kept by
  // build (which then needs kp and this precision).
  cudaError_t run(int precision, int nd, const dev::KParams& kp, const void* str_sorted,
                  double* partial, cudaStream_t st, const void* sig_sorted = nullptr);
  // original oversampled source index -> sorted position
  const int32_t* sdest() const { return sdest_.p; }
  // per original target: centre of its leaf (3 doubles), the origin of the
  // FP32 coordinates of every pair the leaf evaluates directly
  const double* tcentre() const { return tcen_.p; }
  const TreeStats& stats() const { return stats_; }
  tree::Params params() const { return prm_; }

 private:
  int ensure_scratch(int nd, int precision);
  tree::Params prm_;
  TreeStats stats_;
  int64_t ntarg_ = 0, nptso_ = 0;
  int nleaf_ = 0, npitems_ = 0, nup_ = 0, nred_ = 0;
  DBuf<double> tx_, ty_, tz_, sx_, sy_, sz_, snx_, sny_, snz_, tcen_;
  DBuf<int64_t> tperm_;
  DBuf<int32_t> sdest_;
  DBuf<char> tnodes_, pent_, cent_, upitems_, reds_;
  DBuf<int> leaves_;
  DBuf<int2> pitems_;
  DBuf<double> tpx_, tpy_, tpz_, spx_, spy_, spz_;
  DBuf<double> up_part_;
  DBuf<char> qhat_, phi_, ab_;
  int ab_precision_ = -1;
  int64_t up_len_ = 0;
};

}  // namespace bie
