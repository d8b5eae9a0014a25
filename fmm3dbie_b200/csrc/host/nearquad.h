// Near-field quadrature generator for the combined-field kernels
//   K(x,y) = alpha * G_k(x,y) + beta * dG_k/dn_y(x,y),  G_k = e^{ikr}/(4 pi r)
// in the row-sparse layout of getnearquad_{lap,helm}_comb_dir
// (src/lap_wrappers/lap_comb_dir.f90:86-400,
//  src/helm_wrappers/helm_comb_dir.f:107-440).
//
// For every near pair (target i, patch j) it returns
//   wnear(iquad(k)+l-1) = sum_m umat(m,l) * int_{patch j} K(t_i, y) P_m(u,v) dA
// i.e. the weights that map the patch's nodal density values to the
// potential, the same quantity zgetnearquad_ggq_guru stores
// (src/quadratures/ggq-quads.f:24-478).  The integration rules are this
// project's own: adaptive 4-way triangle refinement with a cached per-patch
// tree for targets off the patch, and, for targets on the patch, a split of
// the patch at the target into triangles each integrated with a Duffy map
// and a sinh map anchored at the closest edge point (the reference's GGQ
// self tables are not available).
#pragma once
#include <complex>
#include <cstdint>
#include <vector>

#include "setup.h"

namespace bie {

struct NearQuadStats {
  int64_t kernel_evals = 0;
  int64_t self_targets = 0;
  int64_t near_targets = 0;
  double device_ms = 0;  // device generator: time of its pair kernel
};

// Rule parameters shared by this generator and the device one
// (cuda/nearquad_gpu.h): points per direction of the collapsed Gauss rule for
// a patch of order norder (8, 10 or 12), points per direction of the self
// rule for tolerance eps, and the collapsed rule itself on the simplex
// (0,0),(1,0),(0,1) (ng*ng nodes, weights summing to 1/2).
int nearquad_tri_ng(int norder);
int nearquad_self_order(double eps);
void nearquad_tri_rule(int ng, std::vector<double>& xi, std::vector<double>& eta,
                       std::vector<double>& w);

// kind 0: Laplace (alpha, beta real; wnear real), kind 1: Helmholtz (complex).
// ipatch_id is 1-based, -1 for off-surface targets; uvs_targ (2,nt).
// wnear_re/wnear_im: output arrays of length nquad (wnear_im may be null for
// Laplace).  Returns 0 on success.
int getnearquad(const Surf& s, int ndt, int64_t nt, const double* targs, const int64_t* ipatch_id,
                const double* uvs_targ, double eps, int kind, cdouble zk, cdouble alpha,
                cdouble beta, int64_t nnz, const int64_t* row_ptr, const int64_t* col_ind,
                const int64_t* iquad, double rfac0, int64_t nquad, double* wnear_re,
                double* wnear_im, NearQuadStats* stats = nullptr);

}  // namespace bie
