// Host-side (FP64) setup for the locally corrected layer-potential path:
// surface generators, near lists, far-field oversampling orders and the
// oversampled geometry.  All index arrays follow the reference convention:
// int64, 1-based (ixyzs, row_ptr, col_ind, iquad, ixyzso).
#pragma once
#include <complex>
#include <cstdint>
#include <vector>

namespace bie {

using cdouble = std::complex<double>;

// Read-only view of a discretised surface (the reference's
// npatches, norders, ixyzs, iptype, npts, srccoefs(9,npts), srcvals(12,npts)).
struct Surf {
  int64_t npatches = 0, npts = 0;
  const int64_t* norders = nullptr;
  const int64_t* ixyzs = nullptr;  // 1-based, npatches+1
  const int64_t* iptype = nullptr;
  const double* srccoefs = nullptr;  // 9 x npts (column-major per point)
  const double* srcvals = nullptr;   // 12 x npts
  int64_t start(int64_t p) const { return ixyzs[p] - 1; }        // 0-based
  int64_t npols(int64_t p) const { return ixyzs[p + 1] - ixyzs[p]; }
};

// ---- surfaces ------------------------------------------------------------
// Icosahedron refined nref times (4-way, flat), each triangle mapped to the
// ellipsoid center + axes * x/|x| (xtri_ellipsoid_eval, sphere when axes=1),
// discretised at order norder with Vioreanu-Rokhlin nodes.
int surf_icosa_ellipsoid(int nref, int norder, const double axes[3], const double center[3],
                         int64_t* norders, int64_t* ixyzs, int64_t* iptype, double* srcvals,
                         double* srccoefs);
int64_t icosa_npatches(int nref);
// Torus x = (R + r(p) cos t) cos p, (R + r(p) cos t) sin p, r(p) sin t with
// r(p) = r0 + r1 cos(m p), split into nu (toroidal) x nv (poloidal) quad
// patches discretised at order norder on tensor Gauss-Legendre nodes
// (iptype 11).
int surf_torus_quad(int nu, int nv, int norder, double R, double r0, double r1, int m,
                    int64_t* norders, int64_t* ixyzs, int64_t* iptype, double* srcvals,
                    double* srccoefs);
// srccoefs = umat * srcvals(1:9) per patch (getgeominfo, surf_routs.f90:3200).
int vals_to_coefs(const Surf& s, const double* srcvals, double* srccoefs);

// ---- geometry helpers -------------------------------------------------------
void centroid_rads(const Surf& s, double* cms, double* rads);   // get_centroid_rads
void rfacs(int norder, int iptype, double* rfac, double* rfac0);  // get_rfacs
void qwts(const Surf& s, double* wts);                           // get_qwts
double fmm_thresh(int64_t ns, const double* src, int nds, int64_t nt, const double* trg,
                  int ndt);                                       // get_fmm_thresh
void patch_id_uvs(const Surf& s, int64_t* ipatch_id, double* uvs);  // get_patch_id_uvs

// ---- near field ----------------------------------------------------------------
// {patch j : |t_i - cms_j| <= rads_j} for each target i (findnear), rows
// sorted by patch index.  row_ptr/col_ind 1-based.
void findnear(int64_t npatches, const double* cms, const double* rads, int ndt, int64_t nt,
              const double* targs, std::vector<int64_t>& row_ptr, std::vector<int64_t>& col_ind);
void iquad_rsc(const Surf& s, int64_t nt, int64_t nnz, const int64_t* row_ptr,
               const int64_t* col_ind, int64_t* iquad);  // get_iquad_rsc
// Row-sparse -> column-sparse transpose (rsc_to_csc); 1-based output.
void rsc_to_csc(int64_t ncol, int64_t nrow, int64_t nnz, const int64_t* row_ptr,
                const int64_t* col_ind, int64_t* col_ptr, int64_t* row_ind, int64_t* iper);

// ---- far field ------------------------------------------------------------
// hkrand(iseed) from src/common/hkrand.f: reseeds the LAPACK DLARAN
// generator with (0,0,0,mod(2*iseed+1,4096)) and draws once.
double hkrand(int64_t iseed);
// Oversampling order per patch (get_far_order, far_field_routs.f90:10-177).
// ikerorder: -1 single layer, 0 double layer.  ixyzso is 1-based.
int far_order(double eps, const Surf& s, const double* cms, const double* rads, int ndt,
              int64_t nt, const double* targs, int ikerorder, cdouble zk, int64_t nnz,
              const int64_t* row_ptr, const int64_t* col_ind, double rfac, int64_t* nfars,
              int64_t* ixyzso);
// oversample_geom (surf_routs.f90:304-449).
int oversample_geom(const Surf& s, const int64_t* nfars, const int64_t* ixyzso, int64_t nptso,
                    double* srcover);
// oversample_fun_surf for nd interleaved real functions.
int oversample_fun(const Surf& s, int nd, const double* u, const int64_t* nfars,
                   const int64_t* ixyzso, int64_t nptso, double* uover);

}  // namespace bie
