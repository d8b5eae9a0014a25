// Patch discretisations and polynomial bases used by the layer-potential path.
//
// iptype = 1  : triangle on the simplex (0,0),(1,0),(0,1), Vioreanu-Rokhlin
//               nodes, orthonormal Koornwinder basis
//               (src/surface_routs/patch_basis_routs.f90:6-340,
//                src/tria_routs/koornexps.f90:206-330)
// iptype = 11 : quadrilateral [-1,1]^2, tensor Gauss-Legendre nodes,
//               tensor Legendre basis in "full" ordering
//               (src/common/polytens.f:255-420,598-640)
// iptype = 12 : quadrilateral [-1,1]^2, tensor Chebyshev nodes/basis.
//
// Matrices are stored row-major: vmat[i*n+j] = basis_j(node_i) maps
// coefficients to values, umat = vmat^{-1} maps values to coefficients
// (coefs_l = sum_j umat[l*n+j] vals_j), the same maps as the reference's
// umatr(l,j)/vmatr(i,j).
#pragma once
#include <cstdint>
#include <vector>

namespace bie {

constexpr int kMaxOrder = 20;

int npols_of(int iptype, int norder);              // get_npols
bool valid_patch(int iptype, int norder);

// Vioreanu-Rokhlin tables (loaded once from the build-time binary cache).
int load_vr_tables(const char* path);               // 0 on success
bool vr_tables_loaded();

// Orthonormal Koornwinder polynomials on the simplex; pols has
// (nmax+1)(nmax+2)/2 entries ordered (0,0),(1,0),(1,1),(2,0),...
void koorn_pols(double u, double v, int nmax, double* pols);

// Unnormalised Legendre P_0..P_n at x (and derivatives if dp != nullptr).
void legendre_pols(double x, int n, double* p, double* dp = nullptr);
// Chebyshev T_0..T_n at x (and derivatives).
void chebyshev_pols(double x, int n, double* p, double* dp = nullptr);
// n-point Gauss-Legendre rule on [-1,1], ascending nodes.
void gauss_legendre(int n, double* x, double* w);
// n-point Chebyshev (first kind) nodes on [-1,1], ascending, with
// Clenshaw-Curtis-type weights for that node set.
void chebyshev_nodes(int n, double* x, double* w);

// Basis values at (u,v) for a patch type (get_basis_pols).
void basis_pols(int iptype, int norder, double u, double v, double* pols);
// Discretisation nodes uvs[2*npols] and weights (get_disc_nodes/_wts).
int disc_nodes(int iptype, int norder, double* uvs);
int disc_wts(int iptype, int norder, double* wts);
// Nodes, weights, vals->coefs (umat) and coefs->vals (vmat) (get_disc_exps).
int disc_exps(int iptype, int norder, double* uvs, double* umat, double* vmat,
              double* wts);
// Corners of the reference domain (get_boundary_vertices).
int boundary_vertices(int iptype, double* uv);     // returns nv (3 or 4)
// Indices (0-based) of nodes shared between order norder and nfar
// (get_clashing_indices); returns nclash.
int clashing_indices(int iptype, int norder, int nfar, int* iclash,
                     int* iclashfar);

// Dense inverse by Gauss-Jordan elimination with partial pivoting.
// Returns 0 on success, 1 if singular.
int invert(int n, const double* a, double* ainv);

// Interpolation matrix from order-norder nodes to order-nfar nodes:
// imat[i*npols+j] (nfar_pols x npols), = basis(order norder at far node i)
// times umat (vals->coefs), exactly the composition in
// oversample_fun_guru (src/surface_routs/surf_routs.f90:511-591).
int interp_matrix(int iptype, int norder, int nfar, std::vector<double>& imat);

}  // namespace bie
