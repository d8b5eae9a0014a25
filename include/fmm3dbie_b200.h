/*
 * fmm3dbie_b200.h -- C-ABI of libfmm3dbie_b200.so, a B200 (sm_100a)
 * implementation of fmm3dbie's locally corrected combined-field layer
 * potentials and the GMRES solvers built on them.
 *
 * Conventions (identical to the Fortran calling sequences they replace):
 *  - integers are int64_t; index arrays (ixyzs, row_ptr, col_ind, iquad,
 *    ixyzso) are 1-based, exactly as getnearquad_* / findnear produce them;
 *  - arrays are column-major Fortran layouts: srccoefs(9,npts),
 *    srcvals(12,npts), targs(ndtarg,ntarg), srcover(12,nptso);
 *  - complex values are interleaved (re, im) doubles, layout-compatible with
 *    complex*16 and C99 double _Complex;
 *  - every function returns an int status (BIE_OK = 0) and never aborts;
 *    bie_last_error() gives a message for the calling thread.
 *  - all pointers are HOST pointers unless the name says "_dev"; the
 *    bie_plan_* family works on device buffers and a caller-supplied CUDA
 *    stream (NULL = legacy default stream).
 */
#ifndef FMM3DBIE_B200_H
#define FMM3DBIE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BIE_OK 0
#define BIE_ERR_ARG 1
#define BIE_ERR_CUDA 2
#define BIE_NOT_CONVERGED 3
#define BIE_BREAKDOWN 4
#define BIE_ERR_NOMEM 5
#define BIE_ERR_TABLES 6
#define BIE_ERR_SINGULAR 7
#define BIE_ERR_TIMEOUT 8

/* ---- library ------------------------------------------------------------ */
const char* bie_version(void);
const char* bie_last_error(void);
/* Load the Vioreanu-Rokhlin node tables (NULL: the file next to the
 * library).  Called implicitly by every entry point that needs them. */
int bie_init(const char* table_path);

/* ---- discretisation (src/surface_routs/patch_basis_routs.f90) ------------ */
/* get_npols (patch_basis_routs.f90:6) */
int bie_get_npols(int64_t iptype, int64_t norder, int64_t* npols);
/* get_disc_exps (patch_basis_routs.f90:234): uvs(2,npols), umat/vmat
 * (npols,npols) column-major as in the reference, wts(npols) */
int bie_get_disc_exps(int64_t norder, int64_t npols, int64_t iptype, double* uvs, double* umatr,
                      double* vmatr, double* wts);
/* get_basis_pols (patch_basis_routs.f90:298) / koorn_pols (koornexps.f90:206) */
int bie_get_basis_pols(const double* uv, int64_t norder, int64_t npols, int64_t iptype,
                       double* pols);

/* ---- surfaces (src/surface_routs/xtri_parameterizations.f90) -------------- */
/* Icosahedron refined nref times, radially projected onto the ellipsoid
 * center + axes .* x/|x| (xtri_platonic + xtri_refine4_flat +
 * xtri_ellipsoid_eval, :1335,:1864,:247), order norder RV nodes; arrays are
 * sized for npatches = 20*4^nref. */
int64_t bie_icosa_npatches(int64_t nref);
int bie_surf_icosa_ellipsoid(int64_t nref, int64_t norder, const double* axes,
                             const double* center, int64_t* norders, int64_t* ixyzs,
                             int64_t* iptype, double* srcvals, double* srccoefs);
/* Torus (R + r(p) cos t) (cos p, sin p) + r(p) sin t e_z, r(p) = r0 + r1
 * cos(m p), nu x nv quad patches with (norder+1)^2 Gauss-Legendre nodes
 * (iptype 11; chart in the style of xquad_wtorus_eval,
 * xquad_parametrizations.f90:6). */
int bie_surf_torus_quad(int64_t nu, int64_t nv, int64_t norder, double R, double r0, double r1,
                        int64_t m, int64_t* norders, int64_t* ixyzs, int64_t* iptype,
                        double* srcvals, double* srccoefs);

/* ---- setup (src/surface_routs/surf_routs.f90, src/quadratures/*) --------- */
/* get_centroid_rads (surf_routs.f90:195) */
int bie_get_centroid_rads(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                          const int64_t* iptype, int64_t npts, const double* srccoefs,
                          double* cms, double* rads);
/* get_rfacs (near_field_routs.f:826) */
int bie_get_rfacs(int64_t norder, int64_t iptype, double* rfac, double* rfac0);
/* get_qwts (surf_routs.f90:1598) */
int bie_get_qwts(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                 const int64_t* iptype, int64_t npts, const double* srcvals, double* qwts);
/* findnearmem / findnear (near_field_routs.f:193,424): row-sparse list of
 * patches j with |t_i - cms_j| <= rad_near_j; rows sorted by patch. */
int bie_findnearmem(const double* cms, int64_t npatches, const double* rad_near, int64_t ndtarg,
                    const double* targs, int64_t ntarg, int64_t* nnz);
int bie_findnear(const double* cms, int64_t npatches, const double* rad_near, int64_t ndtarg,
                 const double* targs, int64_t ntarg, int64_t* row_ptr, int64_t* col_ind);
/* get_iquad_rsc (near_field_routs.f:765) */
int bie_get_iquad_rsc(int64_t npatches, const int64_t* ixyzs, int64_t npts, int64_t nnz,
                      const int64_t* row_ptr, const int64_t* col_ind, int64_t* iquad);
/* get_far_order (far_field_routs.f90:10); zk complex (2 doubles) */
int bie_get_far_order(double eps, int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                      const int64_t* iptype, const double* cms, const double* rads, int64_t npts,
                      const double* srccoefs, int64_t ndtarg, int64_t ntarg,
                      const double* targvals, int64_t ikerorder, const double* zk, int64_t nnz,
                      const int64_t* row_ptr, const int64_t* col_ind, double rfac,
                      int64_t* nfars, int64_t* ixyzso);
/* oversample_geom (surf_routs.f90:304) */
int bie_oversample_geom(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                        const int64_t* iptype, int64_t npts, const double* srccoefs,
                        const double* srcvals, const int64_t* nfars, const int64_t* ixyzso,
                        int64_t nptso, double* srcover);
/* The three setup steps above on the device (same arguments and results;
 * no reference counterpart, the reference runs its setup on the CPU).
 * bie_findnear_gpu fills row_ptr and, when row_ptr[ntarg] - 1 <= col_cap,
 * col_ind; otherwise it returns BIE_ERR_ARG and the caller retries with
 * col_ind of row_ptr[ntarg] - 1 entries.  The near set is decided with the
 * host's rounding (no fused multiply-add), so both return the same lists;
 * far orders and oversampled geometry agree with the host's up to rounding
 * (the order decision compares with a tolerance). */
int bie_findnear_gpu(const double* cms, int64_t npatches, const double* rad_near, int64_t ndtarg,
                     const double* targs, int64_t ntarg, int64_t* row_ptr, int64_t* col_ind,
                     int64_t col_cap);
int bie_get_far_order_gpu(double eps, int64_t npatches, const int64_t* norders,
                          const int64_t* ixyzs, const int64_t* iptype, const double* cms,
                          const double* rads, int64_t npts, const double* srccoefs,
                          int64_t ndtarg, int64_t ntarg, const double* targvals,
                          int64_t ikerorder, const double* zk, int64_t nnz,
                          const int64_t* row_ptr, const int64_t* col_ind, double rfac,
                          int64_t* nfars, int64_t* ixyzso);
int bie_oversample_geom_gpu(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                            const int64_t* iptype, int64_t npts, const double* srccoefs,
                            const double* srcvals, const int64_t* nfars, const int64_t* ixyzso,
                            int64_t nptso, double* srcover);
/* oversample_fun_surf (surf_routs.f90:451), nd interleaved real functions */
int bie_oversample_fun_surf(int64_t nd, int64_t npatches, const int64_t* norders,
                            const int64_t* ixyzs, const int64_t* iptype, int64_t npts,
                            const double* u, const int64_t* nfars, const int64_t* ixyzso,
                            int64_t nptso, double* uover);
/* get_fmm_thresh (get_fmm_thresh.f:1) */
int bie_get_fmm_thresh(int64_t nds, int64_t ns, const double* src, int64_t ndt, int64_t nt,
                       const double* trg, double* thresh);
/* get_patch_id_uvs (surf_routs.f90:1736) */
int bie_get_patch_id_uvs(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                         const int64_t* iptype, int64_t npts, int64_t* ipatch_id,
                         double* uvs_pts);
/* hkrand (src/common/hkrand.f:3) */
double bie_hkrand(int64_t iseed);

/* ---- near quadrature ------------------------------------------------------ */
/* getnearquad_lap_comb_dir_eval (lap_comb_dir.f90:228): dpars = (alpha, beta),
 * wnear(nquad) real.  getnearquad_lap_comb_dir (:86) is the on-surface case
 * ntarg = npts, targs = srcvals, ipatch_id/uvs_targ from get_patch_id_uvs. */
int bie_getnearquad_lap_comb_dir_eval(int64_t npatches, const int64_t* norders,
                                      const int64_t* ixyzs, const int64_t* iptype, int64_t npts,
                                      const double* srccoefs, const double* srcvals,
                                      int64_t ndtarg, int64_t ntarg, const double* targs,
                                      const int64_t* ipatch_id, const double* uvs_targ,
                                      double eps, const double* dpars, int64_t iquadtype,
                                      int64_t nnz, const int64_t* row_ptr,
                                      const int64_t* col_ind, const int64_t* iquad, double rfac0,
                                      int64_t nquad, double* wnear);
/* getnearquad_helm_comb_dir_eval (helm_comb_dir.f:250): zpars = (k, alpha,
 * beta) complex, wnear(nquad) complex. */
int bie_getnearquad_helm_comb_dir_eval(int64_t npatches, const int64_t* norders,
                                       const int64_t* ixyzs, const int64_t* iptype, int64_t npts,
                                       const double* srccoefs, const double* srcvals,
                                       int64_t ndtarg, int64_t ntarg, const double* targs,
                                       const int64_t* ipatch_id, const double* uvs_targ,
                                       double eps, const double* zpars, int64_t iquadtype,
                                       int64_t nnz, const int64_t* row_ptr,
                                       const int64_t* col_ind, const int64_t* iquad,
                                       double rfac0, int64_t nquad, double* wnear);

/* The same two generators on the device (host buffers; the call returns
 * when the weights are in wnear).  Same arguments as the host versions plus
 * stats (nullable, 4 entries): kernel evaluations, self pairs, near pairs,
 * device time of the generator's pair kernel in microseconds.
 * The rules, tolerance and refinement are the host generator's; the weights
 * agree with it to the requested tolerance.  Patches with more than 256
 * basis functions are refused (BIE_ERR_ARG).  No reference counterpart: the
 * reference generates near quadrature on the CPU only. */
int bie_getnearquad_lap_comb_dir_eval_gpu(
    int64_t npatches, const int64_t* norders, const int64_t* ixyzs, const int64_t* iptype,
    int64_t npts, const double* srccoefs, const double* srcvals, int64_t ndtarg, int64_t ntarg,
    const double* targs, const int64_t* ipatch_id, const double* uvs_targ, double eps,
    const double* dpars, int64_t iquadtype, int64_t nnz, const int64_t* row_ptr,
    const int64_t* col_ind, const int64_t* iquad, double rfac0, int64_t nquad, double* wnear,
    int64_t* stats);
int bie_getnearquad_helm_comb_dir_eval_gpu(
    int64_t npatches, const int64_t* norders, const int64_t* ixyzs, const int64_t* iptype,
    int64_t npts, const double* srccoefs, const double* srcvals, int64_t ndtarg, int64_t ntarg,
    const double* targs, const int64_t* ipatch_id, const double* uvs_targ, double eps,
    const double* zpars, int64_t iquadtype, int64_t nnz, const int64_t* row_ptr,
    const int64_t* col_ind, const int64_t* iquad, double rfac0, int64_t nquad, double* wnear,
    int64_t* stats);
/* Setup engine of the simple evaluators and solvers (lap/helm_comb_dir_eval,
 * *_solver): 1 = device near lists, far orders, oversampled geometry and
 * near quadrature (default), 0 = host.  Patches above 256 basis functions
 * always use the host. */
int bie_set_nearquad_engine(int64_t engine);
int64_t bie_get_nearquad_engine(void);

/* ---- layer potentials on the GPU (host buffers) --------------------------- */
/* lpcomp_lap_comb_dir_addsub (lap_comb_dir.f90:633): principal value of
 * (alpha S_0 + beta D_0) sigma at the surface nodes. ndd=2, dpars=(alpha,beta),
 * nker=1, ndim=1; work/lwork/zpars/ipars unused as in the reference. */
int bie_lpcomp_lap_comb_dir_addsub(int64_t npatches, const int64_t* norders,
                                   const int64_t* ixyzs, const int64_t* iptype, int64_t npts,
                                   const double* srccoefs, const double* srcvals, double eps,
                                   int64_t ndd, const double* dpars, int64_t ndz,
                                   const double* zpars, int64_t ndi, const int64_t* ipars,
                                   int64_t nnz, const int64_t* row_ptr, const int64_t* col_ind,
                                   const int64_t* iquad, int64_t nquad, int64_t nker,
                                   const double* wnear, const int64_t* novers, int64_t nptso,
                                   const int64_t* ixyzso, const double* srcover,
                                   const double* whtsover, int64_t lwork, const double* work,
                                   int64_t ndim, const double* sigma, double* pot);
/* lpcomp_helm_comb_dir_addsub (helm_comb_dir.f:658): complex wnear, sigma,
 * pot; zpars = (k, alpha, beta). */
int bie_lpcomp_helm_comb_dir_addsub(int64_t npatches, const int64_t* norders,
                                    const int64_t* ixyzs, const int64_t* iptype, int64_t npts,
                                    const double* srccoefs, const double* srcvals, double eps,
                                    int64_t ndd, const double* dpars, int64_t ndz,
                                    const double* zpars, int64_t ndi, const int64_t* ipars,
                                    int64_t nnz, const int64_t* row_ptr, const int64_t* col_ind,
                                    const int64_t* iquad, int64_t nquad, int64_t nker,
                                    const double* wnear, const int64_t* novers, int64_t nptso,
                                    const int64_t* ixyzso, const double* srcover,
                                    const double* whtsover, int64_t lwork, const double* work,
                                    int64_t ndim, const double* sigma, double* pot);
/* lap_comb_dir_eval_addsub / helm_comb_dir_eval_addsub (lap_comb_dir.f90:806,
 * helm_comb_dir.f:856): the same at ntarg arbitrary targets targs(ndtarg,
 * ntarg) with a near list row_ptr(ntarg+1). */
int bie_lap_comb_dir_eval_addsub(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                                 const int64_t* iptype, int64_t npts, const double* srccoefs,
                                 const double* srcvals, int64_t ndtarg, int64_t ntarg,
                                 const double* targs, double eps, const double* dpars,
                                 int64_t nnz, const int64_t* row_ptr, const int64_t* col_ind,
                                 const int64_t* iquad, int64_t nquad, const double* wnear,
                                 const int64_t* novers, int64_t nptso, const int64_t* ixyzso,
                                 const double* srcover, const double* whtsover,
                                 const double* sigma, double* pot);
int bie_helm_comb_dir_eval_addsub(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                                  const int64_t* iptype, int64_t npts, const double* srccoefs,
                                  const double* srcvals, int64_t ndtarg, int64_t ntarg,
                                  const double* targs, double eps, const double* zpars,
                                  int64_t nnz, const int64_t* row_ptr, const int64_t* col_ind,
                                  const int64_t* iquad, int64_t nquad, const double* wnear,
                                  const int64_t* novers, int64_t nptso, const int64_t* ixyzso,
                                  const double* srcover, const double* whtsover,
                                  const double* sigma, double* pot);
/* lap_comb_dir_eval (lap_comb_dir.f90:408) / helm_comb_dir_eval
 * (helm_comb_dir.f:440; exposed by the Python bindings as lpcomp_helm_comb_dir,
 * python/setup.py:39): setup (near list, far order, oversampling, near
 * quadrature) on the host, evaluation on the GPU. */
int bie_lap_comb_dir_eval(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                          const int64_t* iptype, int64_t npts, const double* srccoefs,
                          const double* srcvals, int64_t ndtarg, int64_t ntarg,
                          const double* targs, const int64_t* ipatch_id, const double* uvs_targ,
                          double eps, const double* dpars, const double* sigma, double* pot);
int bie_helm_comb_dir_eval(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                           const int64_t* iptype, int64_t npts, const double* srccoefs,
                           const double* srcvals, int64_t ndtarg, int64_t ntarg,
                           const double* targs, const int64_t* ipatch_id, const double* uvs_targ,
                           double eps, const double* zpars, const double* sigma, double* pot);

/* ---- solvers (host buffers) ----------------------------------------------- */
/* lap_comb_dir_solver_guru (lap_comb_dir.f90:1459): dgmres on
 * (did I + K) x = rhs, did = -(-1)^ifinout beta/2; errs(numit+1). */
int bie_lap_comb_dir_solver_guru(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                                 const int64_t* iptype, int64_t npts, const double* srccoefs,
                                 const double* srcvals, double eps, const double* dpars,
                                 int64_t numit, int64_t ifinout, const double* rhs, int64_t nnz,
                                 const int64_t* row_ptr, const int64_t* col_ind,
                                 const int64_t* iquad, int64_t nquad, int64_t nker,
                                 const double* wnear, const int64_t* novers, int64_t nptso,
                                 const int64_t* ixyzso, const double* srcover,
                                 const double* whtsover, double eps_gmres, int64_t* niter,
                                 double* errs, double* rres, double* soln);
/* helm_comb_dir_solver_guru (helm_comb_dir.f:2071): zgmres, zid =
 * -(-1)^ifinout zpars(3)/2. */
int bie_helm_comb_dir_solver_guru(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                                  const int64_t* iptype, int64_t npts, const double* srccoefs,
                                  const double* srcvals, double eps, const double* zpars,
                                  int64_t numit, int64_t ifinout, const double* rhs, int64_t nnz,
                                  const int64_t* row_ptr, const int64_t* col_ind,
                                  const int64_t* iquad, int64_t nquad, int64_t nker,
                                  const double* wnear, const int64_t* novers, int64_t nptso,
                                  const int64_t* ixyzso, const double* srcover,
                                  const double* whtsover, double eps_gmres, int64_t* niter,
                                  double* errs, double* rres, double* soln);
/* lap_comb_dir_solver (lap_comb_dir.f90:1189) / helm_comb_dir_solver
 * (helm_comb_dir.f:1808): setup on the host + GMRES on the GPU. */
int bie_lap_comb_dir_solver(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                            const int64_t* iptype, int64_t npts, const double* srccoefs,
                            const double* srcvals, double eps, const double* dpars, int64_t numit,
                            int64_t ifinout, const double* rhs, double eps_gmres, int64_t* niter,
                            double* errs, double* rres, double* soln);
int bie_helm_comb_dir_solver(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                             const int64_t* iptype, int64_t npts, const double* srccoefs,
                             const double* srcvals, double eps, const double* zpars,
                             int64_t numit, int64_t ifinout, const double* rhs, double eps_gmres,
                             int64_t* niter, double* errs, double* rres, double* soln);
/* Extension of helm_comb_dir_solver_guru (no reference counterpart for the
 * precision/batch arguments): nrhs independent right-hand sides rhs(nrhs,
 * npts) point-major; iprec 0 = FP64 GMRES (the reference method), 1 = FP32
 * matvec GMRES inside FP64 iterative refinement to relative residual
 * eps_gmres.  niter(nrhs), rres(nrhs). */
int bie_helm_comb_dir_solver_guru_ext(int64_t npatches, const int64_t* norders,
                                      const int64_t* ixyzs, const int64_t* iptype, int64_t npts,
                                      const double* srccoefs, const double* srcvals, double eps,
                                      const double* zpars, int64_t numit, int64_t ifinout,
                                      int64_t nrhs, const double* rhs, int64_t nnz,
                                      const int64_t* row_ptr, const int64_t* col_ind,
                                      const int64_t* iquad, int64_t nquad, const double* wnear,
                                      const int64_t* novers, int64_t nptso, const int64_t* ixyzso,
                                      const double* srcover, const double* whtsover,
                                      double eps_gmres, int64_t iprec, int64_t* niter,
                                      double* rres, double* soln);

/* ---- device-resident plans (device buffers, caller stream) ---------------- */
/* kind 0 Laplace (params = alpha, beta), 1 Helmholtz (params = k, alpha, beta
 * complex). Targets: ntarg = 0 means the surface nodes (lpcomp/solver case),
 * otherwise targs(ndtarg, ntarg) on the host. Host arrays are copied. */
int bie_plan_create(int64_t kind, const double* params, int64_t npatches,
                    const int64_t* norders, const int64_t* ixyzs, const int64_t* iptype,
                    int64_t npts, const double* srccoefs, const double* srcvals, int64_t ndtarg,
                    int64_t ntarg, const double* targs, int64_t nnz, const int64_t* row_ptr,
                    const int64_t* col_ind, const int64_t* iquad, int64_t nquad,
                    const double* wnear, const int64_t* novers, int64_t nptso,
                    const int64_t* ixyzso, const double* srcover, const double* whtsover,
                    void** plan);
int bie_plan_destroy(void* plan);
/* info[0..9] = npts, ntarg, nptso, nnz, nquad, far-field source chunks (f64),
 * (f32), kind, far-kernel shape variant (f64), (f32) -- the far-field shape
 * is the tuned one once a matvec of that precision has run */
int bie_plan_info(void* plan, int64_t* info);
/* pot_dev = K sigma_dev for nd densities per point; iprec 0 f64, 1 f32 */
int bie_plan_matvec(void* plan, int64_t iprec, int64_t nd, const double* sigma_dev,
                    double* pot_dev, void* stream);
/* GMRES on (zid I + K) x = rhs, nd independent systems (point-major).
 * mode 0: FP64 GMRES (reference method); 1: mixed precision refinement.
 * x0_dev (initial guess) may be NULL; with a guess the stopping test stays
 * relative to ||rhs||_w, and mode 1 takes the guess's residual with the
 * FP32 operator and replaces, per system, a guess whose residual is not
 * below ||rhs||_w by zero.  niter(nd), rres(nd), errs or NULL: mode 0 fills
 * errs((numit+1)*nd) with the residual history (relative to ||rhs||_w),
 * mode 1 fills errs[0] = number of FP64 matvecs, errs[1] = number of FP32
 * matvecs and, with a guess, errs[2+q] = 1 where system q's guess was
 * replaced by zero. */
int bie_plan_solve(void* plan, int64_t mode, int64_t nd, const double* zid,
                   const double* rhs_dev, const double* x0_dev, int64_t numit, double eps_gmres,
                   double* soln_dev, int64_t* niter, double* errs, double* rres, void* stream);
/* Stage timing with CUDA events on the call's stream: enable = 1 turns it
 * on, 0 off (both clear the totals), -1 only reads; times[0..7] =
 * strengths, far, combine (ms totals), calls for the f64 matvecs, then the
 * same four for the f32 matvecs. */
int bie_plan_timing(void* plan, int64_t enable, double* times);
/* Refinement residual of the mixed-precision solvers (mode 1 of
 * bie_plan_solve / bie_batch_solve, iprec 1 of *_solver_guru_ext), process
 * wide: 1 (default; BIE_MIXED_RESIDUAL=increment) keeps K x in FP64 from the
 * first refinement step's FP64 matvec and adds the FP32 operator's K d for a
 * later correction d whose FP32 error cannot reach the target
 * (1e-6 ||d||_w / ||x||_w <= eps_gmres / 4 for every active system), taken
 * from the inner GMRES's residual vector without a matvec, else applies the
 * FP64 operator to x again; 0 (BIE_MIXED_RESIDUAL=full) applies the FP64
 * operator to x after every inner solve.  bie_last_mixed_stats: the calling
 * thread's last mixed solve: out[0] FP64 matvecs, out[1] FP32 matvecs,
 * out[2] increment steps, out[3] largest ||d||_w / ||x||_w of an increment.
 * No reference counterpart. */
int bie_set_mixed_residual(int64_t mode);
int bie_get_mixed_residual(void);
int bie_last_mixed_stats(double* out);
/* Oversampling of several complex densities (oversample_fun_guru,
 * surf_routs.f90:511-591, nd at once) on the tensor cores: per patch the
 * interpolation matrix times the patch densities as a tcgen05.mma kind::tf32
 * GEMM with 3xTF32 products and an FP32 accumulator.  Engine 0: CUDA cores
 * (FP64 sums, the default in the plans' FP32 matvecs); 1: tensor cores where
 * they apply (Helmholtz, FP32 path, nd a multiple of 8 up to 128, patches of
 * at most 64 nodes and 128 far nodes; BIE_OVERSAMPLE_ENGINE=1).
 * bie_plan_oversample writes the FP32 oversampled densities of the plan's
 * surface, out_dev[2 (s nd + m) + re/im] for oversampled node s (1..nptso)
 * and density m, from sigma_dev (npts x nd complex, point-major), with the
 * engine given; stream-ordered.  No reference counterpart. */
int bie_set_oversample_engine(int64_t engine);
int bie_get_oversample_engine(void);
int bie_plan_oversample(void* plan, int64_t engine, int64_t nd, const double* sigma_dev,
                        float* out_dev, void* stream);
/* Far-field shape of (iprec, nd): bie_plan_set_far pins it (variant 0-2:
 * CUDA-core block shapes; 3-4: tensor-core kernel of the FP32 Helmholtz
 * multi-density path, 16/32 or 64 densities per CTA, nd >= 4; nchunks source
 * chunks) instead of the autotuner's choice; bie_plan_get_far returns the
 * variant, the chunk count and a nonzero flag if a tensor-core launch timed
 * out waiting for its MMAs.  No reference counterpart. */
int bie_plan_set_far(void* plan, int64_t iprec, int64_t nd, int64_t variant, int64_t nchunks);
int bie_plan_get_far(void* plan, int64_t iprec, int64_t nd, int64_t* out);
/* Far-field method of precision iprec, replacing the lfmm3d / hfmm3d calls
 * of lpcomp_*_addsub (lap_comb_dir.f90:1094, helm_comb_dir.f:1117):
 * method 0 = direct sum over all target-source pairs, 1 = hierarchical
 * (dual-tree barycentric Lagrange interpolation on Chebyshev proxy grids;
 * theta = opening angle of the acceptance test r_T + r_S < theta |c_T - c_S|,
 * p = grid points along a cluster's longest side, leaf_t / leaf_s = most
 * targets (<= 128) / sources per leaf; values <= 0 select the defaults,
 * theta 0.5, p 10 (FP64) / 8 (FP32), leaves 128 / 256).  A plan picks method
 * 1 by itself when ntarg * nptso >= 1.5e10 (BIE_FAR_METHOD = direct | tree |
 * auto and BIE_TREE_PAIRS override).  Switching the FP32 method refolds
 * the FP32 W_eff.  bie_plan_get_far_method: out[16] = method, p, theta,
 * target nodes, source nodes, target leaves, interactions by form (PP with
 * the self test, PP, PC, CP, CC), source proxies, target proxies, kernel
 * evaluations per density, build ms, basis terms of the upward and downward
 * passes per density (zeros after the method for method 0). */
int bie_plan_set_far_method(void* plan, int64_t iprec, int64_t method, double theta, int64_t p,
                            int64_t leaf_t, int64_t leaf_s, void* stream);
int bie_plan_get_far_method(void* plan, int64_t iprec, double* out);
/* Host-only check of the hierarchical far field's lists: builds the target
 * tree (leaves <= leaf_t points) and source tree (<= leaf_s) of the points
 * targ[3 nt] and src[3 ns] (xyz per point), the proxy grids for (theta, p,
 * wavenumber k) and the dual traversal.  out[14] = number of (target leaf,
 * source leaf) pairs not covered exactly once (0 when correct), target
 * nodes, source nodes, interactions by form (5), kernel evaluations of the
 * lists, ntarg * nsrc, smallest and largest target leaf, nodes of either
 * tree whose grid the caps could not hold, nodes whose point range is not
 * the union of its children's (0 when correct).  No GPU is used. */
int bie_tree_check(int64_t nt, const double* targ, int64_t ns, const double* src, double theta,
                   int64_t p, double k, int64_t leaf_t, int64_t leaf_s, double* out);

/* ---- far field on device buffers ----------------------------------------- */
/* The far-field sum that lfmm3d / hfmm3d compute inside lpcomp_*_addsub
 * (lap_comb_dir.f90:1094, helm_comb_dir.f:1117), evaluated directly:
 *   pot(t) = sum_s [charge_s G(t,s) + dipstr_s n_s . grad_s G(t,s)],
 *   G = e^{ikr}/(4 pi r) (k = 0 for Laplace), pairs with r^2 < thresh^2
 *   skipped (get_fmm_thresh.f:81).
 * Device pointers; coordinates are SoA: src_dev = x[ns], y[ns], z[ns];
 * nrm_dev (unit vectors) likewise; targ_dev = x[nt], y[nt], z[nt].
 * kind 0: real charge/dipstr/pot; kind 1: complex interleaved, zk = (re,im).
 * iprec 0: FP64 sum, 1: FP32 pair sum accumulated in FP64 per source tile.
 * From ns * nt >= 1.5e10 on (BIE_FAR_METHOD = direct | tree | auto,
 * BIE_TREE_PAIRS) the sum is evaluated hierarchically, as by a plan
 * (bie_plan_set_far_method defaults; about 1e-9 relative in FP64, 1e-6 in
 * FP32) -- the FMM's contract of a sum accurate to a tolerance.
 * Allocates its scratch (per-chunk partial sums) with cudaMalloc and
 * returns after the stream has finished the call. */
int bie_farfield_dev(int64_t kind, const double* zk, int64_t ns, const double* src_dev,
                     const double* nrm_dev, const double* charge_dev, const double* dipstr_dev,
                     int64_t nt, const double* targ_dev, double thresh, int64_t iprec,
                     double* pot_dev, void* stream);
/* The direct far-field sum of bie_farfield_dev, allocating nothing: for
 * callers that cannot allocate device memory at this point (their memory
 * belongs to their own pool or to a budget fixed at start-up, or a
 * cudaMalloc/cudaFree here would stall their other streams).  No counterpart
 * in the reference.  It always evaluates the direct sum and ignores
 * BIE_FAR_METHOD / BIE_TREE_PAIRS (bie_farfield_dev may switch to the
 * hierarchical sum from ns * nt >= 1.5e10 on).  Its scratch is a fixed
 * 48 MiB array inside the library that every GPU loading the library keeps
 * until exit; ns <= 1,048,576, nt <= 1,048,576 (Helmholtz) or 2,097,152
 * (Laplace), larger calls return BIE_ERR_ARG.  All calls share that array:
 * calls that overlap on the GPU race and must be ordered (one stream) by the
 * caller.  The first call on a device resolves the array's address and should
 * come before any stream capture on that device; the address is not valid
 * after cudaDeviceReset.  Returns without synchronising. */
int bie_farfield_dev_noalloc(int64_t kind, const double* zk, int64_t ns, const double* src_dev,
                             const double* nrm_dev, const double* charge_dev,
                             const double* dipstr_dev, int64_t nt, const double* targ_dev,
                             double thresh, int64_t iprec, double* pot_dev, void* stream);

/* ---- batches of surfaces (no reference counterpart) ---------------------
 * Many surfaces of uneven size solved together as one operator whose nodes
 * are the surfaces' nodes back to back (vectors: all nodes of surface 0,
 * then surface 1, ...; nd densities per node, point-major).  Each matvec
 * stage runs as one persistent launch over all surfaces (work lists of
 * patches, target-block x source-chunk items and row groups), captured once
 * per (precision, nd) in a CUDA graph; the far-field shape is autotuned on
 * the first matvec of each (precision, nd).  Every (surface, density) is an
 * independent system of the solvers. */
int bie_batch_create(void** batch);
int bie_batch_destroy(void* batch);
/* Adds an on-surface plan (bie_plan_create with ntarg = 0).  On success the
 * batch owns the plan (do not destroy it); on failure the caller keeps it.
 * All plans share one kernel kind and one device. */
int bie_batch_add(void* batch, void* plan);
int bie_batch_finalize(void* batch, void* stream);
/* info[6]: surfaces, nodes, kind, reduction chunks, far-kernel variant and
 * source chunk length kept for (f32, nd = 1) (-1 / 0 before the first use). */
int bie_batch_info(void* batch, int64_t* info);
/* 1 (default): replay the captured graph; 0: launch the three kernels. */
int bie_batch_set_graph(void* batch, int64_t enable);
int bie_batch_matvec(void* batch, int64_t iprec, int64_t nd, const double* x_dev, double* y_dev,
                     void* stream);
/* bie_plan_solve for a batch: zid per surface (complex, 2 doubles each);
 * niter(nsurf*nd), rres(nsurf*nd) per system (surface-major); mode 1:
 * stats[0] = FP64 matvecs, stats[1] = FP32 matvecs. */
int bie_batch_solve(void* batch, int64_t mode, int64_t nd, const double* zid,
                    const double* rhs_dev, const double* x0_dev, int64_t numit, double eps_gmres,
                    double* soln_dev, int64_t* niter, double* rres, double* stats, void* stream);

/* ---- learned warm start (no reference counterpart) ----------------------
 * The reference solvers always start GMRES from zero
 * (helm_comb_dir_solver_guru, helm_comb_dir.f:2071, calls zgmres_guru at
 * helm_comb_dir.f:2222; gmres_routs.f90:13).  These entry points train and run a per-node MLP
 * that predicts the density of the plane-wave problem
 * (zid I + K) sigma = -exp(i k d.x); the prediction is passed as x0 to
 * bie_plan_solve.  Network 10 -> 256 -> 256 -> 256 -> 256 -> 2 (tanh),
 * bf16 weights, fp32 accumulation, fp32 master weights, Adam.  Inputs per
 * row: d (3), (k - kc)/ks, x/xs (3), unit normal (3); output: the
 * demodulated density tau = sigma exp(-i k d.x) (re, im).
 * params: 200,706 floats: W0[256][10], W1..W3[256][256], W4[2][256], then
 * b0..b3[256], b4[2].  dirk: per solve (dx, dy, dz, k).  norm: (xs, kc, ks).
 * srcvals_dev: the surface's srcvals (12 x npts, reference layout) on the
 * device.  All pointers are device pointers; calls are asynchronous on
 * `stream`. */
/* Allocates the network (zero parameters) and its workspace for batches
 * of up to max_rows rows. */
int bie_mlp_create(int64_t max_rows, void** mlp);
int bie_mlp_destroy(void* mlp);
/* info[10]: nparams, max_rows, inputs, width, hidden layers, outputs, Adam
 * steps taken, number of weight (non-bias) parameters, engine, and a flag
 * that is non-zero if a tcgen05 kernel's completion wait ever timed out
 * (reading it synchronises the device). */
int bie_mlp_info(void* mlp, int64_t* info);
/* Hidden-layer forward GEMM engine: 0 = mma.sync bf16 tiles, 1 = tcgen05
 * (UMMA with the accumulator in tensor memory).  Backward GEMMs use mma.sync. */
int bie_mlp_set_engine(void* mlp, int64_t engine);
/* Sets the fp32 parameters (and their bf16 copy) and resets Adam. */
int bie_mlp_set_params(void* mlp, const float* params_dev, void* stream);
int bie_mlp_get_params(void* mlp, float* params_dev, void* stream);
/* y[m][2] = MLP(x[m][10]), 1 <= m <= max_rows. */
int bie_mlp_forward(void* mlp, const float* x_dev, int64_t m, float* y_dev, void* stream);
/* Gradient of mean_r |MLP(x_r) - t_r|^2 into grad_dev[nparams] (may be NULL)
 * and the loss into loss_dev[0] (may be NULL). */
int bie_mlp_grad(void* mlp, const float* x_dev, const float* t_dev, int64_t m, float* grad_dev,
                 float* loss_dev, void* stream);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on that loss. */
int bie_mlp_train_step(void* mlp, const float* x_dev, const float* t_dev, int64_t m, double lr,
                       float* loss_dev, void* stream);
/* m training rows drawn from nsolves solves: row r takes sample
 * hash(seed, r) mod (nsolves * npts); tau_dev[(j*npts + i)] complex fp32. */
int bie_mlp_gather(const double* srcvals_dev, int64_t npts, const double* dirk_dev,
                   int64_t nsolves, const float* tau_dev, const double* norm, uint64_t seed,
                   int64_t m, float* x_dev, float* t_dev, void* stream);
/* tau[(q*npts + i)] = sigma[(i*nd + q)] exp(-i k_q d_q.x_i) (complex fp32 out,
 * complex128 point-major in). */
int bie_mlp_demodulate(const double* srcvals_dev, int64_t npts, const double* dirk_dev,
                       int64_t nd, const double* sigma_dev, float* tau_dev, void* stream);
/* x0[(i*nd + q)] = tau_hat(d_q, k_q, x_i, n_i) exp(i k_q d_q.x_i), complex128
 * point-major: the initial guess for nd plane-wave systems. */
int bie_mlp_predict_density(void* mlp, const double* srcvals_dev, int64_t npts,
                            const double* dirk_dev, int64_t nd, const double* norm,
                            double* x0_dev, void* stream);

/* ---- measurement helpers (no reference counterpart) ---------------------- */
/* Number of kernels this library has launched in the process. */
int64_t bie_launch_count(void);
/* FP32 FFMA throughput of the current device (TFLOP/s) from a register-
 * resident FMA loop kernel, timed with CUDA events on the default stream. */
int bie_measure_fp32_peak(double* tflops, double* ms);
/* MUFU (special-function unit) throughput of the current device in G ops/s
 * from a register-resident rsqrt.approx loop kernel, timed with CUDA events. */
int bie_measure_mufu_peak(double* gops, double* ms);

#ifdef __cplusplus
}
#endif
#endif /* FMM3DBIE_B200_H */
