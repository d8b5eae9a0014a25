// extern "C" entry points of libfmm3dbie_b200.so (declared in
// include/fmm3dbie_b200.h).  Host-buffer entry points build a plan, copy
// the inputs to the device, run, copy the result back and release the plan;
// the bie_plan_* family keeps everything resident on the device.
#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../../include/fmm3dbie_b200.h"
#include "../host/basis.h"
#include "../host/nearquad.h"
#include "../host/setup.h"
#include "nearquad_gpu.h"
#include "setup_gpu.h"
#include "plan.h"
#include "tree_far.h"

using bie::cdouble;

namespace {

std::mutex g_init_mu;

int ensure_tables(const char* path = nullptr) {
  if (bie::vr_tables_loaded()) return BIE_OK;
  std::lock_guard<std::mutex> lk(g_init_mu);
  if (bie::vr_tables_loaded()) return BIE_OK;
  std::string p;
  if (path && *path) {
    p = path;
  } else if (const char* env = std::getenv("BIE_TABLES")) {
    p = env;
  } else {
    Dl_info info;
    if (dladdr((void*)&ensure_tables, &info) && info.dli_fname) {
      std::string so = info.dli_fname;
      const size_t cut = so.find_last_of('/');
      p = (cut == std::string::npos ? std::string(".") : so.substr(0, cut)) +
          "/_data/vioreanu_rokhlin.bin";
    }
  }
  if (bie::load_vr_tables(p.c_str()) != 0) {
    bie::set_last_error("cannot load Vioreanu-Rokhlin tables from '" + p + "'");
    return BIE_ERR_TABLES;
  }
  return BIE_OK;
}

bie::Surf make_surf(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                    const int64_t* iptype, int64_t npts, const double* srccoefs,
                    const double* srcvals) {
  bie::Surf s;
  s.npatches = npatches;
  s.npts = npts;
  s.norders = norders;
  s.ixyzs = ixyzs;
  s.iptype = iptype;
  s.srccoefs = srccoefs;
  s.srcvals = srcvals;
  return s;
}

int check_surf(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
               const int64_t* iptype, int64_t npts) {
  if (npatches <= 0 || npts <= 0 || !norders || !ixyzs || !iptype) {
    bie::set_last_error("empty surface");
    return BIE_ERR_ARG;
  }
  if (ixyzs[0] != 1 || ixyzs[npatches] != npts + 1) {
    bie::set_last_error("ixyzs inconsistent with npts");
    return BIE_ERR_ARG;
  }
  for (int64_t p = 0; p < npatches; ++p)
    if (!bie::valid_patch(int(iptype[p]), int(norders[p])) ||
        ixyzs[p + 1] - ixyzs[p] != bie::npols_of(int(iptype[p]), int(norders[p]))) {
      bie::set_last_error("patch " + std::to_string(p + 1) + " has an invalid type/order/size");
      return BIE_ERR_ARG;
    }
  return BIE_OK;
}

// Stream-ordered host<->device staging of one host-buffer call.
struct Stage {
  cudaStream_t st = nullptr;
  Stage() { cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking); }
  ~Stage() {
    if (st) cudaStreamDestroy(st);
  }
};

// Everything the simple interfaces derive from the geometry (the setup part
// of lap_comb_dir_eval / helm_comb_dir_solver).
struct Setup {
  std::vector<double> cms, rads;
  std::vector<int64_t> row_ptr, col_ind, iquad, novers, ixyzso;
  std::vector<double> srcover, wover, wnear;
  int64_t nnz = 0, nquad = 0, nptso = 0;
  double rfac = 0, rfac0 = 0;
};

// Setup engine: 1 = device (near lists, far orders, oversampled geometry,
// near quadrature; the default), 0 = host.  Surfaces with patches above the
// device generators' basis limit use the host.
std::atomic<int> g_nearquad_engine{1};

int64_t max_npols(const bie::Surf& s) {
  int64_t m = 0;
  for (int64_t p = 0; p < s.npatches; ++p) m = std::max(m, s.npols(p));
  return m;
}

int run_setup(const bie::Surf& s, int kind, cdouble zk, cdouble alpha, cdouble beta, double eps,
              int ndtarg, int64_t ntarg, const double* targs, const int64_t* ipatch_id,
              const double* uvs_targ, Setup& o) {
  int64_t sump = 0, sumo = 0;
  for (int64_t p = 0; p < s.npatches; ++p) {
    sump += s.iptype[p];
    sumo += s.norders[p];
  }
  const int iptype_avg = int(std::floor(double(sump) / s.npatches));
  const int norder_avg = int(std::floor(double(sumo) / s.npatches));
  bie::rfacs(norder_avg, iptype_avg, &o.rfac, &o.rfac0);
  o.cms.resize(3 * s.npatches);
  o.rads.resize(s.npatches);
  bie::centroid_rads(s, o.cms.data(), o.rads.data());
  std::vector<double> rad_near(s.npatches);
  for (int64_t p = 0; p < s.npatches; ++p) rad_near[p] = o.rads[p] * o.rfac;
  const bool on_device = g_nearquad_engine.load() == 1 && max_npols(s) <= bie::kNearQuadMaxNp;
  std::unique_ptr<Stage> stg;
  std::unique_ptr<bie::AllocStreamScope> alloc_scope;
  if (on_device) {
    stg = std::make_unique<Stage>();
    alloc_scope = std::make_unique<bie::AllocStreamScope>(stg->st);
  }
  int ier = 0;
  if (on_device) {
    ier = bie::findnear_gpu(s.npatches, o.cms.data(), rad_near.data(), ndtarg, ntarg, targs,
                            o.row_ptr, o.col_ind, stg->st);
    if (ier) return ier;
  } else {
    bie::findnear(s.npatches, o.cms.data(), rad_near.data(), ndtarg, ntarg, targs, o.row_ptr,
                  o.col_ind);
  }
  o.nnz = int64_t(o.col_ind.size());
  o.iquad.resize(o.nnz + 1);
  bie::iquad_rsc(s, ntarg, o.nnz, o.row_ptr.data(), o.col_ind.data(), o.iquad.data());
  o.nquad = o.iquad[o.nnz] - 1;
  const int ikerorder = std::abs(beta) > 1e-16 ? 0 : -1;
  o.novers.resize(s.npatches);
  o.ixyzso.resize(s.npatches + 1);
  ier = on_device
            ? bie::far_order_gpu(eps, s, o.cms.data(), o.rads.data(), ndtarg, ntarg, targs,
                                 ikerorder, kind == 1 ? zk : cdouble(0), o.nnz, o.row_ptr.data(),
                                 o.col_ind.data(), o.rfac, o.novers.data(), o.ixyzso.data(),
                                 stg->st)
            : bie::far_order(eps, s, o.cms.data(), o.rads.data(), ndtarg, ntarg, targs,
                             ikerorder, kind == 1 ? zk : cdouble(0), o.nnz, o.row_ptr.data(),
                             o.col_ind.data(), o.rfac, o.novers.data(), o.ixyzso.data());
  if (ier) {
    bie::set_last_error("get_far_order failed");
    return BIE_ERR_ARG;
  }
  o.nptso = o.ixyzso[s.npatches] - 1;
  o.srcover.resize(12 * o.nptso);
  o.wover.resize(o.nptso);
  if (on_device) {
    ier = bie::oversample_geom_gpu(s, o.novers.data(), o.ixyzso.data(), o.nptso,
                                   o.srcover.data(), stg->st);
    if (ier) return ier;
  } else {
    bie::oversample_geom(s, o.novers.data(), o.ixyzso.data(), o.nptso, o.srcover.data());
  }
  bie::Surf so = make_surf(s.npatches, o.novers.data(), o.ixyzso.data(), s.iptype, o.nptso,
                           nullptr, o.srcover.data());
  bie::qwts(so, o.wover.data());
  const size_t wl = size_t(o.nquad) * (kind == 1 ? 2 : 1);
  o.wnear.assign(wl, 0.0);
  if (on_device && o.nnz > 0) {
    bie::DBuf<double> d_w;
    if (d_w.alloc(wl) != cudaSuccess) {
      bie::set_last_error("near quadrature: device allocation failed");
      return BIE_ERR_NOMEM;
    }
    ier = bie::getnearquad_gpu(s, ndtarg, ntarg, targs, ipatch_id, uvs_targ, eps, kind, zk, alpha,
                               beta, o.nnz, o.row_ptr.data(), o.col_ind.data(), o.iquad.data(),
                               o.nquad, d_w.p, stg->st);
    if (ier) return ier;
    if (cudaMemcpyAsync(o.wnear.data(), d_w.p, wl * sizeof(double), cudaMemcpyDeviceToHost,
                        stg->st) != cudaSuccess ||
        cudaStreamSynchronize(stg->st) != cudaSuccess) {
      bie::set_last_error("near quadrature: copy to host failed");
      return BIE_ERR_CUDA;
    }
    return BIE_OK;
  }
  std::vector<double> wre(o.nquad), wim(kind == 1 ? o.nquad : 0);
  ier = bie::getnearquad(s, ndtarg, ntarg, targs, ipatch_id, uvs_targ, eps, kind, zk, alpha, beta,
                         o.nnz, o.row_ptr.data(), o.col_ind.data(), o.iquad.data(), o.rfac0,
                         o.nquad, wre.data(), kind == 1 ? wim.data() : nullptr);
  if (ier) {
    bie::set_last_error("near quadrature generation failed");
    return BIE_ERR_ARG;
  }
  for (int64_t q = 0; q < o.nquad; ++q) {
    if (kind == 1) {
      o.wnear[2 * q] = wre[q];
      o.wnear[2 * q + 1] = wim[q];
    } else {
      o.wnear[q] = wre[q];
    }
  }
  return BIE_OK;
}

int plan_from_arrays(bie::Plan& P, int kind, cdouble zk, cdouble alpha, cdouble beta,
                     int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                     const int64_t* iptype, int64_t npts, const double* srccoefs,
                     const double* srcvals, int ndtarg, int64_t ntarg, const double* targs,
                     int64_t nnz, const int64_t* row_ptr, const int64_t* col_ind,
                     const int64_t* iquad, int64_t nquad, const double* wnear,
                     const int64_t* novers, int64_t nptso, const int64_t* ixyzso,
                     const double* srcover, const double* whtsover, bool keep_f32,
                     cudaStream_t st, bool async_weff = false) {
  int ier = ensure_tables();
  if (ier) return ier;
  ier = check_surf(npatches, norders, ixyzs, iptype, npts);
  if (ier) return ier;
  bie::PlanSpec sp;
  sp.kind = kind;
  sp.zk = zk;
  sp.alpha = alpha;
  sp.beta = beta;
  sp.npatches = npatches;
  sp.npts = npts;
  sp.norders = norders;
  sp.ixyzs = ixyzs;
  sp.iptype = iptype;
  sp.srccoefs = srccoefs;
  sp.srcvals = srcvals;
  sp.ndtarg = ndtarg;
  sp.ntarg = ntarg;
  sp.targs = targs;
  sp.nnz = nnz;
  sp.nquad = nquad;
  sp.row_ptr = row_ptr;
  sp.col_ind = col_ind;
  sp.iquad = iquad;
  sp.wnear = wnear;
  sp.novers = novers;
  sp.nptso = nptso;
  sp.ixyzso = ixyzso;
  sp.srcover = srcover;
  sp.whtsover = whtsover;
  sp.keep_f32 = keep_f32;
  sp.async_weff = async_weff;
  return P.build(sp, st);
}

template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc&) {
    bie::set_last_error("host allocation failed");
    return BIE_ERR_NOMEM;
  } catch (const std::exception& e) {
    bie::set_last_error(e.what());
    return BIE_ERR_ARG;
  }
}

int eval_on_gpu(int kind, cdouble zk, cdouble alpha, cdouble beta, int64_t npatches,
                const int64_t* norders, const int64_t* ixyzs, const int64_t* iptype, int64_t npts,
                const double* srccoefs, const double* srcvals, int ndtarg, int64_t ntarg,
                const double* targs, int64_t nnz, const int64_t* row_ptr, const int64_t* col_ind,
                const int64_t* iquad, int64_t nquad, const double* wnear, const int64_t* novers,
                int64_t nptso, const int64_t* ixyzso, const double* srcover,
                const double* whtsover, const double* sigma, double* pot) {
  Stage stg;
  bie::AllocStreamScope alloc_scope(stg.st);  // plan buffers return to the pool on stg.st
  bie::Plan P;
  int ier = plan_from_arrays(P, kind, zk, alpha, beta, npatches, norders, ixyzs, iptype, npts,
                             srccoefs, srcvals, ndtarg, ntarg, targs, nnz, row_ptr, col_ind, iquad,
                             nquad, wnear, novers, nptso, ixyzso, srcover, whtsover, false, stg.st);
  if (ier) return ier;
  const int c = kind == 1 ? 2 : 1;
  bie::DBuf<double> ds, dp;
  if (ds.alloc(size_t(npts) * c) || dp.alloc(size_t(std::max<int64_t>(ntarg, 1)) * c)) {
    bie::set_last_error("device allocation failed");
    return BIE_ERR_NOMEM;
  }
  cudaMemcpyAsync(ds.p, sigma, sizeof(double) * npts * c, cudaMemcpyHostToDevice, stg.st);
  ier = P.matvec(0, 1, ds.p, dp.p, stg.st);
  if (ier) return ier;
  cudaMemcpyAsync(pot, dp.p, sizeof(double) * ntarg * c, cudaMemcpyDeviceToHost, stg.st);
  const cudaError_t e = cudaStreamSynchronize(stg.st);
  if (e != cudaSuccess) {
    bie::set_last_error(cudaGetErrorString(e));
    return BIE_ERR_CUDA;
  }
  return BIE_OK;
}

int solve_on_gpu(int kind, cdouble zk, cdouble alpha, cdouble beta, int64_t npatches,
                 const int64_t* norders, const int64_t* ixyzs, const int64_t* iptype, int64_t npts,
                 const double* srccoefs, const double* srcvals, int64_t numit, int64_t ifinout,
                 int64_t nrhs, const double* rhs, int64_t nnz, const int64_t* row_ptr,
                 const int64_t* col_ind, const int64_t* iquad, int64_t nquad, const double* wnear,
                 const int64_t* novers, int64_t nptso, const int64_t* ixyzso,
                 const double* srcover, const double* whtsover, double eps_gmres, int iprec,
                 int64_t* niter, double* errs, double* rres, double* soln) {
  if (numit < 1 || nrhs < 1 || nrhs > 256) {
    bie::set_last_error("numit must be >= 1 and 1 <= nrhs <= 256");
    return BIE_ERR_ARG;
  }
  Stage stg;
  bie::AllocStreamScope alloc_scope(stg.st);  // plan buffers return to the pool on stg.st
  // The right-hand sides go first: a copy issued while the near quadrature's
  // chunk copies are queued lands after all of them (measured).
  const int c = kind == 1 ? 2 : 1;
  const size_t len = size_t(npts) * nrhs * c;
  bie::DBuf<double> dr, dx;
  if (dr.alloc(len) || dx.alloc(len)) {
    bie::set_last_error("device allocation failed");
    return BIE_ERR_NOMEM;
  }
  if (cudaMemcpyAsync(dr.p, rhs, sizeof(double) * len, cudaMemcpyHostToDevice, stg.st) != cudaSuccess) {
    bie::set_last_error("right-hand side upload failed");
    return BIE_ERR_CUDA;
  }
  bie::Plan P;
  // the near quadrature's upload and folds overlap the start of the solve
  int ier = plan_from_arrays(P, kind, zk, alpha, beta, npatches, norders, ixyzs, iptype, npts,
                             srccoefs, srcvals, 12, npts, srcvals, nnz, row_ptr, col_ind, iquad,
                             nquad, wnear, novers, nptso, ixyzso, srcover, whtsover, iprec == 1,
                             stg.st, true);
  if (ier) return ier;
  P.targets_on_surface = true;
  // zid = -(-1)^ifinout beta/2 (helm_comb_dir.f:2215, lap_comb_dir.f90:1619)
  const double sgn = (ifinout % 2 == 0) ? -1.0 : 1.0;
  const std::vector<cdouble> zid(size_t(nrhs), sgn * beta / 2.0);  // one per system
  int status = BIE_OK;
  if (iprec == 1) {
    bie::MixedOut mo;
    status = bie::solve_mixed(P, int(nrhs), zid.data(), dr.p, nullptr, numit, eps_gmres, 1e-5, 6,
                              dx.p, mo, stg.st);
    if (status != BIE_OK && status != BIE_NOT_CONVERGED) return status;
    for (int64_t q = 0; q < nrhs; ++q) {
      if (niter) niter[q] = mo.inner_iters[q];
      if (rres) rres[q] = mo.rres[q];
    }
  } else {
    bie::GmresOut go;
    status = bie::gmres(P, 0, 0, int(nrhs), zid.data(), dr.p, nullptr, numit, eps_gmres, dx.p, go,
                        stg.st);
    if (status != BIE_OK && status != BIE_NOT_CONVERGED && status != BIE_BREAKDOWN) return status;
    for (int64_t q = 0; q < nrhs; ++q) {
      if (niter) niter[q] = go.niter[q];
      if (rres) rres[q] = go.rres[q];
      if (errs)
        for (int64_t j = 0; j <= numit; ++j) errs[q * (numit + 1) + j] = go.errs[q * (numit + 1) + j];
    }
  }
  cudaMemcpyAsync(soln, dx.p, sizeof(double) * len, cudaMemcpyDeviceToHost, stg.st);
  const cudaError_t e = cudaStreamSynchronize(stg.st);
  if (e != cudaSuccess) {
    bie::set_last_error(cudaGetErrorString(e));
    return BIE_ERR_CUDA;
  }
  return status;
}

cdouble zpar(const double* z, int i) { return cdouble(z[2 * i], z[2 * i + 1]); }

}  // namespace

extern "C" {

const char* bie_version(void) { return "fmm3dbie_b200 0.1.0 (sm_100a)"; }
const char* bie_last_error(void) { return bie::last_error(); }
int bie_init(const char* table_path) { return ensure_tables(table_path); }

int bie_get_npols(int64_t iptype, int64_t norder, int64_t* npols) {
  *npols = bie::npols_of(int(iptype), int(norder));
  return *npols > 0 ? BIE_OK : BIE_ERR_ARG;
}

int bie_get_disc_exps(int64_t norder, int64_t npols, int64_t iptype, double* uvs, double* umatr,
                      double* vmatr, double* wts) {
  return guarded([&] {
    int ier = ensure_tables();
    if (ier) return ier;
    if (bie::npols_of(int(iptype), int(norder)) != npols) return BIE_ERR_ARG;
    const int n = int(npols);
    std::vector<double> um(n * n), vm(n * n);
    ier = bie::disc_exps(int(iptype), int(norder), uvs, um.data(), vm.data(), wts);
    if (ier) return ier == 6 ? BIE_ERR_TABLES : BIE_ERR_SINGULAR;
    // row-major -> Fortran column-major
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        umatr[i + j * n] = um[i * n + j];
        vmatr[i + j * n] = vm[i * n + j];
      }
    return BIE_OK;
  });
}

int bie_get_basis_pols(const double* uv, int64_t norder, int64_t npols, int64_t iptype,
                       double* pols) {
  if (bie::npols_of(int(iptype), int(norder)) != npols) return BIE_ERR_ARG;
  bie::basis_pols(int(iptype), int(norder), uv[0], uv[1], pols);
  return BIE_OK;
}

int64_t bie_icosa_npatches(int64_t nref) { return bie::icosa_npatches(int(nref)); }

int bie_surf_icosa_ellipsoid(int64_t nref, int64_t norder, const double* axes,
                             const double* center, int64_t* norders, int64_t* ixyzs,
                             int64_t* iptype, double* srcvals, double* srccoefs) {
  return guarded([&] {
    int ier = ensure_tables();
    if (ier) return ier;
    ier = bie::surf_icosa_ellipsoid(int(nref), int(norder), axes, center, norders, ixyzs, iptype,
                                    srcvals, srccoefs);
    return ier == 0 ? BIE_OK : (ier == 6 ? BIE_ERR_TABLES : BIE_ERR_ARG);
  });
}

int bie_surf_torus_quad(int64_t nu, int64_t nv, int64_t norder, double R, double r0, double r1,
                        int64_t m, int64_t* norders, int64_t* ixyzs, int64_t* iptype,
                        double* srcvals, double* srccoefs) {
  return guarded([&] {
    const int ier = bie::surf_torus_quad(int(nu), int(nv), int(norder), R, r0, r1, int(m), norders,
                                         ixyzs, iptype, srcvals, srccoefs);
    return ier == 0 ? BIE_OK : BIE_ERR_ARG;
  });
}

int bie_get_centroid_rads(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                          const int64_t* iptype, int64_t npts, const double* srccoefs,
                          double* cms, double* rads) {
  return guarded([&] {
    int ier = check_surf(npatches, norders, ixyzs, iptype, npts);
    if (ier) return ier;
    bie::centroid_rads(make_surf(npatches, norders, ixyzs, iptype, npts, srccoefs, nullptr), cms,
                       rads);
    return BIE_OK;
  });
}

int bie_get_rfacs(int64_t norder, int64_t iptype, double* rfac, double* rfac0) {
  bie::rfacs(int(norder), int(iptype), rfac, rfac0);
  return BIE_OK;
}

int bie_get_qwts(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                 const int64_t* iptype, int64_t npts, const double* srcvals, double* qwts) {
  return guarded([&] {
    int ier = ensure_tables();
    if (ier) return ier;
    ier = check_surf(npatches, norders, ixyzs, iptype, npts);
    if (ier) return ier;
    bie::qwts(make_surf(npatches, norders, ixyzs, iptype, npts, nullptr, srcvals), qwts);
    return BIE_OK;
  });
}

int bie_findnearmem(const double* cms, int64_t npatches, const double* rad_near, int64_t ndtarg,
                    const double* targs, int64_t ntarg, int64_t* nnz) {
  return guarded([&] {
    std::vector<int64_t> rp, ci;
    bie::findnear(npatches, cms, rad_near, int(ndtarg), ntarg, targs, rp, ci);
    *nnz = int64_t(ci.size());
    return BIE_OK;
  });
}

int bie_findnear(const double* cms, int64_t npatches, const double* rad_near, int64_t ndtarg,
                 const double* targs, int64_t ntarg, int64_t* row_ptr, int64_t* col_ind) {
  return guarded([&] {
    std::vector<int64_t> rp, ci;
    bie::findnear(npatches, cms, rad_near, int(ndtarg), ntarg, targs, rp, ci);
    std::copy(rp.begin(), rp.end(), row_ptr);
    std::copy(ci.begin(), ci.end(), col_ind);
    return BIE_OK;
  });
}

int bie_findnear_gpu(const double* cms, int64_t npatches, const double* rad_near, int64_t ndtarg,
                     const double* targs, int64_t ntarg, int64_t* row_ptr, int64_t* col_ind,
                     int64_t col_cap) {
  return guarded([&] {
    if (!cms || !rad_near || !targs || !row_ptr || ndtarg < 3 || ntarg < 0 || npatches < 0) {
      bie::set_last_error("findnear_gpu: invalid arguments");
      return BIE_ERR_ARG;
    }
    Stage stg;
    bie::AllocStreamScope alloc_scope(stg.st);
    std::vector<int64_t> rp, ci;
    int ier = bie::findnear_gpu(npatches, cms, rad_near, int(ndtarg), ntarg, targs, rp, ci, stg.st);
    if (ier) return ier;
    std::copy(rp.begin(), rp.end(), row_ptr);
    if (int64_t(ci.size()) > col_cap || (!ci.empty() && !col_ind)) {
      bie::set_last_error("findnear_gpu: col_ind needs " + std::to_string(ci.size()) + " entries");
      return BIE_ERR_ARG;
    }
    std::copy(ci.begin(), ci.end(), col_ind);
    return BIE_OK;
  });
}

int bie_get_iquad_rsc(int64_t npatches, const int64_t* ixyzs, int64_t npts, int64_t nnz,
                      const int64_t* row_ptr, const int64_t* col_ind, int64_t* iquad) {
  bie::Surf s;
  s.npatches = npatches;
  s.ixyzs = ixyzs;
  for (int64_t k = 0; k < nnz; ++k)
    if (col_ind[k] < 1 || col_ind[k] > npatches) return BIE_ERR_ARG;
  bie::iquad_rsc(s, npts, nnz, row_ptr, col_ind, iquad);
  return BIE_OK;
}

int bie_get_far_order(double eps, int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                      const int64_t* iptype, const double* cms, const double* rads, int64_t npts,
                      const double* srccoefs, int64_t ndtarg, int64_t ntarg,
                      const double* targvals, int64_t ikerorder, const double* zk, int64_t nnz,
                      const int64_t* row_ptr, const int64_t* col_ind, double rfac,
                      int64_t* nfars, int64_t* ixyzso) {
  return guarded([&] {
    int ier = ensure_tables();
    if (ier) return ier;
    ier = check_surf(npatches, norders, ixyzs, iptype, npts);
    if (ier) return ier;
    ier = bie::far_order(eps, make_surf(npatches, norders, ixyzs, iptype, npts, srccoefs, nullptr),
                         cms, rads, int(ndtarg), ntarg, targvals, int(ikerorder),
                         cdouble(zk[0], zk[1]), nnz, row_ptr, col_ind, rfac, nfars, ixyzso);
    return ier ? BIE_ERR_ARG : BIE_OK;
  });
}

int bie_get_far_order_gpu(double eps, int64_t npatches, const int64_t* norders,
                          const int64_t* ixyzs, const int64_t* iptype, const double* cms,
                          const double* rads, int64_t npts, const double* srccoefs,
                          int64_t ndtarg, int64_t ntarg, const double* targvals,
                          int64_t ikerorder, const double* zk, int64_t nnz,
                          const int64_t* row_ptr, const int64_t* col_ind, double rfac,
                          int64_t* nfars, int64_t* ixyzso) {
  return guarded([&] {
    int ier = ensure_tables();
    if (ier) return ier;
    ier = check_surf(npatches, norders, ixyzs, iptype, npts);
    if (ier) return ier;
    Stage stg;
    bie::AllocStreamScope alloc_scope(stg.st);
    return bie::far_order_gpu(eps, make_surf(npatches, norders, ixyzs, iptype, npts, srccoefs,
                                             nullptr),
                              cms, rads, int(ndtarg), ntarg, targvals, int(ikerorder),
                              cdouble(zk[0], zk[1]), nnz, row_ptr, col_ind, rfac, nfars, ixyzso,
                              stg.st);
  });
}

int bie_oversample_geom_gpu(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                            const int64_t* iptype, int64_t npts, const double* srccoefs,
                            const double* srcvals, const int64_t* nfars, const int64_t* ixyzso,
                            int64_t nptso, double* srcover) {
  return guarded([&] {
    int ier = ensure_tables();
    if (ier) return ier;
    ier = check_surf(npatches, norders, ixyzs, iptype, npts);
    if (ier) return ier;
    Stage stg;
    bie::AllocStreamScope alloc_scope(stg.st);
    return bie::oversample_geom_gpu(make_surf(npatches, norders, ixyzs, iptype, npts, srccoefs,
                                              srcvals),
                                    nfars, ixyzso, nptso, srcover, stg.st);
  });
}

int bie_oversample_geom(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                        const int64_t* iptype, int64_t npts, const double* srccoefs,
                        const double* srcvals, const int64_t* nfars, const int64_t* ixyzso,
                        int64_t nptso, double* srcover) {
  return guarded([&] {
    int ier = ensure_tables();
    if (ier) return ier;
    ier = check_surf(npatches, norders, ixyzs, iptype, npts);
    if (ier) return ier;
    ier = bie::oversample_geom(make_surf(npatches, norders, ixyzs, iptype, npts, srccoefs, srcvals),
                               nfars, ixyzso, nptso, srcover);
    return ier ? BIE_ERR_ARG : BIE_OK;
  });
}

int bie_oversample_fun_surf(int64_t nd, int64_t npatches, const int64_t* norders,
                            const int64_t* ixyzs, const int64_t* iptype, int64_t npts,
                            const double* u, const int64_t* nfars, const int64_t* ixyzso,
                            int64_t nptso, double* uover) {
  return guarded([&] {
    int ier = ensure_tables();
    if (ier) return ier;
    ier = check_surf(npatches, norders, ixyzs, iptype, npts);
    if (ier) return ier;
    ier = bie::oversample_fun(make_surf(npatches, norders, ixyzs, iptype, npts, nullptr, nullptr),
                              int(nd), u, nfars, ixyzso, nptso, uover);
    return ier ? BIE_ERR_ARG : BIE_OK;
  });
}

int bie_get_fmm_thresh(int64_t nds, int64_t ns, const double* src, int64_t ndt, int64_t nt,
                       const double* trg, double* thresh) {
  *thresh = bie::fmm_thresh(ns, src, int(nds), nt, trg, int(ndt));
  return BIE_OK;
}

int bie_get_patch_id_uvs(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                         const int64_t* iptype, int64_t npts, int64_t* ipatch_id,
                         double* uvs_pts) {
  return guarded([&] {
    int ier = ensure_tables();
    if (ier) return ier;
    ier = check_surf(npatches, norders, ixyzs, iptype, npts);
    if (ier) return ier;
    bie::patch_id_uvs(make_surf(npatches, norders, ixyzs, iptype, npts, nullptr, nullptr),
                      ipatch_id, uvs_pts);
    return BIE_OK;
  });
}

double bie_hkrand(int64_t iseed) { return bie::hkrand(iseed); }

int bie_getnearquad_lap_comb_dir_eval(int64_t npatches, const int64_t* norders,
                                      const int64_t* ixyzs, const int64_t* iptype, int64_t npts,
                                      const double* srccoefs, const double* srcvals,
                                      int64_t ndtarg, int64_t ntarg, const double* targs,
                                      const int64_t* ipatch_id, const double* uvs_targ,
                                      double eps, const double* dpars, int64_t /*iquadtype*/,
                                      int64_t nnz, const int64_t* row_ptr,
                                      const int64_t* col_ind, const int64_t* iquad, double rfac0,
                                      int64_t nquad, double* wnear) {
  return guarded([&] {
    int ier = ensure_tables();
    if (ier) return ier;
    ier = check_surf(npatches, norders, ixyzs, iptype, npts);
    if (ier) return ier;
    ier = bie::getnearquad(make_surf(npatches, norders, ixyzs, iptype, npts, srccoefs, srcvals),
                           int(ndtarg), ntarg, targs, ipatch_id, uvs_targ, eps, 0, 0.0, dpars[0],
                           dpars[1], nnz, row_ptr, col_ind, iquad, rfac0, nquad, wnear, nullptr);
    return ier ? BIE_ERR_ARG : BIE_OK;
  });
}

int bie_getnearquad_helm_comb_dir_eval(int64_t npatches, const int64_t* norders,
                                       const int64_t* ixyzs, const int64_t* iptype, int64_t npts,
                                       const double* srccoefs, const double* srcvals,
                                       int64_t ndtarg, int64_t ntarg, const double* targs,
                                       const int64_t* ipatch_id, const double* uvs_targ,
                                       double eps, const double* zpars, int64_t /*iquadtype*/,
                                       int64_t nnz, const int64_t* row_ptr,
                                       const int64_t* col_ind, const int64_t* iquad,
                                       double rfac0, int64_t nquad, double* wnear) {
  return guarded([&] {
    int ier = ensure_tables();
    if (ier) return ier;
    ier = check_surf(npatches, norders, ixyzs, iptype, npts);
    if (ier) return ier;
    std::vector<double> wre(nquad), wim(nquad);
    ier = bie::getnearquad(make_surf(npatches, norders, ixyzs, iptype, npts, srccoefs, srcvals),
                           int(ndtarg), ntarg, targs, ipatch_id, uvs_targ, eps, 1, zpar(zpars, 0),
                           zpar(zpars, 1), zpar(zpars, 2), nnz, row_ptr, col_ind, iquad, rfac0,
                           nquad, wre.data(), wim.data());
    for (int64_t q = 0; q < nquad; ++q) {
      wnear[2 * q] = wre[q];
      wnear[2 * q + 1] = wim[q];
    }
    return ier ? BIE_ERR_ARG : BIE_OK;
  });
}

namespace {
int nearquad_gpu_call(int kind, cdouble zk, cdouble alpha, cdouble beta, int64_t npatches,
                      const int64_t* norders, const int64_t* ixyzs, const int64_t* iptype,
                      int64_t npts, const double* srccoefs, const double* srcvals,
                      int64_t ndtarg, int64_t ntarg, const double* targs,
                      const int64_t* ipatch_id, const double* uvs_targ, double eps, int64_t nnz,
                      const int64_t* row_ptr, const int64_t* col_ind, const int64_t* iquad,
                      int64_t nquad, double* wnear, int64_t* stats) {
  int ier = ensure_tables();
  if (ier) return ier;
  ier = check_surf(npatches, norders, ixyzs, iptype, npts);
  if (ier) return ier;
  if (nquad < 0 || (nquad > 0 && !wnear)) {
    bie::set_last_error("getnearquad: missing output");
    return BIE_ERR_ARG;
  }
  const size_t wl = size_t(nquad) * (kind == 1 ? 2 : 1);
  Stage stg;
  bie::AllocStreamScope alloc_scope(stg.st);
  bie::DBuf<double> d_w;
  if (d_w.alloc(std::max<size_t>(wl, 1)) != cudaSuccess) {
    bie::set_last_error("getnearquad: device allocation failed");
    return BIE_ERR_NOMEM;
  }
  bie::NearQuadStats st;
  ier = bie::getnearquad_gpu(make_surf(npatches, norders, ixyzs, iptype, npts, srccoefs, srcvals),
                             int(ndtarg), ntarg, targs, ipatch_id, uvs_targ, eps, kind, zk, alpha,
                             beta, nnz, row_ptr, col_ind, iquad, nquad, d_w.p, stg.st, &st);
  if (ier) return ier;
  if (wl && (cudaMemcpyAsync(wnear, d_w.p, wl * sizeof(double), cudaMemcpyDeviceToHost,
                             stg.st) != cudaSuccess ||
             cudaStreamSynchronize(stg.st) != cudaSuccess)) {
    bie::set_last_error("getnearquad: copy to host failed");
    return BIE_ERR_CUDA;
  }
  if (stats) {
    stats[0] = st.kernel_evals;
    stats[1] = st.self_targets;
    stats[2] = st.near_targets;
    stats[3] = int64_t(st.device_ms * 1e3);
  }
  return BIE_OK;
}
}  // namespace

int bie_getnearquad_lap_comb_dir_eval_gpu(
    int64_t npatches, const int64_t* norders, const int64_t* ixyzs, const int64_t* iptype,
    int64_t npts, const double* srccoefs, const double* srcvals, int64_t ndtarg, int64_t ntarg,
    const double* targs, const int64_t* ipatch_id, const double* uvs_targ, double eps,
    const double* dpars, int64_t /*iquadtype*/, int64_t nnz, const int64_t* row_ptr,
    const int64_t* col_ind, const int64_t* iquad, double /*rfac0*/, int64_t nquad, double* wnear,
    int64_t* stats) {
  return guarded([&] {
    return nearquad_gpu_call(0, 0.0, dpars[0], dpars[1], npatches, norders, ixyzs, iptype, npts,
                             srccoefs, srcvals, ndtarg, ntarg, targs, ipatch_id, uvs_targ, eps,
                             nnz, row_ptr, col_ind, iquad, nquad, wnear, stats);
  });
}

int bie_getnearquad_helm_comb_dir_eval_gpu(
    int64_t npatches, const int64_t* norders, const int64_t* ixyzs, const int64_t* iptype,
    int64_t npts, const double* srccoefs, const double* srcvals, int64_t ndtarg, int64_t ntarg,
    const double* targs, const int64_t* ipatch_id, const double* uvs_targ, double eps,
    const double* zpars, int64_t /*iquadtype*/, int64_t nnz, const int64_t* row_ptr,
    const int64_t* col_ind, const int64_t* iquad, double /*rfac0*/, int64_t nquad, double* wnear,
    int64_t* stats) {
  return guarded([&] {
    return nearquad_gpu_call(1, zpar(zpars, 0), zpar(zpars, 1), zpar(zpars, 2), npatches, norders,
                             ixyzs, iptype, npts, srccoefs, srcvals, ndtarg, ntarg, targs,
                             ipatch_id, uvs_targ, eps, nnz, row_ptr, col_ind, iquad, nquad, wnear,
                             stats);
  });
}

int bie_set_nearquad_engine(int64_t engine) {
  if (engine != 0 && engine != 1) {
    bie::set_last_error("nearquad engine must be 0 (host) or 1 (device)");
    return BIE_ERR_ARG;
  }
  g_nearquad_engine.store(int(engine));
  return BIE_OK;
}

int64_t bie_get_nearquad_engine(void) { return g_nearquad_engine.load(); }

int bie_lpcomp_lap_comb_dir_addsub(int64_t npatches, const int64_t* norders,
                                   const int64_t* ixyzs, const int64_t* iptype, int64_t npts,
                                   const double* srccoefs, const double* srcvals, double /*eps*/,
                                   int64_t ndd, const double* dpars, int64_t, const double*,
                                   int64_t, const int64_t*, int64_t nnz, const int64_t* row_ptr,
                                   const int64_t* col_ind, const int64_t* iquad, int64_t nquad,
                                   int64_t nker, const double* wnear, const int64_t* novers,
                                   int64_t nptso, const int64_t* ixyzso, const double* srcover,
                                   const double* whtsover, int64_t, const double*, int64_t ndim,
                                   const double* sigma, double* pot) {
  if (ndd < 2 || nker != 1 || ndim != 1) {
    bie::set_last_error("lpcomp_lap_comb_dir_addsub needs ndd>=2, nker=1, ndim=1");
    return BIE_ERR_ARG;
  }
  return guarded([&] {
    return eval_on_gpu(0, 0.0, dpars[0], dpars[1], npatches, norders, ixyzs, iptype, npts,
                       srccoefs, srcvals, 12, npts, srcvals, nnz, row_ptr, col_ind, iquad, nquad,
                       wnear, novers, nptso, ixyzso, srcover, whtsover, sigma, pot);
  });
}

int bie_lpcomp_helm_comb_dir_addsub(int64_t npatches, const int64_t* norders,
                                    const int64_t* ixyzs, const int64_t* iptype, int64_t npts,
                                    const double* srccoefs, const double* srcvals, double /*eps*/,
                                    int64_t, const double*, int64_t ndz, const double* zpars,
                                    int64_t, const int64_t*, int64_t nnz, const int64_t* row_ptr,
                                    const int64_t* col_ind, const int64_t* iquad, int64_t nquad,
                                    int64_t nker, const double* wnear, const int64_t* novers,
                                    int64_t nptso, const int64_t* ixyzso, const double* srcover,
                                    const double* whtsover, int64_t, const double*, int64_t ndim,
                                    const double* sigma, double* pot) {
  if (ndz < 3 || nker != 1 || ndim != 1) {
    bie::set_last_error("lpcomp_helm_comb_dir_addsub needs ndz>=3, nker=1, ndim=1");
    return BIE_ERR_ARG;
  }
  return guarded([&] {
    return eval_on_gpu(1, zpar(zpars, 0), zpar(zpars, 1), zpar(zpars, 2), npatches, norders, ixyzs,
                       iptype, npts, srccoefs, srcvals, 12, npts, srcvals, nnz, row_ptr, col_ind,
                       iquad, nquad, wnear, novers, nptso, ixyzso, srcover, whtsover, sigma, pot);
  });
}

int bie_lap_comb_dir_eval_addsub(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                                 const int64_t* iptype, int64_t npts, const double* srccoefs,
                                 const double* srcvals, int64_t ndtarg, int64_t ntarg,
                                 const double* targs, double /*eps*/, const double* dpars,
                                 int64_t nnz, const int64_t* row_ptr, const int64_t* col_ind,
                                 const int64_t* iquad, int64_t nquad, const double* wnear,
                                 const int64_t* novers, int64_t nptso, const int64_t* ixyzso,
                                 const double* srcover, const double* whtsover,
                                 const double* sigma, double* pot) {
  return guarded([&] {
    return eval_on_gpu(0, 0.0, dpars[0], dpars[1], npatches, norders, ixyzs, iptype, npts,
                       srccoefs, srcvals, int(ndtarg), ntarg, targs, nnz, row_ptr, col_ind, iquad,
                       nquad, wnear, novers, nptso, ixyzso, srcover, whtsover, sigma, pot);
  });
}

int bie_helm_comb_dir_eval_addsub(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                                  const int64_t* iptype, int64_t npts, const double* srccoefs,
                                  const double* srcvals, int64_t ndtarg, int64_t ntarg,
                                  const double* targs, double /*eps*/, const double* zpars,
                                  int64_t nnz, const int64_t* row_ptr, const int64_t* col_ind,
                                  const int64_t* iquad, int64_t nquad, const double* wnear,
                                  const int64_t* novers, int64_t nptso, const int64_t* ixyzso,
                                  const double* srcover, const double* whtsover,
                                  const double* sigma, double* pot) {
  return guarded([&] {
    return eval_on_gpu(1, zpar(zpars, 0), zpar(zpars, 1), zpar(zpars, 2), npatches, norders, ixyzs,
                       iptype, npts, srccoefs, srcvals, int(ndtarg), ntarg, targs, nnz, row_ptr,
                       col_ind, iquad, nquad, wnear, novers, nptso, ixyzso, srcover, whtsover,
                       sigma, pot);
  });
}

static int eval_simple(int kind, cdouble zk, cdouble alpha, cdouble beta, int64_t npatches,
                       const int64_t* norders, const int64_t* ixyzs, const int64_t* iptype,
                       int64_t npts, const double* srccoefs, const double* srcvals, int64_t ndtarg,
                       int64_t ntarg, const double* targs, const int64_t* ipatch_id,
                       const double* uvs_targ, double eps, const double* sigma, double* pot) {
  int ier = ensure_tables();
  if (ier) return ier;
  ier = check_surf(npatches, norders, ixyzs, iptype, npts);
  if (ier) return ier;
  const bie::Surf s = make_surf(npatches, norders, ixyzs, iptype, npts, srccoefs, srcvals);
  Setup o;
  ier = run_setup(s, kind, zk, alpha, beta, eps, int(ndtarg), ntarg, targs, ipatch_id, uvs_targ, o);
  if (ier) return ier;
  return eval_on_gpu(kind, zk, alpha, beta, npatches, norders, ixyzs, iptype, npts, srccoefs,
                     srcvals, int(ndtarg), ntarg, targs, o.nnz, o.row_ptr.data(),
                     o.col_ind.data(), o.iquad.data(), o.nquad, o.wnear.data(), o.novers.data(),
                     o.nptso, o.ixyzso.data(), o.srcover.data(), o.wover.data(), sigma, pot);
}

int bie_lap_comb_dir_eval(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                          const int64_t* iptype, int64_t npts, const double* srccoefs,
                          const double* srcvals, int64_t ndtarg, int64_t ntarg,
                          const double* targs, const int64_t* ipatch_id, const double* uvs_targ,
                          double eps, const double* dpars, const double* sigma, double* pot) {
  return guarded([&] {
    return eval_simple(0, 0.0, dpars[0], dpars[1], npatches, norders, ixyzs, iptype, npts,
                       srccoefs, srcvals, ndtarg, ntarg, targs, ipatch_id, uvs_targ, eps, sigma,
                       pot);
  });
}

int bie_helm_comb_dir_eval(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                           const int64_t* iptype, int64_t npts, const double* srccoefs,
                           const double* srcvals, int64_t ndtarg, int64_t ntarg,
                           const double* targs, const int64_t* ipatch_id, const double* uvs_targ,
                           double eps, const double* zpars, const double* sigma, double* pot) {
  return guarded([&] {
    return eval_simple(1, zpar(zpars, 0), zpar(zpars, 1), zpar(zpars, 2), npatches, norders, ixyzs,
                       iptype, npts, srccoefs, srcvals, ndtarg, ntarg, targs, ipatch_id, uvs_targ,
                       eps, sigma, pot);
  });
}

int bie_lap_comb_dir_solver_guru(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                                 const int64_t* iptype, int64_t npts, const double* srccoefs,
                                 const double* srcvals, double /*eps*/, const double* dpars,
                                 int64_t numit, int64_t ifinout, const double* rhs, int64_t nnz,
                                 const int64_t* row_ptr, const int64_t* col_ind,
                                 const int64_t* iquad, int64_t nquad, int64_t nker,
                                 const double* wnear, const int64_t* novers, int64_t nptso,
                                 const int64_t* ixyzso, const double* srcover,
                                 const double* whtsover, double eps_gmres, int64_t* niter,
                                 double* errs, double* rres, double* soln) {
  if (nker != 1) return BIE_ERR_ARG;
  return guarded([&] {
    return solve_on_gpu(0, 0.0, dpars[0], dpars[1], npatches, norders, ixyzs, iptype, npts,
                        srccoefs, srcvals, numit, ifinout, 1, rhs, nnz, row_ptr, col_ind, iquad,
                        nquad, wnear, novers, nptso, ixyzso, srcover, whtsover, eps_gmres, 0,
                        niter, errs, rres, soln);
  });
}

int bie_helm_comb_dir_solver_guru(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                                  const int64_t* iptype, int64_t npts, const double* srccoefs,
                                  const double* srcvals, double /*eps*/, const double* zpars,
                                  int64_t numit, int64_t ifinout, const double* rhs, int64_t nnz,
                                  const int64_t* row_ptr, const int64_t* col_ind,
                                  const int64_t* iquad, int64_t nquad, int64_t nker,
                                  const double* wnear, const int64_t* novers, int64_t nptso,
                                  const int64_t* ixyzso, const double* srcover,
                                  const double* whtsover, double eps_gmres, int64_t* niter,
                                  double* errs, double* rres, double* soln) {
  if (nker != 1) return BIE_ERR_ARG;
  return guarded([&] {
    return solve_on_gpu(1, zpar(zpars, 0), zpar(zpars, 1), zpar(zpars, 2), npatches, norders,
                        ixyzs, iptype, npts, srccoefs, srcvals, numit, ifinout, 1, rhs, nnz,
                        row_ptr, col_ind, iquad, nquad, wnear, novers, nptso, ixyzso, srcover,
                        whtsover, eps_gmres, 0, niter, errs, rres, soln);
  });
}

int bie_helm_comb_dir_solver_guru_ext(int64_t npatches, const int64_t* norders,
                                      const int64_t* ixyzs, const int64_t* iptype, int64_t npts,
                                      const double* srccoefs, const double* srcvals,
                                      double /*eps*/, const double* zpars, int64_t numit,
                                      int64_t ifinout, int64_t nrhs, const double* rhs,
                                      int64_t nnz, const int64_t* row_ptr,
                                      const int64_t* col_ind, const int64_t* iquad, int64_t nquad,
                                      const double* wnear, const int64_t* novers, int64_t nptso,
                                      const int64_t* ixyzso, const double* srcover,
                                      const double* whtsover, double eps_gmres, int64_t iprec,
                                      int64_t* niter, double* rres, double* soln) {
  if (iprec != 0 && iprec != 1) return BIE_ERR_ARG;
  return guarded([&] {
    return solve_on_gpu(1, zpar(zpars, 0), zpar(zpars, 1), zpar(zpars, 2), npatches, norders,
                        ixyzs, iptype, npts, srccoefs, srcvals, numit, ifinout, nrhs, rhs, nnz,
                        row_ptr, col_ind, iquad, nquad, wnear, novers, nptso, ixyzso, srcover,
                        whtsover, eps_gmres, int(iprec), niter, nullptr, rres, soln);
  });
}

static int solver_simple(int kind, cdouble zk, cdouble alpha, cdouble beta, int64_t npatches,
                         const int64_t* norders, const int64_t* ixyzs, const int64_t* iptype,
                         int64_t npts, const double* srccoefs, const double* srcvals, double eps,
                         int64_t numit, int64_t ifinout, const double* rhs, double eps_gmres,
                         int64_t* niter, double* errs, double* rres, double* soln) {
  int ier = ensure_tables();
  if (ier) return ier;
  ier = check_surf(npatches, norders, ixyzs, iptype, npts);
  if (ier) return ier;
  const bie::Surf s = make_surf(npatches, norders, ixyzs, iptype, npts, srccoefs, srcvals);
  std::vector<int64_t> ipatch(npts);
  std::vector<double> uvs(2 * npts);
  bie::patch_id_uvs(s, ipatch.data(), uvs.data());
  Setup o;
  ier = run_setup(s, kind, zk, alpha, beta, eps, 12, npts, srcvals, ipatch.data(), uvs.data(), o);
  if (ier) return ier;
  return solve_on_gpu(kind, zk, alpha, beta, npatches, norders, ixyzs, iptype, npts, srccoefs,
                      srcvals, numit, ifinout, 1, rhs, o.nnz, o.row_ptr.data(), o.col_ind.data(),
                      o.iquad.data(), o.nquad, o.wnear.data(), o.novers.data(), o.nptso,
                      o.ixyzso.data(), o.srcover.data(), o.wover.data(), eps_gmres, 0, niter, errs,
                      rres, soln);
}

int bie_lap_comb_dir_solver(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                            const int64_t* iptype, int64_t npts, const double* srccoefs,
                            const double* srcvals, double eps, const double* dpars, int64_t numit,
                            int64_t ifinout, const double* rhs, double eps_gmres, int64_t* niter,
                            double* errs, double* rres, double* soln) {
  return guarded([&] {
    return solver_simple(0, 0.0, dpars[0], dpars[1], npatches, norders, ixyzs, iptype, npts,
                         srccoefs, srcvals, eps, numit, ifinout, rhs, eps_gmres, niter, errs, rres,
                         soln);
  });
}

int bie_helm_comb_dir_solver(int64_t npatches, const int64_t* norders, const int64_t* ixyzs,
                             const int64_t* iptype, int64_t npts, const double* srccoefs,
                             const double* srcvals, double eps, const double* zpars,
                             int64_t numit, int64_t ifinout, const double* rhs, double eps_gmres,
                             int64_t* niter, double* errs, double* rres, double* soln) {
  return guarded([&] {
    return solver_simple(1, zpar(zpars, 0), zpar(zpars, 1), zpar(zpars, 2), npatches, norders,
                         ixyzs, iptype, npts, srccoefs, srcvals, eps, numit, ifinout, rhs,
                         eps_gmres, niter, errs, rres, soln);
  });
}

// ---- plans ------------------------------------------------------------------
int bie_plan_create(int64_t kind, const double* params, int64_t npatches,
                    const int64_t* norders, const int64_t* ixyzs, const int64_t* iptype,
                    int64_t npts, const double* srccoefs, const double* srcvals, int64_t ndtarg,
                    int64_t ntarg, const double* targs, int64_t nnz, const int64_t* row_ptr,
                    const int64_t* col_ind, const int64_t* iquad, int64_t nquad,
                    const double* wnear, const int64_t* novers, int64_t nptso,
                    const int64_t* ixyzso, const double* srcover, const double* whtsover,
                    void** plan) {
  if (!plan || (kind != 0 && kind != 1)) return BIE_ERR_ARG;
  *plan = nullptr;
  return guarded([&] {
    auto P = std::make_unique<bie::Plan>();
    cdouble zk = 0, alpha, beta;
    if (kind == 0) {
      alpha = params[0];
      beta = params[1];
    } else {
      zk = zpar(params, 0);
      alpha = zpar(params, 1);
      beta = zpar(params, 2);
    }
    const bool on_surface = ntarg == 0;
    Stage stg;
    int ier = plan_from_arrays(*P, int(kind), zk, alpha, beta, npatches, norders, ixyzs, iptype,
                               npts, srccoefs, srcvals, on_surface ? 12 : int(ndtarg),
                               on_surface ? npts : ntarg, on_surface ? srcvals : targs, nnz,
                               row_ptr, col_ind, iquad, nquad, wnear, novers, nptso, ixyzso,
                               srcover, whtsover, true, stg.st);
    if (ier) return ier;
    P->targets_on_surface = on_surface;
    *plan = P.release();
    return BIE_OK;
  });
}

// ---- batches of surfaces (no reference counterpart) --------------------------
int bie_batch_create(void** batch) {
  if (!batch) return BIE_ERR_ARG;
  *batch = new bie::BatchPlan();
  return BIE_OK;
}

int bie_batch_destroy(void* batch) {
  delete static_cast<bie::BatchPlan*>(batch);
  return BIE_OK;
}

int bie_batch_add(void* batch, void* plan) {
  if (!batch || !plan) return BIE_ERR_ARG;
  // on failure the caller keeps the plan
  return static_cast<bie::BatchPlan*>(batch)->add(static_cast<bie::Plan*>(plan));
}

int bie_batch_finalize(void* batch, void* stream) {
  if (!batch) return BIE_ERR_ARG;
  return guarded([&] {
    return static_cast<bie::BatchPlan*>(batch)->finalize(static_cast<cudaStream_t>(stream));
  });
}

int bie_batch_info(void* batch, int64_t* info) {
  if (!batch || !info) return BIE_ERR_ARG;
  const auto* B = static_cast<const bie::BatchPlan*>(batch);
  info[0] = int64_t(B->plans.size());
  info[1] = B->nodes;
  info[2] = B->kind;
  info[3] = B->segs.nchunk;
  int v = -1;
  int64_t ch = 0;
  info[4] = B->far_choice(1, 1, &v, &ch) ? v : -1;
  info[5] = ch;
  return BIE_OK;
}

int bie_batch_set_graph(void* batch, int64_t enable) {
  if (!batch) return BIE_ERR_ARG;
  static_cast<bie::BatchPlan*>(batch)->use_graph = enable != 0;
  return BIE_OK;
}

int bie_batch_matvec(void* batch, int64_t iprec, int64_t nd, const double* x_dev, double* y_dev,
                     void* stream) {
  if (!batch || (iprec != 0 && iprec != 1) || nd < 1) return BIE_ERR_ARG;
  return guarded([&] {
    return static_cast<bie::BatchPlan*>(batch)->apply(int(iprec), int(nd), x_dev, y_dev,
                                                      static_cast<cudaStream_t>(stream));
  });
}

int bie_batch_solve(void* batch, int64_t mode, int64_t nd, const double* zid,
                    const double* rhs_dev, const double* x0_dev, int64_t numit, double eps_gmres,
                    double* soln_dev, int64_t* niter, double* rres, double* stats, void* stream) {
  if (!batch || (mode != 0 && mode != 1) || nd < 1 || nd > 256 || numit < 1 || !zid)
    return BIE_ERR_ARG;
  return guarded([&] {
    bie::BatchPlan& B = *static_cast<bie::BatchPlan*>(batch);
    const int ns = B.nseg();
    std::vector<cdouble> z(size_t(ns) * nd);
    for (int g = 0; g < ns; ++g)
      for (int64_t d = 0; d < nd; ++d) z[size_t(g) * nd + d] = cdouble(zid[2 * g], zid[2 * g + 1]);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t nsys = z.size();
    if (mode == 0) {
      bie::GmresOut go;
      const int s = bie::gmres(B, 0, 0, int(nd), z.data(), rhs_dev, x0_dev, numit, eps_gmres,
                               soln_dev, go, st);
      if (s == BIE_OK || s == BIE_NOT_CONVERGED || s == BIE_BREAKDOWN)
        for (size_t q = 0; q < nsys; ++q) {
          if (niter) niter[q] = go.niter[q];
          if (rres) rres[q] = go.rres[q];
        }
      return s;
    }
    bie::MixedOut mo;
    const int s = bie::solve_mixed(B, int(nd), z.data(), rhs_dev, x0_dev, numit, eps_gmres, 1e-5, 6,
                                   soln_dev, mo, st);
    if (s == BIE_OK || s == BIE_NOT_CONVERGED) {
      for (size_t q = 0; q < nsys; ++q) {
        if (niter) niter[q] = mo.inner_iters[q];
        if (rres) rres[q] = mo.rres[q];
      }
      if (stats) {
        stats[0] = mo.fp64_matvecs;
        stats[1] = mo.fp32_matvecs;
      }
    }
    return s;
  });
}

int bie_plan_destroy(void* plan) {
  delete static_cast<bie::Plan*>(plan);
  return BIE_OK;
}

int bie_plan_info(void* plan, int64_t* info) {
  if (!plan) return BIE_ERR_ARG;
  const bie::Plan* P = static_cast<bie::Plan*>(plan);
  info[0] = P->npts;
  info[1] = P->ntarg;
  info[2] = P->nptso;
  info[3] = P->nnz;
  info[4] = P->nquad;
  info[5] = P->nchunks_for(0, 1);
  info[6] = P->nchunks_for(1, 1);
  info[7] = P->kind;
  info[8] = P->far_config(0, 1).variant;
  info[9] = P->far_config(1, 1).variant;
  return BIE_OK;
}

int bie_plan_set_far(void* plan, int64_t iprec, int64_t nd, int64_t variant, int64_t nchunks) {
  if (!plan) return BIE_ERR_ARG;
  return guarded([&] {
    return static_cast<bie::Plan*>(plan)->set_far_config(int(iprec), int(nd), int(variant),
                                                         int(nchunks));
  });
}

int bie_set_oversample_engine(int64_t engine) {
  if (engine != 0 && engine != 1) return BIE_ERR_ARG;
  bie::dev::set_oversample_engine(int(engine));
  return BIE_OK;
}

int bie_get_oversample_engine(void) { return bie::dev::oversample_engine(); }

int bie_plan_oversample(void* plan, int64_t engine, int64_t nd, const double* sigma_dev,
                        float* out_dev, void* stream) {
  if (!plan || !sigma_dev || !out_dev || nd < 1 || (engine != 0 && engine != 1)) return BIE_ERR_ARG;
  return guarded([&] {
    bie::Plan& P = *static_cast<bie::Plan*>(plan);
    if (!P.cplx) {
      bie::set_last_error("bie_plan_oversample: complex (Helmholtz) plans only");
      return BIE_ERR_ARG;
    }
    if (engine == 1 && !bie::dev::oversample_tc_fits(P.g, P.kp, 1, int(nd))) {
      bie::set_last_error("bie_plan_oversample: the tensor-core engine takes nd a multiple of 8 "
                          "up to 128 and patches of at most 64 nodes and 128 far nodes");
      return BIE_ERR_ARG;
    }
    bie::dev::MatvecArgs a;
    a.precision = 1;
    a.nd = int(nd);
    a.sigma = sigma_dev;
    a.strengths = out_dev;
    a.tc_err = P.tc_err_ptr();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const cudaError_t e = engine == 1 ? bie::dev::launch_oversample_tc(P.g, P.kp, a, st)
                                      : bie::dev::launch_oversample(P.g, P.kp, a, st);
    if (e != cudaSuccess) {
      bie::set_last_error(cudaGetErrorString(e));
      return BIE_ERR_CUDA;
    }
    return BIE_OK;
  });
}

int bie_plan_get_far(void* plan, int64_t iprec, int64_t nd, int64_t* out) {
  if (!plan || !out || (iprec != 0 && iprec != 1) || nd < 1) return BIE_ERR_ARG;
  const bie::Plan* P = static_cast<bie::Plan*>(plan);
  const auto c = P->far_config(int(iprec), int(nd));
  out[0] = c.variant;
  out[1] = c.nchunks;
  out[2] = P->tc_error();
  return BIE_OK;
}

int bie_plan_set_far_method(void* plan, int64_t iprec, int64_t method, double theta, int64_t p,
                            int64_t leaf_t, int64_t leaf_s, void* stream) {
  if (!plan || (iprec != 0 && iprec != 1) || (method != 0 && method != 1)) return BIE_ERR_ARG;
  return guarded([&] {
    bie::Plan& P = *static_cast<bie::Plan*>(plan);
    bie::tree::Params prm = bie::Plan::default_tree_params(int(iprec), P.kp);
    if (theta > 0.0) prm.theta = theta;
    if (p > 0) prm.p = int(p);
    if (leaf_t > 0) prm.leaf_t = int(std::min<int64_t>(leaf_t, 1 << 20));
    if (leaf_s > 0) prm.leaf_s = int(std::min<int64_t>(leaf_s, 1 << 20));
    return P.set_far_method(int(iprec), int(method), method == 1 ? &prm : nullptr,
                            static_cast<cudaStream_t>(stream));
  });
}

int bie_plan_get_far_method(void* plan, int64_t iprec, double* out) {
  if (!plan || !out || (iprec != 0 && iprec != 1)) return BIE_ERR_ARG;
  const bie::Plan& P = *static_cast<bie::Plan*>(plan);
  for (int q = 0; q < 16; ++q) out[q] = 0.0;
  out[0] = P.far_method(int(iprec));
  const bie::TreeStats* s = P.tree_stats(int(iprec));
  if (!s) return BIE_OK;
  const bie::tree::Params prm = P.tree_params(int(iprec));
  out[1] = prm.p;
  out[2] = prm.theta;
  out[3] = double(s->tnodes);
  out[4] = double(s->snodes);
  out[5] = double(s->leaves);
  for (int q = 0; q < 5; ++q) out[6 + q] = double(s->interactions[q]);
  out[11] = double(s->source_proxies);
  out[12] = double(s->target_proxies);
  out[13] = s->pair_evals;
  out[14] = s->build_ms;
  out[15] = s->up_evals + s->down_evals;
  return BIE_OK;
}

int bie_tree_check(int64_t nt, const double* targ, int64_t ns, const double* src, double theta,
                   int64_t p, double k, int64_t leaf_t, int64_t leaf_s, double* out) {
  if (nt < 1 || ns < 1 || !targ || !src || !out || !(theta > 0.0 && theta < 1.0) || p < 1 ||
      p > bie::tree::kMaxP || leaf_t < 1 || leaf_s < 1)
    return BIE_ERR_ARG;
  return guarded([&] {
    std::vector<double> tx(nt), ty(nt), tz(nt), sx(ns), sy(ns), sz(ns);
    for (int64_t i = 0; i < nt; ++i) {
      tx[i] = targ[3 * i];
      ty[i] = targ[3 * i + 1];
      tz[i] = targ[3 * i + 2];
    }
    for (int64_t i = 0; i < ns; ++i) {
      sx[i] = src[3 * i];
      sy[i] = src[3 * i + 1];
      sz[i] = src[3 * i + 2];
    }
    bie::tree::Params prm;
    prm.theta = theta;
    prm.p = int(p);
    prm.k = k;
    prm.leaf_t = int(leaf_t);
    prm.leaf_s = int(leaf_s);
    bie::tree::Tree T, S;
    bie::tree::build_tree(nt, tx.data(), ty.data(), tz.data(), prm.leaf_t, T);
    bie::tree::build_tree(ns, sx.data(), sy.data(), sz.data(), prm.leaf_s, S);
    bie::tree::set_proxies(T, prm);
    bie::tree::set_proxies(S, prm);
    std::vector<bie::tree::Interaction> ia;
    bie::tree::traverse(T, S, prm, 0.0, ia);
    for (int q = 0; q < 14; ++q) out[q] = 0.0;
    out[0] = bie::tree::check_coverage(T, S, ia);
    out[1] = double(T.nodes.size());
    out[2] = double(S.nodes.size());
    double evals = 0.0;
    for (const auto& x : ia) {
      out[3 + x.kind] += 1.0;
      const auto& a = T.nodes[x.t];
      const auto& b = S.nodes[x.s];
      const double nt_ = x.kind == bie::tree::kCP || x.kind == bie::tree::kCC ? a.nprox() : a.n();
      const double ns_ = x.kind == bie::tree::kPC || x.kind == bie::tree::kCC ? b.nprox() : b.n();
      evals += nt_ * ns_;
    }
    out[8] = evals;
    out[9] = double(nt) * double(ns);
    int64_t lmin = nt, lmax = 0, capped = 0, broken = 0;
    for (const bie::tree::Tree* tr : {&T, &S})
      for (const auto& nd : tr->nodes) {
        capped += nd.capped ? 1 : 0;
        if (nd.nchild == 0) continue;
        // children are contiguous and tile the parent's range in order
        int64_t pos = nd.b;
        for (int c = 0; c < nd.nchild; ++c) {
          const auto& ch = tr->nodes[nd.child0 + c];
          if (ch.b != pos || ch.parent < 0 || &tr->nodes[ch.parent] != &nd) ++broken;
          pos = ch.e;
        }
        if (pos != nd.e) ++broken;
      }
    for (const auto& nd : T.nodes)
      if (nd.nchild == 0) {
        lmin = std::min<int64_t>(lmin, nd.n());
        lmax = std::max<int64_t>(lmax, nd.n());
      }
    out[10] = double(lmin);
    out[11] = double(lmax);
    out[12] = double(capped);
    out[13] = double(broken);
    return int(bie::kOk);
  });
}

int bie_plan_matvec(void* plan, int64_t iprec, int64_t nd, const double* sigma_dev,
                    double* pot_dev, void* stream) {
  if (!plan || (iprec != 0 && iprec != 1) || nd < 1) return BIE_ERR_ARG;
  return guarded([&] {
    return static_cast<bie::Plan*>(plan)->matvec(int(iprec), int(nd), sigma_dev, pot_dev,
                                                 static_cast<cudaStream_t>(stream));
  });
}

int bie_plan_solve(void* plan, int64_t mode, int64_t nd, const double* zid,
                   const double* rhs_dev, const double* x0_dev, int64_t numit, double eps_gmres,
                   double* soln_dev, int64_t* niter, double* errs, double* rres, void* stream) {
  if (!plan || (mode != 0 && mode != 1) || nd < 1 || nd > 256 || numit < 1) return BIE_ERR_ARG;
  return guarded([&] {
    bie::Plan& P = *static_cast<bie::Plan*>(plan);
    const std::vector<cdouble> z(size_t(nd), cdouble(zid[0], P.cplx ? zid[1] : 0.0));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (mode == 0) {
      bie::GmresOut go;
      const int s = bie::gmres(P, 0, 0, int(nd), z.data(), rhs_dev, x0_dev, numit, eps_gmres,
                               soln_dev, go, st);
      if (s == BIE_OK || s == BIE_NOT_CONVERGED || s == BIE_BREAKDOWN) {
        for (int64_t q = 0; q < nd; ++q) {
          if (niter) niter[q] = go.niter[q];
          if (rres) rres[q] = go.rres[q];
          if (errs)
            for (int64_t j = 0; j <= numit; ++j) errs[q * (numit + 1) + j] = go.errs[q * (numit + 1) + j];
        }
      }
      return s;
    }
    bie::MixedOut mo;
    const int s = bie::solve_mixed(P, int(nd), z.data(), rhs_dev, x0_dev, numit, eps_gmres, 1e-5, 6,
                                   soln_dev, mo, st);
    if (s == BIE_OK || s == BIE_NOT_CONVERGED) {
      for (int64_t q = 0; q < nd; ++q) {
        if (niter) niter[q] = mo.inner_iters[q];
        if (rres) rres[q] = mo.rres[q];
      }
      if (errs) {
        errs[0] = mo.fp64_matvecs;
        errs[1] = mo.fp32_matvecs;
        if (x0_dev && (numit + 1) * nd >= 2 + nd)
          for (int64_t q = 0; q < nd; ++q) errs[2 + q] = double(mo.x0_dropped[q]);
      }
    }
    return s;
  });
}

int bie_set_mixed_residual(int64_t mode) {
  if (mode != 0 && mode != 1) return BIE_ERR_ARG;
  bie::set_mixed_residual_mode(int(mode));
  return BIE_OK;
}

int bie_get_mixed_residual(void) { return bie::mixed_residual_mode(); }

int bie_last_mixed_stats(double* out) {
  if (!out) return BIE_ERR_ARG;
  const bie::MixedOut& m = bie::last_mixed_out();
  out[0] = m.fp64_matvecs;
  out[1] = m.fp32_matvecs;
  out[2] = m.incr_matvecs;
  out[3] = m.max_incr_ratio;
  return BIE_OK;
}

int bie_plan_timing(void* plan, int64_t enable, double* times) {
  if (!plan) return BIE_ERR_ARG;
  bie::Plan& P = *static_cast<bie::Plan*>(plan);
  if (times) {
    for (int p = 0; p < 2; ++p) {
      times[4 * p + 0] = P.times.strengths_ms[p];
      times[4 * p + 1] = P.times.far_ms[p];
      times[4 * p + 2] = P.times.combine_ms[p];
      times[4 * p + 3] = double(P.times.calls[p]);
    }
  }
  if (enable >= 0) {
    P.timing = enable != 0;
    P.times = bie::StageTimes{};
  }
  return BIE_OK;
}

int bie_farfield_dev(int64_t kind, const double* zk, int64_t ns, const double* src_dev,
                     const double* nrm_dev, const double* charge_dev, const double* dipstr_dev,
                     int64_t nt, const double* targ_dev, double thresh, int64_t iprec,
                     double* pot_dev, void* stream) {
  if ((kind != 0 && kind != 1) || (iprec != 0 && iprec != 1) || ns < 0 || nt < 0) {
    bie::set_last_error("bie_farfield_dev: bad kind/iprec/sizes");
    return BIE_ERR_ARG;
  }
  if (nt == 0) return BIE_OK;
  return guarded([&] {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int devn = 0, sms = 148;
    cudaGetDevice(&devn);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, devn);
    bie::dev::Geometry g;
    g.ntarg = nt;
    g.nptso = ns;
    g.tx = targ_dev;
    g.ty = targ_dev + nt;
    g.tz = targ_dev + 2 * nt;
    g.sx = src_dev;
    g.sy = src_dev + ns;
    g.sz = src_dev + 2 * ns;
    g.snx = nrm_dev;
    g.sny = nrm_dev + ns;
    g.snz = nrm_dev + 2 * ns;
    bie::dev::KParams kp;
    kp.kind = int(kind);
    if (kind == 1) {
      kp.kr = zk[0];
      kp.ki = zk[1];
    }
    kp.thresh = thresh;
    const int c = kind == 1 ? 2 : 1;
    // large sums: the hierarchical far field (same selection rule as a plan)
    {
      const char* fm = std::getenv("BIE_FAR_METHOD");
      const std::string m = fm ? fm : "auto";
      const char* tp = std::getenv("BIE_TREE_PAIRS");
      const double pairs_min = tp && *tp ? std::atof(tp) : bie::kTreeAutoPairs;
      if (ns > 0 && (m == "tree" || (m == "auto" && double(ns) * double(nt) >= pairs_min))) {
        bie::TreeFar T;
        const int ier = T.build(g, bie::Plan::default_tree_params(int(iprec), kp), thresh, st);
        if (ier == bie::kOk) {
          bie::DBuf<double> str;
          if (str.alloc(size_t(ns) * 2 * c)) {
            bie::set_last_error("device allocation failed");
            return BIE_ERR_NOMEM;
          }
          cudaError_t e = bie::dev::launch_pack_strengths(int(kind), int(iprec), ns, charge_dev,
                                                          dipstr_dev, str.p, st, T.sdest());
          if (e == cudaSuccess) e = T.run(int(iprec), 1, kp, str.p, pot_dev, st);
          if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // scratch is released below
          if (e != cudaSuccess) {
            bie::set_last_error(cudaGetErrorString(e));
            return BIE_ERR_CUDA;
          }
          return BIE_OK;
        }
        if (ier != bie::kErrArg) return ier;  // else: inputs the trees cannot take
      }
    }
    const int nch = bie::dev::far_nchunks(nt, std::max<int64_t>(ns, 1), int(kind), int(iprec), 1, sms);
    bie::DBuf<double> str, partial;
    if (str.alloc(std::max<int64_t>(ns, 1) * 2 * c) ||
        partial.alloc(size_t(nch) * nt * c)) {
      bie::set_last_error("device allocation failed");
      return BIE_ERR_NOMEM;
    }
    bie::dev::MatvecArgs a;
    a.precision = int(iprec);
    a.nd = 1;
    a.nchunks = nch;
    a.strengths = str.p;
    a.partial = partial.p;
    cudaError_t e = bie::dev::launch_pack_strengths(int(kind), int(iprec), ns, charge_dev,
                                                    dipstr_dev, str.p, st);
    if (e == cudaSuccess) e = bie::dev::launch_far(g, kp, a, st);
    if (e == cudaSuccess) e = bie::dev::launch_reduce_partials(int(kind), partial.p, nch, nt, pot_dev, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // scratch is released below
    if (e != cudaSuccess) {
      bie::set_last_error(cudaGetErrorString(e));
      return BIE_ERR_CUDA;
    }
    return BIE_OK;
  });
}

int64_t bie_launch_count(void) { return bie::dev::launch_count(); }

int bie_measure_fp32_peak(double* tflops, double* ms) {
  return guarded([&] {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int threads = 256, blocks = sms * 8, iters = 4096;
    bie::DBuf<float> out;
    if (out.alloc(size_t(blocks) * threads)) return BIE_ERR_NOMEM;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    bie::dev::launch_ffma_peak(out.p, blocks, threads, iters / 8, 0);  // warm-up
    cudaEventRecord(a, 0);
    bie::dev::launch_ffma_peak(out.p, blocks, threads, iters, 0);
    cudaEventRecord(b, 0);
    cudaEventSynchronize(b);
    float t = 0;
    cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    const double flops = double(blocks) * threads * iters * 16.0 * 8.0 * 2.0;
    *ms = t;
    *tflops = flops / (t * 1e-3) / 1e12;
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? BIE_OK : BIE_ERR_CUDA;
  });
}

int bie_measure_mufu_peak(double* gops, double* ms) {
  return guarded([&] {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int threads = 256, blocks = sms * 8, iters = 1024;
    bie::DBuf<float> out;
    if (out.alloc(size_t(blocks) * threads)) return BIE_ERR_NOMEM;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    bie::dev::launch_mufu_peak(out.p, blocks, threads, iters / 8, 0);  // warm-up
    cudaEventRecord(a, 0);
    bie::dev::launch_mufu_peak(out.p, blocks, threads, iters, 0);
    cudaEventRecord(b, 0);
    cudaEventSynchronize(b);
    float t = 0;
    cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    const double ops = double(blocks) * threads * iters * 16.0 * 8.0;
    *ms = t;
    *gops = ops / (t * 1e-3) / 1e9;
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? BIE_OK : BIE_ERR_CUDA;
  });
}

}  // extern "C"
