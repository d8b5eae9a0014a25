// GMRES and the mixed-precision refinement solver on an Operator: a single
// plan (one segment) or a batch of surfaces (one segment per surface).  Every
// system (segment, density) has its own inner products, Hessenberg matrix,
// Givens rotations and stopping test; all systems share every launch.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include "plan.h"

namespace bie {

namespace {

#define BIE_CUDA(call)                                                             \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_));          \
      return e_ == cudaErrorMemoryAllocation ? kErrNoMem : kErrCuda;               \
    }                                                                              \
  } while (0)

// host complex per system -> interleaved doubles
std::vector<double> interleave(const std::vector<cdouble>& v) {
  std::vector<double> o(2 * v.size());
  for (size_t i = 0; i < v.size(); ++i) {
    o[2 * i] = v[i].real();
    o[2 * i + 1] = v[i].imag();
  }
  return o;
}

}  // namespace

int Operator::init_segments(cudaStream_t st) {
  const int ns = nseg();
  if (ns < 1 || seg_start.front() != 0 || seg_start.back() != nodes) {
    set_last_error("segment table inconsistent with the node count");
    return kErrArg;
  }
  // chunks of about nodes / (2 SMs), at least 64 nodes, never across segments
  const int64_t target = std::max<int64_t>(64, nodes / std::max(1, 2 * num_sms));
  std::vector<int64_t> lo, hi;
  std::vector<int32_t> c0(ns + 1, 0);
  for (int g = 0; g < ns; ++g) {
    c0[g] = int32_t(lo.size());
    const int64_t a = seg_start[g], b = seg_start[g + 1];
    const int64_t nc = std::max<int64_t>(1, (b - a + target - 1) / target);
    for (int64_t c = 0; c < nc; ++c) {
      lo.push_back(a + (b - a) * c / nc);
      hi.push_back(a + (b - a) * (c + 1) / nc);
    }
  }
  c0[ns] = int32_t(lo.size());
  BIE_CUDA(chunk_lo_.alloc(lo.size()));
  BIE_CUDA(chunk_hi_.alloc(hi.size()));
  BIE_CUDA(seg_chunk0_.alloc(c0.size()));
  BIE_CUDA(cudaMemcpyAsync(chunk_lo_.p, lo.data(), lo.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  BIE_CUDA(cudaMemcpyAsync(chunk_hi_.p, hi.data(), hi.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  BIE_CUDA(cudaMemcpyAsync(seg_chunk0_.p, c0.data(), c0.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  segs.nseg = ns;
  segs.nchunk = int(lo.size());
  segs.chunk_lo = chunk_lo_.p;
  segs.chunk_hi = chunk_hi_.p;
  segs.seg_chunk0 = seg_chunk0_.p;
  segs.node_seg = nullptr;
  if (ns > 1) {
    std::vector<int32_t> ns_of(nodes);
    for (int g = 0; g < ns; ++g)
      for (int64_t i = seg_start[g]; i < seg_start[g + 1]; ++i) ns_of[i] = g;
    BIE_CUDA(node_seg_.alloc(ns_of.size()));
    BIE_CUDA(cudaMemcpyAsync(node_seg_.p, ns_of.data(), ns_of.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    segs.node_seg = node_seg_.p;
  }
  // the host vectors above are pageable: finish the copies before they go
  BIE_CUDA(cudaStreamSynchronize(st));
  return kOk;
}

int gmres(Operator& P, int precision, int rres_precision, int nd, const cdouble* zid,
          const double* d_rhs, const double* d_x0, int64_t numit, double eps_gmres,
          double* d_soln, GmresOut& out, cudaStream_t st, const double* eps_sys,
          double* d_res) {
  if (!P.square()) {
    set_last_error("GMRES needs an operator whose targets are its nodes");
    return kErrArg;
  }
  if (numit < 1 || nd < 1 || nd > 256) return kErrArg;
  const int cplx = P.cplx ? 1 : 0;
  const dev::Segs& sg = P.segs;
  const int nsys = sg.nseg * nd;
  const int64_t n = P.nodes * nd;
  const int64_t ldv = n * (cplx ? 2 : 1);
  GmresWorkspace& ws = P.gws;
  BIE_CUDA(ws.V.alloc(size_t(ldv) * (numit + 1)));
  BIE_CUDA(ws.w.alloc(size_t(ldv)));
  BIE_CUDA(ws.partial.alloc(size_t(2) * (numit + 1) * nd * sg.nchunk));
  BIE_CUDA(ws.dots.alloc(size_t(2) * 3 * (numit + 1) * nsys));
  BIE_CUDA(ws.coef.alloc(size_t(2) * (numit + 1) * nsys));
  BIE_CUDA(ws.scale.alloc(size_t(2) * 2 * nsys));
  double* d_h1 = ws.dots.p;
  double* d_h2 = ws.dots.p + 2 * (numit + 1) * nsys;
  double* d_nrm = ws.dots.p + 4 * (numit + 1) * nsys;
  double* d_zid = ws.scale.p + 2 * nsys;  // zid per system
  const double* wts = P.d_node_wts;
  double* V = ws.V.p;
  std::vector<cdouble> zv(zid, zid + nsys);
  {
    const std::vector<double> zh = interleave(zv);
    BIE_CUDA(cudaMemcpyAsync(d_zid, zh.data(), zh.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  // residual start: r0 = rhs - (zid x0 + K x0)  (stored in V_0 before scaling)
  if (d_x0) {
    int ier = P.apply(precision, nd, d_x0, V, st);
    if (ier) return ier;
    // V0 = zid x0 + K x0, then V0 = rhs - V0
    BIE_CUDA(dev::launch_axpbys(d_x0, V, d_zid, 1.0, 0.0, n, nd, cplx, sg, st));
    BIE_CUDA(dev::launch_axpby(d_rhs, V, 1.0, 0.0, -1.0, 0.0, n, cplx, st));
  } else {
    BIE_CUDA(cudaMemcpyAsync(V, d_rhs, ldv * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }
  BIE_CUDA(dev::launch_mdot(V, ldv, 1, V, wts, nd, cplx, sg, ws.partial.p, d_nrm, st));
  std::vector<double> hbuf(2 * nsys);
  BIE_CUDA(cudaMemcpyAsync(hbuf.data(), d_nrm, 2 * nsys * sizeof(double), cudaMemcpyDeviceToHost, st));
  BIE_CUDA(cudaStreamSynchronize(st));
  std::vector<double> rb(nsys), bnorm(nsys);
  std::vector<double> hscale(2 * nsys, 0.0);
  for (int q = 0; q < nsys; ++q) {
    rb[q] = std::sqrt(std::max(hbuf[2 * q], 0.0));
    hscale[2 * q] = rb[q] > 0 ? 1.0 / rb[q] : 0.0;
    bnorm[q] = rb[q];
  }
  // With an initial guess the stopping test stays relative to ||rhs||_w, so a
  // warm-started solve meets the same accuracy as one from zero.
  if (d_x0) {
    BIE_CUDA(dev::launch_mdot(d_rhs, ldv, 1, d_rhs, wts, nd, cplx, sg, ws.partial.p, d_nrm, st));
    std::vector<double> hb(2 * nsys);
    BIE_CUDA(cudaMemcpyAsync(hb.data(), d_nrm, 2 * nsys * sizeof(double), cudaMemcpyDeviceToHost, st));
    BIE_CUDA(cudaStreamSynchronize(st));
    for (int q = 0; q < nsys; ++q) bnorm[q] = std::sqrt(std::max(hb[2 * q], 0.0));
  }
  BIE_CUDA(cudaMemcpyAsync(ws.scale.p, hscale.data(), 2 * nsys * sizeof(double), cudaMemcpyHostToDevice, st));
  BIE_CUDA(dev::launch_dscale(V, V, ws.scale.p, n, nd, cplx, sg, st));
  // Per-system Hessenberg columns, rotations and residual vector live on the
  // device; the Givens step and the back-substitution run there in FP64, and
  // the host reads back only the per-system stop flags each iteration.
  const int64_t M = numit;
  const size_t nH = size_t(2) * nsys * (M + 1) * M, nR = size_t(2) * nsys * M,
               nS = size_t(2) * nsys * (M + 1), nE = size_t(nsys) * (M + 1);
  BIE_CUDA(ws.ls.alloc(nH + 2 * nR + nS + 2 * size_t(nsys) + nE));
  BIE_CUDA(ws.done.alloc(nsys));
  BIE_CUDA(ws.brk.alloc(nsys));
  double* d_H = ws.ls.p;
  double* d_cs = d_H + nH;
  double* d_sn = d_cs + nR;
  double* d_sv = d_sn + nR;
  double* d_bnorm = d_sv + nS;
  double* d_eps = d_bnorm + nsys;
  double* d_errs = d_eps + nsys;
  std::vector<int64_t> done(nsys, 0);
  std::vector<double> sv0(2 * nsys, 0.0), epsv(nsys);
  int nactive = 0;
  for (int q = 0; q < nsys; ++q) {
    sv0[2 * q] = rb[q];
    epsv[q] = eps_sys ? eps_sys[q] : eps_gmres;
    if (rb[q] == 0.0) done[q] = -1;  // zero right-hand side: solution 0
    else ++nactive;
  }
  // s(0) of system q = ||r0||; the rest of s is written as the rotations go
  BIE_CUDA(cudaMemcpy2DAsync(d_sv, 2 * (M + 1) * sizeof(double), sv0.data(), 2 * sizeof(double),
                             2 * sizeof(double), nsys, cudaMemcpyHostToDevice, st));
  BIE_CUDA(cudaMemcpyAsync(d_bnorm, bnorm.data(), nsys * sizeof(double), cudaMemcpyHostToDevice, st));
  BIE_CUDA(cudaMemcpyAsync(d_eps, epsv.data(), nsys * sizeof(double), cudaMemcpyHostToDevice, st));
  BIE_CUDA(cudaMemcpyAsync(ws.done.p, done.data(), nsys * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  BIE_CUDA(cudaMemsetAsync(d_errs, 0, nE * sizeof(double), st));
  BIE_CUDA(cudaMemsetAsync(ws.brk.p, 0, nsys * sizeof(int), st));
  out.niter.assign(nsys, 0);
  out.errs.assign(nE, 0.0);
  out.rres.assign(nsys, 0.0);
  out.status = kOk;
  std::vector<double> hn(2 * nsys);
  int64_t it = 0;
  for (; it < M && nactive > 0; ++it) {
    double* vit = V + size_t(it) * ldv;
    double* vnext = V + size_t(it + 1) * ldv;
    // segments whose systems have all converged skip their matvec work
    std::vector<uint8_t> act(sg.nseg, 0);
    for (int q = 0; q < nsys; ++q)
      if (done[q] == 0) act[q / nd] = 1;
    int ier = P.set_active(act, st);
    if (ier) return ier;
    ier = P.apply(precision, nd, vit, ws.w.p, st);
    if (ier) return ier;
    const int m = int(it + 1);
    BIE_CUDA(dev::launch_mdot(V, ldv, m, ws.w.p, wts, nd, cplx, sg, ws.partial.p, d_h1, st));
    BIE_CUDA(dev::launch_maxpy(V, ldv, m, d_h1, ws.w.p, n, nd, cplx, sg, st));
    BIE_CUDA(dev::launch_mdot(V, ldv, m, ws.w.p, wts, nd, cplx, sg, ws.partial.p, d_h2, st));
    BIE_CUDA(dev::launch_maxpy(V, ldv, m, d_h2, ws.w.p, n, nd, cplx, sg, st));
    BIE_CUDA(dev::launch_mdot(ws.w.p, ldv, 1, ws.w.p, wts, nd, cplx, sg, ws.partial.p, d_nrm, st));
    BIE_CUDA(dev::launch_gmres_givens(int(it), int(M), nsys, d_h1, d_h2, d_nrm, d_zid, d_H, d_cs,
                                      d_sn, d_sv, d_bnorm, d_eps, ws.done.p, ws.brk.p, d_errs,
                                      ws.scale.p, st));
    BIE_CUDA(dev::launch_dscale(ws.w.p, vnext, ws.scale.p, n, nd, cplx, sg, st));
    BIE_CUDA(cudaMemcpyAsync(done.data(), ws.done.p, nsys * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    BIE_CUDA(cudaStreamSynchronize(st));
    nactive = 0;
    for (int q = 0; q < nsys; ++q) nactive += done[q] == 0 ? 1 : 0;
  }
  {
    int ier = P.set_active(std::vector<uint8_t>(sg.nseg, 1), st);
    if (ier) return ier;
  }
  // back-substitution per system on the device: y = triu(H)\s, soln = V y (+ x0)
  const int mused = int(std::max<int64_t>(it, 1));
  BIE_CUDA(dev::launch_gmres_backsolve(int(M), nsys, mused, d_H, d_sv, ws.done.p, ws.coef.p, st));
  BIE_CUDA(dev::launch_combo(V, ldv, mused, ws.coef.p, d_soln, n, nd, cplx, sg, st));
  if (d_res) {
    // r0 - A V y = V_{0..mused} z: the Krylov vectors V_0 .. V_done of each
    // system (the last one normalised by the Givens step) and z from the
    // rotations
    BIE_CUDA(ws.zc.alloc(size_t(2) * (M + 1) * nsys));
    BIE_CUDA(dev::launch_gmres_resvec(int(M), nsys, mused + 1, d_cs, d_sn, d_sv, ws.done.p,
                                      ws.zc.p, st));
    BIE_CUDA(dev::launch_combo(V, ldv, mused + 1, ws.zc.p, d_res, n, nd, cplx, sg, st));
  }
  std::vector<int> brk(nsys);
  BIE_CUDA(cudaMemcpyAsync(out.errs.data(), d_errs, nE * sizeof(double), cudaMemcpyDeviceToHost, st));
  BIE_CUDA(cudaMemcpyAsync(brk.data(), ws.brk.p, nsys * sizeof(int), cudaMemcpyDeviceToHost, st));
  BIE_CUDA(cudaStreamSynchronize(st));
  for (int q = 0; q < nsys; ++q)
    if (brk[q]) out.status = kBreakdown;
  for (int q = 0; q < nsys; ++q) {
    if (done[q] <= 0) continue;
    const int64_t k = done[q];
    out.niter[q] = k;
    if (out.errs[size_t(q) * (M + 1) + k - 1] > epsv[q] && out.status == kOk)
      out.status = kNotConverged;
  }
  if (d_x0) BIE_CUDA(dev::launch_axpby(d_x0, d_soln, 1.0, 0.0, 1.0, 0.0, n, cplx, st));
  // rres = || zid x + K x - rhs ||_w / ||rhs||_w   (one more matvec)
  if (rres_precision >= 0) {
    int ier = P.apply(rres_precision, nd, d_soln, ws.w.p, st);
    if (ier) return ier;
    BIE_CUDA(dev::launch_axpbys(d_soln, ws.w.p, d_zid, 1.0, 0.0, n, nd, cplx, sg, st));
    BIE_CUDA(dev::launch_axpby(d_rhs, ws.w.p, -1.0, 0.0, 1.0, 0.0, n, cplx, st));
    BIE_CUDA(dev::launch_mdot(ws.w.p, ldv, 1, ws.w.p, wts, nd, cplx, sg, ws.partial.p, d_nrm, st));
    BIE_CUDA(cudaMemcpyAsync(hn.data(), d_nrm, 2 * nsys * sizeof(double), cudaMemcpyDeviceToHost, st));
    // ||rhs|| (the initial residual norm is ||rhs - A x0||, not ||rhs||)
    BIE_CUDA(dev::launch_mdot(d_rhs, ldv, 1, d_rhs, wts, nd, cplx, sg, ws.partial.p, d_h1, st));
    std::vector<double> hr(2 * nsys);
    BIE_CUDA(cudaMemcpyAsync(hr.data(), d_h1, 2 * nsys * sizeof(double), cudaMemcpyDeviceToHost, st));
    BIE_CUDA(cudaStreamSynchronize(st));
    for (int q = 0; q < nsys; ++q) {
      const double rn = std::sqrt(std::max(hr[2 * q], 0.0));
      out.rres[q] = rn > 0 ? std::sqrt(std::max(hn[2 * q], 0.0)) / rn : 0.0;
    }
  }
  return out.status;
}

namespace {
std::atomic<int> g_mixed_mode{-1};
thread_local MixedOut t_last_mixed;
}  // namespace

int mixed_residual_mode() {
  int m = g_mixed_mode.load();
  if (m < 0) {
    const char* e = std::getenv("BIE_MIXED_RESIDUAL");
    m = (e && std::string(e) == "full") ? 0 : 1;
    g_mixed_mode.store(m);
  }
  return m;
}

void set_mixed_residual_mode(int mode) { g_mixed_mode.store(mode ? 1 : 0); }

const MixedOut& last_mixed_out() { return t_last_mixed; }

static int solve_mixed_impl(Operator& P, int nd, const cdouble* zid, const double* d_rhs,
                            const double* d_x0, int64_t numit, double eps_target,
                            double inner_floor, int max_outer, double* d_soln, MixedOut& out,
                            cudaStream_t st);

int solve_mixed(Operator& P, int nd, const cdouble* zid, const double* d_rhs, const double* d_x0,
                int64_t numit, double eps_target, double inner_floor, int max_outer,
                double* d_soln, MixedOut& out, cudaStream_t st) {
  const int s = solve_mixed_impl(P, nd, zid, d_rhs, d_x0, numit, eps_target, inner_floor,
                                 max_outer, d_soln, out, st);
  t_last_mixed = out;
  return s;
}

static int solve_mixed_impl(Operator& P, int nd, const cdouble* zid, const double* d_rhs,
                            const double* d_x0, int64_t numit, double eps_target,
                            double inner_floor, int max_outer, double* d_soln, MixedOut& out,
                            cudaStream_t st) {
  if (!P.square()) {
    set_last_error("the solver needs an operator whose targets are its nodes");
    return kErrArg;
  }
  if (nd < 1 || nd > 256) return kErrArg;
  const int cplx = P.cplx ? 1 : 0;
  const dev::Segs& sg = P.segs;
  const int nsys = sg.nseg * nd;
  const int64_t n = P.nodes * nd;
  const int64_t ldv = n * (cplx ? 2 : 1);
  // buffers live in the operator: after the first solve no call allocates (a
  // cudaFree would synchronise the device and serialise concurrent solves)
  DBuf<double>& r = P.mws.r;
  DBuf<double>& d = P.mws.d;
  DBuf<double>& partial = P.mws.partial;
  DBuf<double>& nrm = P.mws.nrm;
  DBuf<double>& kx = P.mws.kx;  // K x in FP64 (see MixedOut)
  DBuf<double>& rn = P.mws.rn;  // an inner solve's own residual vector
  BIE_CUDA(r.alloc(ldv));
  BIE_CUDA(d.alloc(ldv));
  BIE_CUDA(kx.alloc(ldv));
  BIE_CUDA(partial.alloc(size_t(2) * nd * sg.nchunk));
  BIE_CUDA(nrm.alloc(size_t(8) * nsys));
  double* d_zid = nrm.p + 4 * nsys;  // zid per system
  {
    std::vector<cdouble> zv(zid, zid + nsys);
    const std::vector<double> zh = interleave(zv);
    BIE_CUDA(cudaMemcpyAsync(d_zid, zh.data(), zh.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  out.inner_iters.assign(nsys, 0);
  out.outer.assign(nsys, 0);
  out.rres.assign(nsys, 1.0);
  out.fp64_matvecs = out.fp32_matvecs = out.incr_matvecs = 0;
  out.max_incr_ratio = 0.0;
  out.status = kOk;
  const bool increments = mixed_residual_mode() == 1;
  bool kx_valid = false;
  const double* wts = P.d_node_wts;
  // r = rhs - (zid x + K x) from K x already in r
  auto finish_residual = [&]() -> int {
    BIE_CUDA(dev::launch_axpbys(d_soln, r.p, d_zid, 1.0, 0.0, n, nd, cplx, sg, st));
    BIE_CUDA(dev::launch_axpby(d_rhs, r.p, 1.0, 0.0, -1.0, 0.0, n, cplx, st));
    return kOk;
  };
  // ||rhs||_w per system
  std::vector<double> hb(2 * nsys), hr(2 * nsys);
  BIE_CUDA(dev::launch_mdot(d_rhs, ldv, 1, d_rhs, wts, nd, cplx, sg, partial.p, nrm.p, st));
  BIE_CUDA(cudaMemcpyAsync(hb.data(), nrm.p, 2 * nsys * sizeof(double), cudaMemcpyDeviceToHost, st));
  // x = x0 or 0; r = rhs - (zid x + K x).  The residual of a guess is taken
  // with the FP32 operator: it only seeds the first correction, and every
  // convergence decision below is made on an FP64 residual.
  bool r_is_f64 = true;
  std::vector<double> bn(nsys);
  out.x0_dropped.assign(nsys, 0);
  if (d_x0) {
    BIE_CUDA(cudaMemcpyAsync(d_soln, d_x0, ldv * sizeof(double), cudaMemcpyDeviceToDevice, st));
    int ier = P.apply(1, nd, d_soln, r.p, st);
    if (ier) return ier;
    ++out.fp32_matvecs;
    if ((ier = finish_residual())) return ier;
    r_is_f64 = false;
    // fallback per system: a guess whose residual is not below ||rhs|| is
    // replaced by zero (x = 0, r = rhs)
    BIE_CUDA(dev::launch_mdot(r.p, ldv, 1, r.p, wts, nd, cplx, sg, partial.p, nrm.p, st));
    BIE_CUDA(cudaMemcpyAsync(hr.data(), nrm.p, 2 * nsys * sizeof(double), cudaMemcpyDeviceToHost, st));
    BIE_CUDA(cudaStreamSynchronize(st));
    std::vector<double> keep(2 * nsys, 0.0), drop(2 * nsys, 0.0);
    bool any_drop = false;
    for (int q = 0; q < nsys; ++q) {
      const double b = std::sqrt(std::max(hb[2 * q], 0.0));
      const double rr = std::sqrt(std::max(hr[2 * q], 0.0));
      const bool ok = rr < b;
      keep[2 * q] = ok ? 1.0 : 0.0;
      drop[2 * q] = ok ? 0.0 : 1.0;
      if (!ok) {
        any_drop = true;
        out.x0_dropped[q] = 1;
      }
    }
    if (any_drop) {
      double* s = nrm.p + 2 * nsys;
      BIE_CUDA(cudaMemcpyAsync(s, keep.data(), 2 * nsys * sizeof(double), cudaMemcpyHostToDevice, st));
      BIE_CUDA(dev::launch_dscale(d_soln, d_soln, s, n, nd, cplx, sg, st));
      BIE_CUDA(dev::launch_dscale(r.p, r.p, s, n, nd, cplx, sg, st));
      BIE_CUDA(cudaStreamSynchronize(st));
      BIE_CUDA(cudaMemcpyAsync(s, drop.data(), 2 * nsys * sizeof(double), cudaMemcpyHostToDevice, st));
      BIE_CUDA(dev::launch_dscale(d_rhs, d.p, s, n, nd, cplx, sg, st));
      BIE_CUDA(dev::launch_axpby(d.p, r.p, 1.0, 0.0, 1.0, 0.0, n, cplx, st));
    }
  } else {
    BIE_CUDA(cudaMemsetAsync(d_soln, 0, ldv * sizeof(double), st));
    BIE_CUDA(cudaMemcpyAsync(r.p, d_rhs, ldv * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }
  BIE_CUDA(cudaStreamSynchronize(st));
  for (int q = 0; q < nsys; ++q) bn[q] = std::sqrt(std::max(hb[2 * q], 0.0));
  // frozen[q]: an FP64 residual has shown system q at the target; it sits
  // out the remaining refinement steps (zero inner residual, and in a batch
  // its surface skips the FP64 residual matvecs once all its systems froze)
  std::vector<uint8_t> frozen(nsys, 0);
  auto seg_mask = [&]() {
    std::vector<uint8_t> act(sg.nseg, 0);
    for (int q = 0; q < nsys; ++q)
      if (!frozen[q]) act[q / nd] = 1;
    return act;
  };
  int ier = kOk;
  for (int outer = 0; outer <= max_outer; ++outer) {
    BIE_CUDA(dev::launch_mdot(r.p, ldv, 1, r.p, wts, nd, cplx, sg, partial.p, nrm.p, st));
    BIE_CUDA(cudaMemcpyAsync(hr.data(), nrm.p, 2 * nsys * sizeof(double), cudaMemcpyDeviceToHost, st));
    BIE_CUDA(cudaStreamSynchronize(st));
    double worst_ratio = 0.0;
    bool all_done = true;
    for (int q = 0; q < nsys; ++q) {
      if (frozen[q]) continue;  // keeps its last FP64 relative residual
      const double rel = bn[q] > 0 ? std::sqrt(std::max(hr[2 * q], 0.0)) / bn[q] : 0.0;
      out.rres[q] = rel;
      if (rel > eps_target) {
        all_done = false;
        worst_ratio = std::max(worst_ratio, eps_target / rel);
      } else if (r_is_f64) {
        frozen[q] = 1;
      }
    }
    if (!r_is_f64 && all_done) {
      // the guess already meets the target in FP32: confirm it in FP64
      if ((ier = P.set_active(std::vector<uint8_t>(sg.nseg, 1), st))) return ier;
      if ((ier = P.apply(0, nd, d_soln, kx.p, st))) return ier;
      ++out.fp64_matvecs;
      kx_valid = true;
      BIE_CUDA(cudaMemcpyAsync(r.p, kx.p, ldv * sizeof(double), cudaMemcpyDeviceToDevice, st));
      if ((ier = finish_residual())) return ier;
      r_is_f64 = true;
      continue;
    }
    if (r_is_f64 && (all_done || outer == max_outer)) {
      if (!all_done) out.status = kNotConverged;
      break;
    }
    // inner relative tolerance per system: what this step must gain for that
    // system, not below the accuracy the f32 operator can deliver
    const double tol = std::max(inner_floor, 0.5 * worst_ratio);
    std::vector<double> tol_sys(nsys, tol);
    for (int q = 0; q < nsys; ++q)
      if (out.rres[q] > eps_target) tol_sys[q] = std::max(inner_floor, 0.5 * eps_target / out.rres[q]);
    // systems at the target (frozen, or below it in an FP32 residual) sit
    // this inner solve out: a zero residual makes GMRES skip them
    {
      std::vector<double> keep(2 * nsys, 0.0);
      bool any = false;
      for (int q = 0; q < nsys; ++q) {
        keep[2 * q] = (!frozen[q] && out.rres[q] > eps_target) ? 1.0 : 0.0;
        any = any || keep[2 * q] == 0.0;
      }
      if (any) {
        double* sk = nrm.p + 2 * nsys;
        BIE_CUDA(cudaMemcpyAsync(sk, keep.data(), 2 * nsys * sizeof(double), cudaMemcpyHostToDevice, st));
        BIE_CUDA(dev::launch_dscale(r.p, r.p, sk, n, nd, cplx, sg, st));
      }
    }
    GmresOut go;
    const bool want_rn = increments && kx_valid;
    if (want_rn) BIE_CUDA(rn.alloc(ldv));
    ier = gmres(P, 1, -1, nd, zid, r.p, nullptr, numit, tol, d.p, go, st, tol_sys.data(),
                want_rn ? rn.p : nullptr);
    if (ier && ier != kNotConverged) return ier;
    int64_t maxit = 0;
    for (int q = 0; q < nsys; ++q) {
      if (frozen[q]) continue;
      out.inner_iters[q] += go.niter[q];
      out.outer[q] += 1;
      maxit = std::max(maxit, go.niter[q]);
    }
    out.fp32_matvecs += int(maxit);
    // x += d ; r = rhs - (zid x + K x) for the systems still refined
    // (frozen surfaces of a batch skip the matvec; their r is not read again)
    BIE_CUDA(dev::launch_axpby(d.p, d_soln, 1.0, 0.0, 1.0, 0.0, n, cplx, st));
    bool incr = false;
    double ratio_max = 0.0;
    if (increments && kx_valid) {
      // ||d||_w and ||x||_w per system decide whether K x may be updated
      // with the FP32 operator applied to d
      std::vector<double> hd(2 * nsys), hx(2 * nsys);
      BIE_CUDA(dev::launch_mdot(d.p, ldv, 1, d.p, wts, nd, cplx, sg, partial.p, nrm.p, st));
      BIE_CUDA(cudaMemcpyAsync(hd.data(), nrm.p, 2 * nsys * sizeof(double), cudaMemcpyDeviceToHost, st));
      BIE_CUDA(dev::launch_mdot(d_soln, ldv, 1, d_soln, wts, nd, cplx, sg, partial.p,
                                nrm.p + 6 * nsys, st));
      BIE_CUDA(cudaMemcpyAsync(hx.data(), nrm.p + 6 * nsys, 2 * nsys * sizeof(double),
                               cudaMemcpyDeviceToHost, st));
      BIE_CUDA(cudaStreamSynchronize(st));
      incr = true;
      for (int q = 0; q < nsys; ++q) {
        if (frozen[q]) continue;
        const double xn = std::sqrt(std::max(hx[2 * q], 0.0));
        const double dn = std::sqrt(std::max(hd[2 * q], 0.0));
        const double ratio = xn > 0 ? dn / xn : (dn > 0 ? 1.0 : 0.0);
        ratio_max = std::max(ratio_max, ratio);
        if (kFp32OpErr * ratio > 0.25 * eps_target) incr = false;
      }
    }
    if ((ier = P.set_active(seg_mask(), st))) return ier;
    if (incr) {
      // K32 d = A32 d - zid d = (r - rn) - zid d, with rn = r - A32 d the
      // inner solve's residual vector from its Krylov basis: no matvec
      BIE_CUDA(dev::launch_kx_update(kx.p, r.p, rn.p, d.p, d_zid, n, nd, cplx, sg, st));
      ++out.incr_matvecs;
      out.max_incr_ratio = std::max(out.max_incr_ratio, ratio_max);
    } else {
      ier = P.apply(0, nd, d_soln, kx.p, st);
      if (ier) return ier;
      ++out.fp64_matvecs;
      kx_valid = true;
    }
    if ((ier = P.set_active(std::vector<uint8_t>(sg.nseg, 1), st))) return ier;
    BIE_CUDA(cudaMemcpyAsync(r.p, kx.p, ldv * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if ((ier = finish_residual())) return ier;
    r_is_f64 = true;
  }
  if ((ier = P.set_active(std::vector<uint8_t>(sg.nseg, 1), st))) return ier;
  return out.status;
}

}  // namespace bie
