// Device-resident operator plan for lpcomp_{lap,helm}_comb_dir_addsub and the
// GMRES solvers built on it.
#pragma once
#include <complex>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "../host/tree.h"
#include "device.cuh"

namespace bie {

class TreeFar;
struct TreeStats;

// Default problem size (targets x oversampled sources) from which a plan
// uses the hierarchical far field.
constexpr double kTreeAutoPairs = 1.5e10;

using cdouble = std::complex<double>;

// Status codes shared with the C-ABI (include/fmm3dbie_b200.h).
enum Status {
  kOk = 0,
  kErrArg = 1,
  kErrCuda = 2,
  kNotConverged = 3,
  kBreakdown = 4,
  kErrNoMem = 5,
  kErrTables = 6,
  kErrSingular = 7,
  kErrTimeout = 8,
};

void set_last_error(const std::string& msg);
const char* last_error();

// Stream on which the calling thread's DBuf allocations are stream-ordered
// (cudaMallocAsync / cudaFreeAsync from the device's default memory pool,
// which keeps freed memory for reuse); null means cudaMalloc / cudaFree.
cudaStream_t& alloc_stream();
// Sets alloc_stream() for a scope.  Used by entry points that build a plan,
// run it and release it on one private stream: their buffers come back to
// the pool without a device-wide synchronisation, and the next call reuses
// them.  Every buffer allocated in the scope must be released before the
// stream is destroyed.
struct AllocStreamScope {
  cudaStream_t prev;
  explicit AllocStreamScope(cudaStream_t s);
  ~AllocStreamScope() { alloc_stream() = prev; }
  AllocStreamScope(const AllocStreamScope&) = delete;
  AllocStreamScope& operator=(const AllocStreamScope&) = delete;
};

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t st = nullptr;  // stream of a stream-ordered allocation
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  cudaError_t alloc(size_t count) {
    if (count <= n && p) return cudaSuccess;
    release();
    if (count == 0) return cudaSuccess;
    cudaStream_t s = alloc_stream();
    cudaError_t e = s ? cudaMallocAsync(reinterpret_cast<void**>(&p), count * sizeof(T), s)
                      : cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    n = count;
    st = s;
    return cudaSuccess;
  }
  void release() {
    if (p) {
      if (st)
        cudaFreeAsync(p, st);
      else
        cudaFree(p);
    }
    p = nullptr;
    n = 0;
    st = nullptr;
  }
};

// Host description of one operator (reference calling sequence, 1-based
// index arrays, complex values interleaved).
struct PlanSpec {
  int kind = 0;  // 0 Laplace, 1 Helmholtz
  cdouble zk = 0, alpha = 1, beta = 1;
  int64_t npatches = 0, npts = 0;
  const int64_t* norders = nullptr;
  const int64_t* ixyzs = nullptr;
  const int64_t* iptype = nullptr;
  const double* srccoefs = nullptr;
  const double* srcvals = nullptr;
  int ndtarg = 12;
  int64_t ntarg = 0;
  const double* targs = nullptr;  // ndtarg x ntarg
  int64_t nnz = 0, nquad = 0;
  const int64_t* row_ptr = nullptr;
  const int64_t* col_ind = nullptr;
  const int64_t* iquad = nullptr;
  const double* wnear = nullptr;  // nquad reals (Laplace) or 2*nquad (Helmholtz)
  const int64_t* novers = nullptr;
  int64_t nptso = 0;
  const int64_t* ixyzso = nullptr;
  const double* srcover = nullptr;  // 12 x nptso
  const double* whtsover = nullptr;
  bool keep_f32 = true;  // also keep an f32 copy of W_eff
  // Upload the near quadrature and fold W_eff on a second stream that the
  // plan's matvecs wait on at their near correction (an event), so that a
  // solve started right after the build runs its first far field while the
  // near quadrature is still on its way.  Only for plans whose W_eff is read
  // through Plan::matvec (not the batch engine).
  bool async_weff = false;
};

struct GmresWorkspace {
  DBuf<double> V, w, partial, dots, coef, scale;
  // least squares on the device: Hessenberg columns, rotations, residual
  // vector, norms, tolerances and error history per system
  DBuf<double> ls;
  DBuf<int64_t> done;
  DBuf<int> brk;
  DBuf<double> zc;  // Krylov-basis coefficients of the residual vector
};

struct MixedWorkspace {
  DBuf<double> r, d, partial, nrm, kx, rn;
};

// Per-precision stage totals (index 0 = f64 matvecs, 1 = f32 matvecs).
struct StageTimes {
  double strengths_ms[2] = {0, 0}, far_ms[2] = {0, 0}, combine_ms[2] = {0, 0};
  int64_t calls[2] = {0, 0};
};

// A linear operator K of the second-kind systems (zid I + K) x = b.
// Vectors hold `nodes` nodes x nd densities (point-major).  The nodes form
// segments (the surfaces of a batch, one for a single plan): system
// (segment g, density d) is independent of the others, so the solvers run
// nseg * nd systems with their own inner products, Hessenberg matrices and
// stopping tests.
class Operator {
 public:
  virtual ~Operator() = default;
  // y = K x for nd densities; precision 0 = f64, 1 = f32 far field + f32 W_eff.
  virtual int apply(int precision, int nd, const double* x, double* y, cudaStream_t st) = 0;
  // whether the operator maps node values to node values (GMRES needs it)
  virtual bool square() const = 0;
  // Segments whose systems have all converged (active[g] == 0) may skip
  // their work in later apply() calls; their output is then zero.  The
  // default does the full work.
  virtual int set_active(const std::vector<uint8_t>& active, cudaStream_t st) {
    (void)active;
    (void)st;
    return 0;
  }

  bool cplx = false;
  int device = 0, num_sms = 148;
  int64_t nodes = 0;                      // rows per density
  const double* d_node_wts = nullptr;     // smooth quadrature weight per node (device)
  std::vector<int64_t> seg_start{0, 0};   // host, nseg + 1 node offsets
  int nseg() const { return int(seg_start.size()) - 1; }
  // device reduction tables for seg_start (chunks of about nodes/(2 SMs));
  // call after seg_start and nodes are set
  int init_segments(cudaStream_t st);
  dev::Segs segs;

  GmresWorkspace gws;  // reused across solves
  MixedWorkspace mws;

 private:
  DBuf<int64_t> chunk_lo_, chunk_hi_;
  DBuf<int32_t> seg_chunk0_, node_seg_;
};

class Plan : public Operator {
 public:
  Plan();
  ~Plan() override;
  Plan(const Plan&) = delete;
  Plan& operator=(const Plan&) = delete;
  int kind = 0;
  dev::KParams kp;
  dev::Geometry g;
  dev::Near nr;
  int64_t npts = 0, ntarg = 0, nptso = 0, npatches = 0, nnz = 0, nquad = 0;
  bool targets_on_surface = false;

  int build(const PlanSpec& spec, cudaStream_t st);
  // pot = K sigma (principal value, no identity term), nd densities,
  // precision 0 = f64, 1 = f32 far field + f32 W_eff.
  int matvec(int precision, int nd, const double* d_sigma, double* d_pot, cudaStream_t st);
  int apply(int precision, int nd, const double* x, double* y, cudaStream_t st) override {
    return matvec(precision, nd, x, y, st);
  }
  bool square() const override { return targets_on_surface && ntarg == npts; }
  int nchunks_for(int precision, int nd) const;

  // Far-kernel launch shape: block-shape variant and number of source
  // chunks.  Chosen on first use per (precision, nd) by timing the
  // candidates on this plan's data (cached process-wide per problem shape);
  // BIE_FAR_VARIANT / BIE_FAR_WAVES fix it, BIE_AUTOTUNE=0 uses the default.
  struct FarConfig {
    int variant = 0, nchunks = 1;
    double ms = 0;
  };
  FarConfig far_config(int precision, int nd) const;
  // Pins the far-field shape and chunk count of (precision, nd) instead of
  // tuning it; variant as dev::far_variants().
  int set_far_config(int precision, int nd, int variant, int nchunks);
  // Nonzero once a tensor-core far-field launch timed out waiting for its MMAs.
  int tc_error() const;
  int* tc_err_ptr() { return tc_err_.p; }
  // makes st wait for W_eff (a no-op unless the plan was built with async_weff)
  int wait_weff(cudaStream_t st);
  // several-density oversampling of a matvec on the engine of
  // dev::oversample_engine() (a.tc_err is the plan's flag)
  cudaError_t oversample(const dev::MatvecArgs& a, cudaStream_t st);
  // Far-field method of a precision: 0 = direct sum over all pairs (the
  // kernels above), 1 = hierarchical (dual-tree barycentric Lagrange
  // interpolation, tree_far.h).  Chosen at build from the problem size
  // (BIE_FAR_METHOD = direct | tree | auto, BIE_TREE_PAIRS the threshold on
  // ntarg * nptso); set_far_method switches it and, for precision 1,
  // refolds the FP32 W_eff for the new FP32 centring.  prm: tree
  // parameters (null: defaults of the precision).
  int set_far_method(int precision, int method, const tree::Params* prm, cudaStream_t st);
  int far_method(int precision) const { return far_method_[precision & 1]; }
  const TreeStats* tree_stats(int precision) const;
  tree::Params tree_params(int precision) const;
  static tree::Params default_tree_params(int precision, const dev::KParams& kp);
  const double* d_wts() const { return wts_.p; }
  // W_eff and the per-source (a, b) constants for precision 0 (f64) / 1 (f32)
  const void* weff_ptr(int precision) const {
    return precision == 1 ? static_cast<const void*>(weff32_.p) : static_cast<const void*>(weff64_.p);
  }
  const void* ab_ptr(int precision) const {
    return precision == 1 ? static_cast<const void*>(ab32_.p) : static_cast<const void*>(ab64_.p);
  }

  // per-stage timing with CUDA events on the launch stream (off by default)
  bool timing = false;
  StageTimes times;

 private:
  int ensure_workspace(int precision, int nd, int nchunks);
  int refold32(const double* tcen, cudaStream_t st);
  int matvec_tree(int precision, int nd, const double* d_sigma, double* d_pot, cudaStream_t st);
  int tune_far(int precision, int nd, dev::MatvecArgs& a, cudaStream_t st, FarConfig& out);
  cudaError_t launch_far_stage(const dev::MatvecArgs& a, cudaStream_t st);
  DBuf<double> ab64_;
  DBuf<float> ab32_;
  std::map<std::pair<int, int>, FarConfig> far_cfg_;
  DBuf<double> tx_, ty_, tz_, sx_, sy_, sz_, snx_, sny_, snz_, sw_, imat_, wts_, tbox_, sbox_;
  DBuf<int32_t> pstart_, ostart_, pclass_, col_, nps_;
  DBuf<int64_t> cmoff_, row_ptr_, wofs_;
  DBuf<double> weff64_;
  DBuf<float> weff32_;
  DBuf<int> tc_err_;  // timeout flag of the tensor-core far field
  std::unique_ptr<TreeFar> tree_[2];
  int far_method_[2] = {0, 0};
  DBuf<char> str_;
  DBuf<double> partial_;
  cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
  // the streams of the near quadrature's chunk copies (wst_) and of the
  // folds (fst_), and the events that order them; a build without
  // async_weff releases them once W_eff is complete
  void release_weff_streams();
  cudaStream_t wst_ = nullptr, fst_ = nullptr;
  cudaEvent_t wev_in_ = nullptr, wev_done_ = nullptr;
  std::vector<cudaEvent_t> wev_copy_;  // one per chunk copy
};

// A batch of surfaces solved together: one operator whose nodes are the
// surfaces' nodes back to back (segment = surface).  Each surface keeps its
// own plan (geometry, near quadrature folded into W_eff); the batch adds a
// device table of surface descriptors and work lists, so each matvec stage
// is one persistent launch over all surfaces, and captures the three
// launches once per (precision, nd) in a CUDA graph that is replayed for
// every matvec (the kernels read the vector pointers from device memory).
class BatchPlan : public Operator {
 public:
  int kind = -1;
  bool ck = false;               // some surface has a complex wavenumber
  bool use_graph = true;
  std::vector<std::unique_ptr<Plan>> plans;
  ~BatchPlan() override;
  int add(Plan* p);  // an on-surface plan; on success the batch owns it
  int finalize(cudaStream_t st);         // node table, weights, reduction segments
  int apply(int precision, int nd, const double* x, double* y, cudaStream_t st) override;
  bool square() const override;
  int set_active(const std::vector<uint8_t>& active, cudaStream_t st) override;
  // far shape kept by the autotuner for (precision, nd): variant, chunk length
  bool far_choice(int precision, int nd, int* variant, int64_t* chunk) const;

 private:
  struct Config {
    int variant = 0;
    int64_t chunk = 0;
    DBuf<dev::BatchSurf> surfs;
    DBuf<int2> patch_items, row_items;
    DBuf<int4> far_items;
    DBuf<char> str;
    DBuf<double> partial;
    DBuf<void*> refs;  // [0] input vector, [1] output vector (device pointer slots)
    DBuf<int> counter;  // far-field work counter
    dev::BatchArgs args;
    cudaGraphExec_t graph = nullptr;
  };
  int build_config(int precision, int nd, int variant, int64_t chunk, Config& c, cudaStream_t st);
  int tune(int precision, int nd, cudaStream_t st, std::unique_ptr<Config>& out);
  std::map<std::pair<int, int>, std::unique_ptr<Config>> cfg_;
  DBuf<double> wts_;
  DBuf<int> live_;                 // per surface, read by the batched kernels
  std::vector<uint8_t> live_host_;
  int64_t nptso_total_ = 0;
  int max_np_ = 0;
};

struct GmresOut {
  std::vector<int64_t> niter;   // per system
  std::vector<double> errs;     // (numit+1) per system, system-major
  std::vector<double> rres;     // per system
  int status = kOk;
};

// Unrestarted GMRES on (zid I + K) x = rhs for the operator's nseg * nd
// independent systems (zgmres_guru / dgmres_guru semantics,
// gmres_routs.f90:13-375, with classical Gram-Schmidt applied twice in
// place of modified Gram-Schmidt).  zid has one value per system
// (system = segment * nd + density).  The inner matvec uses `precision`;
// the final relative residual rres uses `rres_precision` (-1 skips it).
// d_x0 (optional) is an initial guess.
// eps_sys (optional): a relative tolerance per system in place of eps_gmres.
// d_res (optional): receives rhs - (zid I + K) soln under the inner
// operator, formed from the Krylov basis and the rotations (no matvec).
int gmres(Operator& P, int precision, int rres_precision, int nd, const cdouble* zid,
          const double* d_rhs, const double* d_x0, int64_t numit, double eps_gmres,
          double* d_soln, GmresOut& out, cudaStream_t st, const double* eps_sys = nullptr,
          double* d_res = nullptr);

// Mixed-precision solve: FP64 residuals and iterative refinement around
// FP32-matvec GMRES inner solves.  Stops when the FP64 relative residual
// is <= eps_target (per system) or max_outer refinements were done.
//
// The refinement residual r = b - (zid x + K x) needs K x to about 1e-11 of
// ||b||.  With increments on (the default), K x is kept in FP64: the first
// refinement step applies the FP64 operator to the whole x, and a later
// step whose correction d is small, kFp32OpErr ||d||_w / ||x||_w <=
// eps_target / 4 for every active system, adds the FP32 operator's K d to
// it instead (FP32 error on a correction of relative size ||d||/||x||); any
// other step applies the FP64 operator to x again.  The FP32 K d needs no
// matvec: the inner GMRES returns its own residual vector rn = r - A32 d
// (from the Arnoldi relation A32 V_m = V_{m+1} H), so K d = r - rn - zid d.
struct MixedOut {
  std::vector<int64_t> inner_iters;  // total inner GMRES iterations per system
  std::vector<double> rres;          // final FP64 relative residual per system
  std::vector<int64_t> outer;        // refinement steps per system
  std::vector<int64_t> x0_dropped;   // 1 where the initial guess was replaced by 0
  int fp64_matvecs = 0, fp32_matvecs = 0;
  int incr_matvecs = 0;              // refinement steps whose K d came from the inner
                                     // solve's Krylov basis (no matvec)
  double max_incr_ratio = 0.0;       // largest ||d||_w / ||x||_w of an increment step
  int status = kOk;
};
// Relative error assumed for the FP32 operator in the increment test (the
// measured FP32 matvec errors are 2.6e-7 to 9.3e-7 of the FP64 result).
constexpr double kFp32OpErr = 1e-6;
// Refinement residual: 1 = increments (default), 0 = the FP64 operator on x
// at every step.  BIE_MIXED_RESIDUAL=full|increment sets the initial value.
int mixed_residual_mode();
void set_mixed_residual_mode(int mode);
// statistics of the calling thread's last mixed solve: fp64 and fp32
// matvecs, increment steps, largest increment ratio
const MixedOut& last_mixed_out();
int solve_mixed(Operator& P, int nd, const cdouble* zid, const double* d_rhs, const double* d_x0,
                int64_t numit, double eps_target, double inner_floor, int max_outer,
                double* d_soln, MixedOut& out, cudaStream_t st);

}  // namespace bie
