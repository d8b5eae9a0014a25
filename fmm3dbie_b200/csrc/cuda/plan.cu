// Operator plan, batched GMRES and the mixed-precision refinement solver.
#include "plan.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <tuple>

#include "../host/basis.h"
#include "../host/setup.h"
#include "tree_far.h"

namespace bie {

namespace {
thread_local std::string g_last_error;

#define BIE_CUDA(call)                                                             \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_));          \
      return e_ == cudaErrorMemoryAllocation ? kErrNoMem : kErrCuda;               \
    }                                                                              \
  } while (0)

template <class T>
cudaError_t upload(DBuf<T>& b, const std::vector<T>& h, cudaStream_t st) {
  cudaError_t e = b.alloc(std::max<size_t>(h.size(), 1));
  if (e != cudaSuccess) return e;
  if (h.empty()) return cudaSuccess;
  return cudaMemcpyAsync(b.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}
template <class T>
cudaError_t upload(DBuf<T>& b, const T* h, size_t n, cudaStream_t st) {
  cudaError_t e = b.alloc(std::max<size_t>(n, 1));
  if (e != cudaSuccess || n == 0) return e;
  return cudaMemcpyAsync(b.p, h, n * sizeof(T), cudaMemcpyHostToDevice, st);
}

// near-pair chunks of the near quadrature's upload in an async_weff build,
// and how many of them are issued before the host builds the other arrays
// (about the 2 ms that building takes at the PCIe bandwidth, for the
// 287 MB of a 35,840-node Helmholtz surface)
constexpr int kWeffChunks = 8, kWeffEarlyChunks = 3;

// Interpolation matrices by (patch type, order, oversampled order): functions
// of the key alone, computed once per process and shared by every plan.
int cached_interp_matrix(int ip, int no, int nf, const std::vector<double>*& m) {
  static std::mutex mu;
  static auto* cache = new std::map<std::tuple<int, int, int>, std::vector<double>>;
  std::lock_guard<std::mutex> lk(mu);
  const auto key = std::make_tuple(ip, no, nf);
  auto it = cache->find(key);
  if (it == cache->end()) {
    std::vector<double> v;
    if (const int ier = interp_matrix(ip, no, nf, v)) return ier;
    it = cache->emplace(key, std::move(v)).first;
  }
  m = &it->second;
  return 0;
}

// Pinned staging for the arrays a plan build assembles on the host, shared by
// the builds of the process one at a time.  It is allocated (its pages
// faulted in) once and grown when a larger plan comes, so the uploads out of
// it are asynchronous and a build pays no page faults.  A build that finds it
// in use by another thread, or needs more than kMaxPinned bytes, stages in
// pageable memory instead.  The destructor waits for the copies out of it.
class HostStaging {
 public:
  static constexpr size_t kMaxPinned = size_t(256) << 20;
  template <class T>
  static size_t bytes(size_t n) {
    return (n * sizeof(T) + 63) / 64 * 64;
  }
  explicit HostStaging(size_t n) : cap_(n) {
    Pool& pl = pool();
    if (n <= kMaxPinned && pl.mu.try_lock()) {
      locked_ = true;
      if (pl.cap < n) {
        if (pl.p) cudaFreeHost(pl.p);
        pl.p = nullptr;
        pl.cap = 0;
        const size_t want = std::min(kMaxPinned, std::max(n + n / 4, size_t(8) << 20));
        void* q = nullptr;
        if (cudaHostAlloc(&q, want, cudaHostAllocPortable) == cudaSuccess) {
          pl.p = static_cast<char*>(q);
          pl.cap = want;
        } else {
          cudaGetLastError();  // pageable staging below
        }
      }
      base_ = pl.p;
    }
    if (!base_) {
      heap_.reset(new char[n + 64]);
      base_ = heap_.get() + (64 - reinterpret_cast<uintptr_t>(heap_.get()) % 64) % 64;
    }
  }
  ~HostStaging() {
    if (st_set_) cudaStreamSynchronize(st_);
    if (locked_) pool().mu.unlock();
  }
  HostStaging(const HostStaging&) = delete;
  HostStaging& operator=(const HostStaging&) = delete;
  // the stream that the uploads out of the buffer are issued on
  void copies_on(cudaStream_t st) {
    st_ = st;
    st_set_ = true;
  }
  template <class T>
  T* take(size_t n) {
    const size_t b = bytes<T>(n);
    if (off_ + b > cap_) throw std::logic_error("plan staging buffer too small");
    T* r = reinterpret_cast<T*>(base_ + off_);
    off_ += b;
    return r;
  }

 private:
  struct Pool {
    std::mutex mu;
    char* p = nullptr;
    size_t cap = 0;
  };
  static Pool& pool() {
    static Pool* p = new Pool;  // never destroyed: builds may run during exit
    return *p;
  }
  char* base_ = nullptr;
  size_t cap_ = 0, off_ = 0;
  bool locked_ = false, st_set_ = false;
  cudaStream_t st_ = nullptr;
  std::unique_ptr<char[]> heap_;
};
}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

cudaStream_t& alloc_stream() {
  thread_local cudaStream_t s = nullptr;
  return s;
}

AllocStreamScope::AllocStreamScope(cudaStream_t s) : prev(alloc_stream()) {
  // keep the default pool's memory between calls (no release at syncs)
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64) {
    std::lock_guard<std::mutex> lk(mu);
    if (!done[dev]) {
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      }
      done[dev] = true;
    }
  }
  alloc_stream() = s;
}

Plan::Plan() = default;

Plan::~Plan() {
  for (auto& e : ev_)
    if (e) cudaEventDestroy(e);
  release_weff_streams();
}

void Plan::release_weff_streams() {
  // W_eff copies and folds done before their buffers go
  if (wst_) cudaStreamSynchronize(wst_);
  if (fst_) cudaStreamSynchronize(fst_);
  if (wev_in_) cudaEventDestroy(wev_in_);
  if (wev_done_) cudaEventDestroy(wev_done_);
  for (auto e : wev_copy_)
    if (e) cudaEventDestroy(e);
  if (wst_) cudaStreamDestroy(wst_);
  if (fst_) cudaStreamDestroy(fst_);
  wst_ = fst_ = nullptr;
  wev_in_ = wev_done_ = nullptr;
  wev_copy_.clear();
}

int Plan::wait_weff(cudaStream_t st) {
  if (wev_done_) BIE_CUDA(cudaStreamWaitEvent(st, wev_done_, 0));
  return kOk;
}

int Plan::build(const PlanSpec& s, cudaStream_t st) {
  BIE_CUDA(cudaGetDevice(&device));
  BIE_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
  kind = s.kind;
  cplx = s.kind == 1;
  npts = s.npts;
  ntarg = s.ntarg;
  nptso = s.nptso;
  npatches = s.npatches;
  nnz = s.nnz;
  nquad = s.nquad;
  // ---- validate the reference-style inputs --------------------------------
  if (npatches <= 0 || npts <= 0 || ntarg < 0 || nptso <= 0 || nnz < 0) {
    set_last_error("non-positive sizes");
    return kErrArg;
  }
  if (s.ixyzs[0] != 1 || s.ixyzs[npatches] != npts + 1 || s.ixyzso[0] != 1 ||
      s.ixyzso[npatches] != nptso + 1) {
    set_last_error("ixyzs/ixyzso inconsistent with npts/nptso");
    return kErrArg;
  }
  int max_np = 0, max_nf = 0;
  for (int64_t p = 0; p < npatches; ++p) {
    const int ip = int(s.iptype[p]), no = int(s.norders[p]), nf = int(s.novers[p]);
    const int64_t np = s.ixyzs[p + 1] - s.ixyzs[p];
    const int64_t nfp = s.ixyzso[p + 1] - s.ixyzso[p];
    if (!valid_patch(ip, no) || !valid_patch(ip, nf) || np != npols_of(ip, no) ||
        nfp != npols_of(ip, nf)) {
      set_last_error("patch " + std::to_string(p + 1) + ": order/type/size mismatch");
      return kErrArg;
    }
    max_np = std::max<int>(max_np, int(np));
    max_nf = std::max<int>(max_nf, int(nfp));
  }
  if (s.row_ptr[0] != 1 || s.row_ptr[ntarg] != nnz + 1) {
    set_last_error("row_ptr inconsistent with nnz");
    return kErrArg;
  }
  for (int64_t i = 0; i < ntarg; ++i)
    if (s.row_ptr[i + 1] < s.row_ptr[i]) {
      set_last_error("row_ptr not monotone");
      return kErrArg;
    }
  if (nnz > 0 && s.iquad[0] != 1) {
    set_last_error("iquad(1) must be 1");
    return kErrArg;
  }
  if (nquad < 0 || (nnz > 0 && s.iquad[nnz] - 1 != nquad)) {
    set_last_error("nquad != iquad(nnz+1)-1");
    return kErrArg;
  }
  // The near quadrature (the largest input: nquad entries) goes to the device
  // in near-pair chunks.  The first chunks' copies run while the host checks
  // the near list and builds the other arrays; the uploads of those follow,
  // and the other chunks wait for them, so that the geometry lands early
  // (measured: a copy issued on st while chunk copies are queued on their
  // stream lands after all of them).  Each chunk's folds start on their own
  // stream as soon as the chunk has landed.  With async_weff the build
  // returns before they finish and the solve's first far field runs beside
  // them; otherwise the build waits for them.
  const int cw = cplx ? 2 : 1;
  const size_t wlen = size_t(nquad) * cw;
  BIE_CUDA(weff64_.alloc(std::max<size_t>(wlen, 1)));
  const int nwc = nnz >= int64_t(kWeffChunks) * 1024 ? kWeffChunks : 1;
  std::vector<int64_t> kc(nwc + 1, 0), qc(nwc + 1, 0);
  for (int c = 1; c <= nwc; ++c) {
    kc[c] = nnz * c / nwc;
    // clamped into order: an iquad that is not monotone is rejected below,
    // before any fold reads W_eff
    qc[c] = c == nwc ? nquad : std::min(nquad, std::max(qc[c - 1], s.iquad[kc[c]] - 1));
  }
  cudaStream_t wst = st, fst = st;  // streams of the W_eff chunk copies and of the folds
  if (s.async_weff || nwc > 1) {
    BIE_CUDA(cudaStreamCreateWithFlags(&wst_, cudaStreamNonBlocking));
    BIE_CUDA(cudaStreamCreateWithFlags(&fst_, cudaStreamNonBlocking));
    BIE_CUDA(cudaEventCreateWithFlags(&wev_in_, cudaEventDisableTiming));
    BIE_CUDA(cudaEventCreateWithFlags(&wev_done_, cudaEventDisableTiming));
    wev_copy_.assign(size_t(nwc), nullptr);
    for (auto& e : wev_copy_) BIE_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    BIE_CUDA(cudaEventRecord(wev_in_, st));  // the allocation, ordered on st
    BIE_CUDA(cudaStreamWaitEvent(wst_, wev_in_, 0));
    wst = wst_;
    fst = fst_;
  }
  // an input rejected below returns while chunk copies may still read the
  // caller's near quadrature: they finish first
  struct CopyGuard {
    cudaStream_t s;
    bool done = false;
    ~CopyGuard() {
      if (!done) cudaStreamSynchronize(s);
    }
  } copy_guard{wst};
  auto copy_chunk = [&](int c) -> int {
    if (qc[c + 1] > qc[c])
      BIE_CUDA(cudaMemcpyAsync(weff64_.p + qc[c] * cw, s.wnear + qc[c] * cw,
                               size_t(qc[c + 1] - qc[c]) * cw * sizeof(double),
                               cudaMemcpyHostToDevice, wst));
    if (!wev_copy_.empty()) BIE_CUDA(cudaEventRecord(wev_copy_[size_t(c)], wst));
    return kOk;
  };
  const int early = nwc > 1 ? std::min(nwc - 1, kWeffEarlyChunks) : 1;
  for (int c = 0; c < early; ++c)
    if (int e = copy_chunk(c)) return e;
  // ---- interpolation classes -------------------------------------------------
  std::vector<int32_t> cls_of(npatches);
  std::vector<const std::vector<double>*> cls_mat;
  {
    std::map<std::tuple<int, int, int>, int> cls;
    for (int64_t p = 0; p < npatches; ++p) {
      auto key = std::make_tuple(int(s.iptype[p]), int(s.norders[p]), int(s.novers[p]));
      auto it = cls.find(key);
      if (it == cls.end()) {
        const std::vector<double>* m = nullptr;
        const int ier = cached_interp_matrix(std::get<0>(key), std::get<1>(key), std::get<2>(key), m);
        if (ier) {
          set_last_error("interpolation matrix: basis tables unavailable or singular");
          return ier == 6 ? kErrTables : kErrSingular;
        }
        it = cls.emplace(key, int(cls_mat.size())).first;
        cls_mat.push_back(m);
      }
      cls_of[p] = it->second;
    }
  }
  size_t nim = 0;
  for (const auto* m : cls_mat) nim += m->size();
  // ---- host-side arrays, in the pinned staging buffer --------------------------
  const int64_t nbt = (ntarg + dev::kFarBlockTargets32 - 1) / dev::kFarBlockTargets32;
  const int64_t nbs = (nptso + dev::kFarTileSources - 1) / dev::kFarTileSources;
  const size_t nbt6 = size_t(6) * std::max<int64_t>(nbt, 1), nbs6 = size_t(6) * std::max<int64_t>(nbs, 1);
  using HS = HostStaging;
  const size_t stage_bytes =
      3 * HS::bytes<double>(ntarg) + 7 * HS::bytes<double>(nptso) +
      2 * HS::bytes<int32_t>(npatches + 1) + HS::bytes<int32_t>(npatches) +
      HS::bytes<int64_t>(cls_mat.size()) + HS::bytes<double>(nim) + HS::bytes<int64_t>(ntarg + 1) +
      HS::bytes<int64_t>(nnz + 1) + 2 * HS::bytes<int32_t>(nnz) + HS::bytes<double>(npts) +
      HS::bytes<double>(nbt6) + HS::bytes<double>(nbs6);
  HostStaging stage(stage_bytes);
  double* htx = stage.take<double>(ntarg);
  double* hty = stage.take<double>(ntarg);
  double* htz = stage.take<double>(ntarg);
  double* hsrc[7];
  for (auto& h : hsrc) h = stage.take<double>(nptso);
  int32_t* hps = stage.take<int32_t>(npatches + 1);
  int32_t* hos = stage.take<int32_t>(npatches + 1);
  int32_t* hpc = stage.take<int32_t>(npatches);
  int64_t* hcm = stage.take<int64_t>(cls_mat.size());
  double* him = stage.take<double>(nim);
  int64_t* hrp = stage.take<int64_t>(ntarg + 1);
  int64_t* hwo = stage.take<int64_t>(nnz + 1);
  int32_t* hcol = stage.take<int32_t>(nnz);
  int32_t* hnps = stage.take<int32_t>(nnz);
  double* hqw = stage.take<double>(npts);
  double* htb = stage.take<double>(nbt6);
  double* hsb = stage.take<double>(nbs6);
  // the near list, checked and converted in one pass
  int64_t bad = nnz;
#pragma omp parallel for schedule(static) reduction(min : bad) if (nnz >= 65536)
  for (int64_t k = 0; k < nnz; ++k) {
    const int64_t c = s.col_ind[k];
    if (c < 1 || c > npatches || s.iquad[k + 1] - s.iquad[k] != s.ixyzs[c] - s.ixyzs[c - 1]) {
      bad = std::min(bad, k);
      continue;
    }
    hcol[k] = int32_t(c - 1);
    hnps[k] = int32_t(s.ixyzs[c - 1] - 1);
    hwo[k] = s.iquad[k] - 1;
  }
  if (bad < nnz) {
    set_last_error("col_ind/iquad entry " + std::to_string(bad + 1) + " invalid");
    return kErrArg;
  }
  hwo[nnz] = nquad;
  for (int64_t i = 0; i <= ntarg; ++i) hrp[i] = s.row_ptr[i] - 1;
#pragma omp parallel for schedule(static) if (ntarg >= 65536)
  for (int64_t i = 0; i < ntarg; ++i) {
    htx[i] = s.targs[size_t(s.ndtarg) * i];
    hty[i] = s.targs[size_t(s.ndtarg) * i + 1];
    htz[i] = s.targs[size_t(s.ndtarg) * i + 2];
  }
#pragma omp parallel for schedule(static) if (nptso >= 65536)
  for (int64_t j = 0; j < nptso; ++j) {
    const double* o = s.srcover + 12 * j;
    hsrc[0][j] = o[0];
    hsrc[1][j] = o[1];
    hsrc[2][j] = o[2];
    hsrc[3][j] = o[9];
    hsrc[4][j] = o[10];
    hsrc[5][j] = o[11];
    hsrc[6][j] = s.whtsover[j];
  }
  for (int64_t p = 0; p <= npatches; ++p) {
    hps[p] = int32_t(s.ixyzs[p] - 1);
    hos[p] = int32_t(s.ixyzso[p] - 1);
  }
  for (int64_t p = 0; p < npatches; ++p) hpc[p] = cls_of[p];
  {
    size_t o = 0;
    for (size_t c = 0; c < cls_mat.size(); ++c) {
      hcm[c] = int64_t(o);
      std::copy(cls_mat[c]->begin(), cls_mat[c]->end(), him + o);
      o += cls_mat[c]->size();
    }
  }
  // smooth quadrature weights at the nodes (needed by the GMRES inner product)
  {
    Surf sf;
    sf.npatches = npatches;
    sf.npts = npts;
    sf.norders = s.norders;
    sf.ixyzs = s.ixyzs;
    sf.iptype = s.iptype;
    sf.srccoefs = s.srccoefs;
    sf.srcvals = s.srcvals;
    qwts(sf, hqw);
  }
  kp.kind = kind;
  kp.ar = s.alpha.real();
  kp.ai = s.alpha.imag();
  kp.br = s.beta.real();
  kp.bi = s.beta.imag();
  kp.kr = s.zk.real();
  kp.ki = s.zk.imag();
  if (kind == 0) kp.ai = kp.bi = kp.kr = kp.ki = 0.0;
  // bounding boxes of the FP32 far kernel's target blocks and source tiles;
  // margin: the threshold plus 2^-12 of the extent, far above the FP32
  // rounding of the centred coordinates
  auto boxes = [](const double* x, const double* y, const double* z, int64_t n, int64_t per,
                  double* out) {
    const int64_t nb = (n + per - 1) / per;
    if (nb == 0) std::fill(out, out + 6, 0.0);
#pragma omp parallel for schedule(static) if (nb >= 256)
    for (int64_t b = 0; b < nb; ++b) {
      double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
      for (int64_t j = b * per; j < std::min(n, (b + 1) * per); ++j) {
        const double v[3] = {x[j], y[j], z[j]};
        for (int c = 0; c < 3; ++c) {
          lo[c] = std::min(lo[c], v[c]);
          hi[c] = std::max(hi[c], v[c]);
        }
      }
      for (int c = 0; c < 3; ++c) {
        out[6 * b + c] = lo[c];
        out[6 * b + 3 + c] = hi[c];
      }
    }
  };
  boxes(htx, hty, htz, ntarg, dev::kFarBlockTargets32, htb);
  boxes(hsrc[0], hsrc[1], hsrc[2], nptso, dev::kFarTileSources, hsb);
  // get_fmm_thresh (get_fmm_thresh.f:81) from the union of the boxes: the
  // same bounding box of all sources and targets, the extrema being exact
  {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    auto add = [&](const double* bx, int64_t nb) {
      for (int64_t b = 0; b < nb; ++b)
        for (int c = 0; c < 3; ++c) {
          lo[c] = std::min(lo[c], bx[6 * b + c]);
          hi[c] = std::max(hi[c], bx[6 * b + 3 + c]);
        }
    };
    add(htb, nbt);
    add(hsb, nbs);
    kp.thresh = std::ldexp(std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]}), -51);
  }
  double ext = 0.0;
  for (int64_t b = 0; b < nbt; ++b)
    for (int c = 0; c < 3; ++c) ext = std::max(ext, std::fabs(htb[6 * b + c]) + std::fabs(htb[6 * b + 3 + c]));
  for (int64_t b = 0; b < nbs; ++b)
    for (int c = 0; c < 3; ++c) ext = std::max(ext, std::fabs(hsb[6 * b + c]) + std::fabs(hsb[6 * b + 3 + c]));
  const double margin = kp.thresh + std::ldexp(ext, -12);
  // ---- upload ----------------------------------------------------------------
  stage.copies_on(st);
  BIE_CUDA(upload(tx_, htx, ntarg, st));
  BIE_CUDA(upload(ty_, hty, ntarg, st));
  BIE_CUDA(upload(tz_, htz, ntarg, st));
  BIE_CUDA(upload(sx_, hsrc[0], nptso, st));
  BIE_CUDA(upload(sy_, hsrc[1], nptso, st));
  BIE_CUDA(upload(sz_, hsrc[2], nptso, st));
  BIE_CUDA(upload(snx_, hsrc[3], nptso, st));
  BIE_CUDA(upload(sny_, hsrc[4], nptso, st));
  BIE_CUDA(upload(snz_, hsrc[5], nptso, st));
  BIE_CUDA(upload(sw_, hsrc[6], nptso, st));
  BIE_CUDA(upload(pstart_, hps, npatches + 1, st));
  BIE_CUDA(upload(ostart_, hos, npatches + 1, st));
  BIE_CUDA(upload(pclass_, hpc, npatches, st));
  BIE_CUDA(upload(cmoff_, hcm, cls_mat.size(), st));
  BIE_CUDA(upload(imat_, him, nim, st));
  BIE_CUDA(upload(row_ptr_, hrp, ntarg + 1, st));
  BIE_CUDA(upload(col_, hcol, nnz, st));
  BIE_CUDA(upload(nps_, hnps, nnz, st));
  BIE_CUDA(upload(wofs_, hwo, nnz + 1, st));
  BIE_CUDA(upload(wts_, hqw, npts, st));
  BIE_CUDA(upload(tbox_, htb, nbt6, st));
  BIE_CUDA(upload(sbox_, hsb, nbs6, st));
  if (early < nwc) {
    BIE_CUDA(cudaEventRecord(wev_in_, st));  // the uploads above
    BIE_CUDA(cudaStreamWaitEvent(wst_, wev_in_, 0));
  }
  for (int c = early; c < nwc; ++c)
    if (int e = copy_chunk(c)) return e;
  g.ntarg = ntarg;
  g.nptso = nptso;
  g.npatches = npatches;
  g.npts = npts;
  g.tx = tx_.p;
  g.ty = ty_.p;
  g.tz = tz_.p;
  g.sx = sx_.p;
  g.sy = sy_.p;
  g.sz = sz_.p;
  g.snx = snx_.p;
  g.sny = sny_.p;
  g.snz = snz_.p;
  g.sw = sw_.p;
  g.pstart = pstart_.p;
  g.ostart = ostart_.p;
  g.pclass = pclass_.p;
  g.cmoff = cmoff_.p;
  g.imat = imat_.p;
  g.max_np = max_np;
  g.max_nf = max_nf;
  g.tbox = ntarg > 0 ? tbox_.p : nullptr;
  g.sbox = sbox_.p;
  g.box_margin2 = margin * margin;
  nr.nnz = nnz;
  nr.nquad = nquad;
  nr.row_ptr = row_ptr_.p;
  nr.col = col_.p;
  nr.nps = nps_.p;
  nr.wofs = wofs_.p;
  // ---- fold the smooth near part into W_eff (in place over wnear) -----------
  if (s.keep_f32) BIE_CUDA(weff32_.alloc(std::max<size_t>(wlen, 1)));
  if (fst_) {
    // the folds read the geometry uploaded on st and the buffers allocated there
    BIE_CUDA(cudaEventRecord(wev_in_, st));
    BIE_CUDA(cudaStreamWaitEvent(fst_, wev_in_, 0));
  }
  for (int c = 0; c < nwc; ++c) {
    if (fst_) BIE_CUDA(cudaStreamWaitEvent(fst_, wev_copy_[size_t(c)], 0));
    // FP32 path: subtract the smooth part as the FP32 far kernel computes it
    if (s.keep_f32)
      BIE_CUDA(dev::launch_fold(g, nr, kp, weff64_.p, weff32_.p, 1, fst, kc[c], kc[c + 1]));
    BIE_CUDA(dev::launch_fold(g, nr, kp, weff64_.p, weff64_.p, 0, fst, kc[c], kc[c + 1]));
  }
  if (fst_) BIE_CUDA(cudaEventRecord(wev_done_, fst_));
  // per-source constants alpha w/(4pi), beta w/(4pi) for the multi-density far kernel
  BIE_CUDA(ab64_.alloc(size_t(nptso) * (cplx ? 4 : 2)));
  BIE_CUDA(ab32_.alloc(size_t(nptso) * (cplx ? 4 : 2)));
  BIE_CUDA(dev::launch_source_consts(g, kp, 0, ab64_.p, st));
  BIE_CUDA(dev::launch_source_consts(g, kp, 1, ab32_.p, st));
  BIE_CUDA(tc_err_.alloc(1));
  BIE_CUDA(cudaMemsetAsync(tc_err_.p, 0, sizeof(int), st));
  for (auto& e : ev_) BIE_CUDA(cudaEventCreate(&e));
  // without async_weff the build returns with W_eff complete
  if (!s.async_weff && wev_done_) BIE_CUDA(cudaStreamWaitEvent(st, wev_done_, 0));
  // the staged host arrays are consumed by async copies: wait before they go
  BIE_CUDA(cudaStreamSynchronize(st));
  copy_guard.done = true;  // from here the destructor waits for any copy still in flight
  if (!s.async_weff) release_weff_streams();
  // far-field method by problem size
  {
    const char* fm = std::getenv("BIE_FAR_METHOD");
    const std::string m = fm ? fm : "auto";
    const char* tp = std::getenv("BIE_TREE_PAIRS");
    const double pairs_min = tp && *tp ? std::atof(tp) : kTreeAutoPairs;
    const bool tree = m == "tree" || (m == "auto" && double(ntarg) * double(nptso) >= pairs_min);
    if (tree && ntarg > 0)
      for (int prec = 0; prec < 2; ++prec) {
        if (prec == 1 && !s.keep_f32) continue;
        const int ier = set_far_method(prec, 1, nullptr, st);
        // inputs the trees cannot take (more than 128 coincident targets)
        // keep the direct sum; device errors stop the build
        if (ier == kErrArg) continue;
        if (ier) return ier;
      }
  }
  // as a solver operator: one segment of npts nodes
  nodes = npts;
  d_node_wts = wts_.p;
  seg_start = {0, npts};
  return init_segments(st);
}

int Plan::nchunks_for(int precision, int nd) const {
  return far_method_[precision & 1] == 1 ? 1 : far_config(precision, nd).nchunks;
}

tree::Params Plan::default_tree_params(int precision, const dev::KParams& kp) {
  tree::Params prm;
  prm.theta = 0.5;
  // theta 0.5: p = 10 keeps the FP64 matvec within about 1e-10 of the
  // direct sum on the test surfaces (p = 8: 1e-7 .. 1e-6); for the FP32
  // matvec p = 8 stays below the FP32 rounding of the proxy terms.
  // Helmholtz grids grow with k times the side.
  prm.p = precision == 1 ? 8 : 10;
  prm.k = kp.kind == 1 ? std::fabs(kp.kr) : 0.0;
  prm.kscale = 1.0;
  const char* e = std::getenv("BIE_TREE_P");
  if (e && *e) prm.p = std::max(1, std::min(tree::kMaxP, std::atoi(e)));
  e = std::getenv("BIE_TREE_THETA");
  if (e && *e) prm.theta = std::atof(e);
  return prm;
}

tree::Params Plan::tree_params(int precision) const {
  const auto& t = tree_[precision & 1];
  return t ? t->params() : default_tree_params(precision, kp);
}

const TreeStats* Plan::tree_stats(int precision) const {
  const auto& t = tree_[precision & 1];
  return t ? &t->stats() : nullptr;
}

int Plan::refold32(const double* tcen, cudaStream_t st) {
  if (!weff32_.p) return kOk;
  if (int e = wait_weff(st)) return e;
  dev::Geometry gg = g;
  gg.tcen = tcen;
  BIE_CUDA(dev::launch_fold(gg, nr, kp, weff64_.p, weff32_.p, 2, st));
  return kOk;
}

int Plan::set_far_method(int precision, int method, const tree::Params* prm, cudaStream_t st) {
  if ((precision != 0 && precision != 1) || (method != 0 && method != 1)) {
    set_last_error("far method: precision 0/1, method 0 (direct) or 1 (tree)");
    return kErrArg;
  }
  if (precision == 1 && !weff32_.p) {
    set_last_error("plan built without an f32 copy of W_eff");
    return kErrArg;
  }
  if (method == 1) {
    tree::Params p = prm ? *prm : default_tree_params(precision, kp);
    if (!(p.theta > 0.0 && p.theta < 1.0) || p.p < 1 || p.p > tree::kMaxP || p.leaf_t < 1 ||
        p.leaf_t > 128 || p.leaf_s < 1) {
      set_last_error("tree parameters out of range (0 < theta < 1, 1 <= p <= 16, leaf_t <= 128)");
      return kErrArg;
    }
    if (ntarg <= 0) {
      set_last_error("tree far field needs targets");
      return kErrArg;
    }
    auto t = std::make_unique<TreeFar>();
    const int ier = t->build(g, p, kp.thresh, st, &kp, precision);
    if (ier) return ier;
    tree_[precision] = std::move(t);
    if (precision == 1) {
      const int e2 = refold32(tree_[1]->tcentre(), st);
      if (e2) return e2;
    }
  } else {
    if (precision == 1 && far_method_[1] == 1) {
      const int e2 = refold32(nullptr, st);
      if (e2) return e2;
    }
    tree_[precision].reset();
  }
  far_method_[precision] = method;
  BIE_CUDA(cudaStreamSynchronize(st));
  return kOk;
}

namespace {
// Process-wide cache of tuned far-kernel shapes, keyed by everything the
// timing depends on.
using FarKey = std::tuple<int, int, int, int, int, int64_t, int64_t>;
std::mutex g_far_mu;
std::map<FarKey, Plan::FarConfig> g_far_cache;

int env_int(const char* name, int dflt) {
  const char* v = std::getenv(name);
  return v && *v ? std::atoi(v) : dflt;
}
double env_double(const char* name, double dflt) {
  const char* v = std::getenv(name);
  return v && *v ? std::atof(v) : dflt;
}
}  // namespace

int Plan::set_far_config(int precision, int nd, int variant, int nchunks) {
  if ((precision != 0 && precision != 1) || nd < 1 || variant < 0 ||
      variant >= dev::far_variants() || nchunks < 1 ||
      nchunks > std::max<int64_t>(1, (nptso + dev::kFarTileSources - 1) / dev::kFarTileSources)) {
    set_last_error("far configuration out of range");
    return kErrArg;
  }
  FarConfig c;
  c.variant = variant;
  c.nchunks = nchunks;
  far_cfg_[{precision, nd}] = c;
  return ensure_workspace(precision, nd, nchunks);
}

int Plan::tc_error() const {
  int v = 0;
  if (tc_err_.p) cudaMemcpy(&v, tc_err_.p, sizeof(int), cudaMemcpyDeviceToHost);
  return v;
}

Plan::FarConfig Plan::far_config(int precision, int nd) const {
  auto it = far_cfg_.find({precision, nd});
  if (it != far_cfg_.end()) return it->second;
  // default shape before tuning: variant 0, four waves of resident blocks
  FarConfig c;
  const int md = nd > 1;
  c.variant = std::min(std::max(env_int("BIE_FAR_VARIANT", 0), 0), dev::far_variants() - 1);
  const int bps = dev::far_blocks_per_sm(kp, precision, c.variant, md, nd);
  c.nchunks = dev::far_chunks_for_waves(ntarg, nptso, precision, c.variant, nd, num_sms, bps,
                                        env_double("BIE_FAR_WAVES", md ? 2.0 : 4.0), md);
  return c;
}

cudaError_t Plan::launch_far_stage(const dev::MatvecArgs& a, cudaStream_t st) {
  return a.nd > 1 ? dev::launch_far_md(g, kp, a, st) : dev::launch_far(g, kp, a, st);
}

int Plan::ensure_workspace(int precision, int nd, int nchunks) {
  (void)precision;
  const size_t sreals = size_t(nptso) * nd * (cplx ? 4 : 2);
  BIE_CUDA(str_.alloc(sreals * sizeof(double)));
  BIE_CUDA(partial_.alloc(std::max<size_t>(1, size_t(nchunks) * ntarg * nd * (cplx ? 2 : 1))));
  return kOk;
}

int Plan::tune_far(int precision, int nd, dev::MatvecArgs& a, cudaStream_t st, FarConfig& best) {
  const FarKey key{device, kind, kp.ki != 0.0 ? 1 : 0, precision, nd, ntarg, nptso};
  {
    std::lock_guard<std::mutex> lk(g_far_mu);
    auto it = g_far_cache.find(key);
    if (it != g_far_cache.end()) {
      best = it->second;
      return kOk;
    }
  }
  best = far_config(precision, nd);
  const bool fixed = std::getenv("BIE_FAR_VARIANT") || std::getenv("BIE_FAR_WAVES") ||
                     env_int("BIE_AUTOTUNE", 1) == 0;
  if (!fixed && ntarg > 0) {
    std::vector<FarConfig> cand;
    const int md = nd > 1;
    for (int v = 0; v < dev::far_variants(); ++v) {
      const int bps = dev::far_blocks_per_sm(kp, precision, v, md, nd);
      if (bps <= 0) continue;
      for (double waves : {1.0, 2.0, 4.0, 8.0}) {
        FarConfig c;
        c.variant = v;
        c.nchunks =
            dev::far_chunks_for_waves(ntarg, nptso, precision, v, nd, num_sms, bps, waves, md);
        // the partial sums grow with nchunks * nd: keep them under ~1 GiB
        if (double(c.nchunks) * ntarg * nd * 16.0 > double(1 << 30) && waves > 1.0) continue;
        bool dup = false;
        for (const auto& o : cand) dup |= (o.variant == c.variant && o.nchunks == c.nchunks);
        if (!dup) cand.push_back(c);
      }
    }
    int maxch = 1;
    for (const auto& c : cand) maxch = std::max(maxch, c.nchunks);
    int ier = ensure_workspace(precision, nd, maxch);
    if (ier) return ier;
    a.partial = partial_.p;
    cudaEvent_t e0, e1;
    BIE_CUDA(cudaEventCreate(&e0));
    BIE_CUDA(cudaEventCreate(&e1));
    best.ms = 1e30;
    for (auto& c : cand) {
      a.far_variant = c.variant;
      a.nchunks = c.nchunks;
      BIE_CUDA(launch_far_stage(a, st));  // warm
      BIE_CUDA(cudaEventRecord(e0, st));
      BIE_CUDA(launch_far_stage(a, st));
      BIE_CUDA(cudaEventRecord(e1, st));
      BIE_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      c.ms = ms;
      if (ms < best.ms) best = c;
      if (env_int("BIE_AUTOTUNE_LOG", 0))
        std::fprintf(stderr, "far autotune: prec %d nd %d variant %d chunks %d : %.4f ms\n",
                     precision, nd, c.variant, c.nchunks, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  std::lock_guard<std::mutex> lk(g_far_mu);
  g_far_cache[key] = best;
  return kOk;
}

cudaError_t Plan::oversample(const dev::MatvecArgs& a, cudaStream_t st) {
  if (dev::oversample_engine() == 1 && dev::oversample_tc_fits(g, kp, a.precision, a.nd)) {
    dev::MatvecArgs b = a;
    b.tc_err = tc_err_.p;
    return dev::launch_oversample_tc(g, kp, b, st);
  }
  return dev::launch_oversample(g, kp, a, st);
}

int Plan::matvec(int precision, int nd, const double* d_sigma, double* d_pot, cudaStream_t st) {
  if (nd < 1) return kErrArg;
  if (precision == 1 && !weff32_.p) {
    set_last_error("plan built without an f32 copy of W_eff");
    return kErrArg;
  }
  if (far_method_[precision & 1] == 1) return matvec_tree(precision, nd, d_sigma, d_pot, st);
  FarConfig fc = far_config(precision, nd);
  int ier = ensure_workspace(precision, nd, fc.nchunks);
  if (ier) return ier;
  dev::MatvecArgs a;
  a.precision = precision;
  a.nd = nd;
  a.nchunks = fc.nchunks;
  a.far_variant = fc.variant;
  a.sigma = d_sigma;
  a.pot = d_pot;
  a.strengths = str_.p;
  a.partial = partial_.p;
  a.weff = precision == 1 ? (const void*)weff32_.p : (const void*)weff64_.p;
  a.weff_f32 = precision == 1;
  a.ab = precision == 1 ? (const void*)ab32_.p : (const void*)ab64_.p;
  a.tc_err = tc_err_.p;
  if (timing) BIE_CUDA(cudaEventRecord(ev_[0], st));
  if (nd > 1)
    BIE_CUDA(oversample(a, st));
  else
    BIE_CUDA(dev::launch_strengths(g, kp, a, st));
  if (far_cfg_.find({precision, nd}) == far_cfg_.end()) {
    ier = tune_far(precision, nd, a, st, fc);
    if (ier) return ier;
    far_cfg_[{precision, nd}] = fc;
    ier = ensure_workspace(precision, nd, fc.nchunks);
    if (ier) return ier;
    a.nchunks = fc.nchunks;
    a.far_variant = fc.variant;
    a.partial = partial_.p;
    if (timing) BIE_CUDA(cudaEventRecord(ev_[1], st));
  } else if (timing) {
    BIE_CUDA(cudaEventRecord(ev_[1], st));
  }
  BIE_CUDA(launch_far_stage(a, st));
  if (timing) BIE_CUDA(cudaEventRecord(ev_[2], st));
  if (int e = wait_weff(st)) return e;
  BIE_CUDA(dev::launch_combine(g, nr, kp, a, st));
  if (timing) {
    BIE_CUDA(cudaEventRecord(ev_[3], st));
    BIE_CUDA(cudaEventSynchronize(ev_[3]));
    float t01, t12, t23;
    cudaEventElapsedTime(&t01, ev_[0], ev_[1]);
    cudaEventElapsedTime(&t12, ev_[1], ev_[2]);
    cudaEventElapsedTime(&t23, ev_[2], ev_[3]);
    times.strengths_ms[precision] += t01;
    times.far_ms[precision] += t12;
    times.combine_ms[precision] += t23;
    times.calls[precision] += 1;
  }
  return kOk;
}

int Plan::matvec_tree(int precision, int nd, const double* d_sigma, double* d_pot,
                      cudaStream_t st) {
  TreeFar& T = *tree_[precision];
  int ier = ensure_workspace(precision, nd, 1);
  if (ier) return ier;
  dev::MatvecArgs a;
  a.precision = precision;
  a.nd = nd;
  a.nchunks = 1;
  a.sigma = d_sigma;
  a.pot = d_pot;
  a.strengths = str_.p;
  a.partial = partial_.p;
  a.weff = precision == 1 ? (const void*)weff32_.p : (const void*)weff64_.p;
  a.weff_f32 = precision == 1;
  a.sdest = T.sdest();
  if (timing) BIE_CUDA(cudaEventRecord(ev_[0], st));
  // one density: (charge, dipole) strengths; several: oversampled densities
  if (nd > 1)
    BIE_CUDA(oversample(a, st));
  else
    BIE_CUDA(dev::launch_strengths(g, kp, a, st));
  if (timing) BIE_CUDA(cudaEventRecord(ev_[1], st));
  BIE_CUDA(T.run(precision, nd, kp, nd > 1 ? nullptr : str_.p, partial_.p, st,
                 nd > 1 ? str_.p : nullptr));
  if (timing) BIE_CUDA(cudaEventRecord(ev_[2], st));
  if (int e = wait_weff(st)) return e;
  BIE_CUDA(dev::launch_combine(g, nr, kp, a, st));
  if (timing) {
    BIE_CUDA(cudaEventRecord(ev_[3], st));
    BIE_CUDA(cudaEventSynchronize(ev_[3]));
    float t01, t12, t23;
    cudaEventElapsedTime(&t01, ev_[0], ev_[1]);
    cudaEventElapsedTime(&t12, ev_[1], ev_[2]);
    cudaEventElapsedTime(&t23, ev_[2], ev_[3]);
    times.strengths_ms[precision] += t01;
    times.far_ms[precision] += t12;
    times.combine_ms[precision] += t23;
    times.calls[precision] += 1;
  }
  return kOk;
}

}  // namespace bie
