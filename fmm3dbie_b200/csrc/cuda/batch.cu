// BatchPlan: many surfaces of uneven size as one operator.  Each matvec
// stage (strengths or oversampling, far field, near correction) is one
// persistent launch walking a work list that spans all surfaces; the three
// launches are captured once per (precision, nd) in a CUDA graph.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <string>

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

template <class T>
cudaError_t upload_vec(DBuf<T>& b, const std::vector<T>& h, cudaStream_t st) {
  cudaError_t e = b.alloc(std::max<size_t>(h.size(), 1));
  if (e != cudaSuccess || h.empty()) return e;
  return cudaMemcpyAsync(b.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}

constexpr int kFarTileSources = dev::kFarTileSources;

}  // namespace

BatchPlan::~BatchPlan() {
  for (auto& kv : cfg_)
    if (kv.second && kv.second->graph) cudaGraphExecDestroy(kv.second->graph);
}

int BatchPlan::add(Plan* p) {
  if (!p || !p->square()) {
    set_last_error("batch surfaces must be on-surface plans (targets = nodes)");
    return kErrArg;
  }
  if (kind >= 0 && p->kind != kind) {
    set_last_error("all surfaces of a batch must have the same kernel kind");
    return kErrArg;
  }
  if (!plans.empty() && p->device != plans.front()->device) {
    set_last_error("all surfaces of a batch must live on one device");
    return kErrArg;
  }
  kind = p->kind;
  if (p->kp.ki != 0.0) ck = true;
  plans.emplace_back(p);
  return kOk;
}

bool BatchPlan::square() const {
  if (plans.empty()) return false;
  for (const auto& p : plans)
    if (!p->square()) return false;
  return true;
}

int BatchPlan::finalize(cudaStream_t st) {
  if (plans.empty()) {
    set_last_error("empty batch");
    return kErrArg;
  }
  const Plan& p0 = *plans.front();
  cplx = p0.cplx;
  device = p0.device;
  num_sms = p0.num_sms;
  seg_start.assign(1, 0);
  nptso_total_ = 0;
  max_np_ = 0;
  for (const auto& p : plans) {
    seg_start.push_back(seg_start.back() + p->npts);
    nptso_total_ += p->nptso;
    max_np_ = std::max(max_np_, p->g.max_np);
  }
  nodes = seg_start.back();
  BIE_CUDA(wts_.alloc(size_t(nodes)));
  for (size_t s = 0; s < plans.size(); ++s)
    BIE_CUDA(cudaMemcpyAsync(wts_.p + seg_start[s], plans[s]->d_wts(),
                             size_t(plans[s]->npts) * sizeof(double), cudaMemcpyDeviceToDevice, st));
  d_node_wts = wts_.p;
  live_host_.assign(plans.size(), 1);
  std::vector<int> ones(plans.size(), 1);
  BIE_CUDA(upload_vec(live_, ones, st));
  return init_segments(st);  // synchronises st before `ones` goes
}

int BatchPlan::set_active(const std::vector<uint8_t>& active, cudaStream_t st) {
  if (active.size() != plans.size()) {
    set_last_error("active mask size differs from the number of surfaces");
    return kErrArg;
  }
  if (active == live_host_) return kOk;
  live_host_ = active;
  std::vector<int> h(active.begin(), active.end());
  // pageable source: staged before cudaMemcpyAsync returns
  BIE_CUDA(cudaMemcpyAsync(live_.p, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  return kOk;
}

int BatchPlan::build_config(int precision, int nd, int variant, int64_t chunk, Config& c,
                            cudaStream_t st) {
  const int C = cplx ? 2 : 1;
  int tpb = 0, grp = 1;
  dev::batch_far_shape(precision, variant, nd, &tpb, &grp);
  const int groups = nd == 1 ? 1 : (nd + grp - 1) / grp;
  std::vector<dev::BatchSurf> hs(plans.size());
  std::vector<int2> patch_items, row_items;
  std::vector<int4> far_items;
  int64_t vofs = 0, sofs = 0, pofs = 0;
  for (size_t s = 0; s < plans.size(); ++s) {
    const Plan& p = *plans[s];
    dev::BatchSurf& d = hs[s];
    d.g = p.g;
    d.nr = p.nr;
    d.kp = p.kp;
    d.weff[0] = p.weff_ptr(0);
    d.weff[1] = p.weff_ptr(1);
    d.ab[0] = p.ab_ptr(0);
    d.ab[1] = p.ab_ptr(1);
    d.vofs = vofs;
    d.sofs = sofs;
    d.live = live_.p + s;
    const int64_t nch = std::max<int64_t>(1, (p.nptso + chunk - 1) / chunk);
    d.chunk_len[precision] = chunk;
    d.nchunks[precision] = int(nch);
    d.pofs[precision] = pofs;
    pofs += nch * p.ntarg * nd * C;
    const int64_t tblocks = (p.ntarg + tpb - 1) / tpb;
    for (int64_t tb = 0; tb < tblocks; ++tb)
      for (int64_t ch = 0; ch < nch; ++ch)
        for (int gq = 0; gq < groups; ++gq)
          far_items.push_back(make_int4(int(s), int(tb), int(ch), gq));
    for (int64_t q = 0; q < p.npatches; ++q) patch_items.push_back(make_int2(int(s), int(q)));
    for (int64_t r = 0; r < (p.ntarg + 7) / 8; ++r) row_items.push_back(make_int2(int(s), int(r)));
    vofs += p.npts;
    sofs += p.nptso;
  }
  // largest items first: the far kernels draw items in list order as blocks
  // become free, so the cheap ones (partial chunks, short target blocks of
  // small surfaces) fill the tail
  {
    auto cost = [&](const int4& it) {
      const Plan& p = *plans[size_t(it.x)];
      const int64_t nt = std::min<int64_t>(tpb, p.ntarg - int64_t(it.y) * tpb);
      const int64_t ns = std::min<int64_t>(chunk, p.nptso - int64_t(it.z) * chunk);
      return nt * ns;
    };
    std::stable_sort(far_items.begin(), far_items.end(),
                     [&](const int4& a, const int4& b) { return cost(a) > cost(b); });
  }
  if (far_items.size() > size_t(INT32_MAX)) {
    set_last_error("batch work list too long");
    return kErrArg;
  }
  BIE_CUDA(upload_vec(c.surfs, hs, st));
  BIE_CUDA(upload_vec(c.patch_items, patch_items, st));
  BIE_CUDA(upload_vec(c.row_items, row_items, st));
  BIE_CUDA(upload_vec(c.far_items, far_items, st));
  // strengths: nd == 1 -> (c, d) per source; nd > 1 -> oversampled densities
  const size_t sbytes = size_t(nptso_total_) * size_t(nd) * 4 * (precision == 1 ? 4 : 8);
  BIE_CUDA(c.str.alloc(sbytes));
  BIE_CUDA(c.partial.alloc(size_t(std::max<int64_t>(pofs, 1))));
  BIE_CUDA(c.refs.alloc(2));
  BIE_CUDA(c.counter.alloc(1));
  c.variant = variant;
  c.chunk = chunk;
  dev::BatchArgs& a = c.args;
  a.kind = kind;
  a.precision = precision;
  a.nd = nd;
  a.variant = variant;
  a.ck = ck;
  a.surfs = c.surfs.p;
  a.patch_items = c.patch_items.p;
  a.far_items = c.far_items.p;
  a.row_items = c.row_items.p;
  a.npatch_items = int(patch_items.size());
  a.nfar_items = int(far_items.size());
  a.nrow_items = int(row_items.size());
  a.xref = reinterpret_cast<const double* const*>(c.refs.p);
  a.yref = reinterpret_cast<double* const*>(c.refs.p + 1);
  a.str = c.str.p;
  a.partial = c.partial.p;
  a.far_counter = c.counter.p;
  const int bps = std::max(1, dev::batch_far_blocks_per_sm(kind, precision, variant, nd, ck));
  a.grid_far = int(std::min<int64_t>(int64_t(far_items.size()), int64_t(num_sms) * bps));
  a.grid_patch = int(std::min<int64_t>(int64_t(patch_items.size()), int64_t(num_sms) * 8));
  a.grid_row = int(std::min<int64_t>(int64_t(row_items.size()), int64_t(num_sms) * 4));
  a.max_np = max_np_;
  // the host vectors feed async copies: finish them before they go
  BIE_CUDA(cudaStreamSynchronize(st));
  return kOk;
}

int BatchPlan::tune(int precision, int nd, cudaStream_t st, std::unique_ptr<Config>& out) {
  // candidates: the three block shapes x source chunks sized for about
  // {2, 4, 8} waves of resident blocks over the whole batch
  int64_t tot_blocks = 0;
  std::vector<std::pair<int, int64_t>> cand;
  for (int v = 0; v < dev::batch_far_variants(precision, nd); ++v) {
    int tpb = 0, grp = 1;
    dev::batch_far_shape(precision, v, nd, &tpb, &grp);
    const int groups = nd == 1 ? 1 : (nd + grp - 1) / grp;
    tot_blocks = 0;
    for (const auto& p : plans) tot_blocks += (p->ntarg + tpb - 1) / tpb * groups;
    const int bps = std::max(1, dev::batch_far_blocks_per_sm(kind, precision, v, nd, ck));
    const double slots = double(num_sms) * bps;
    for (double waves : {2.0, 4.0, 8.0}) {
      // items = sum_s tblocks_s * ceil(nptso_s / chunk) ~ nptso_total * tot_blocks / (n * chunk)
      const double want_items = slots * waves;
      const double avg_nptso = double(nptso_total_) / double(plans.size());
      int64_t chunk = int64_t(avg_nptso * double(tot_blocks) / std::max(1.0, want_items));
      chunk = std::max<int64_t>(kFarTileSources, (chunk + kFarTileSources - 1) / kFarTileSources * kFarTileSources);
      cand.emplace_back(v, chunk);
    }
  }
  // BIE_BATCH_VARIANT / BIE_BATCH_CHUNK pin the far shape and chunk length
  if (const char* ev = std::getenv("BIE_BATCH_VARIANT")) {
    const int v = std::min(std::max(std::atoi(ev), 0), dev::batch_far_variants(precision, nd) - 1);
    const char* ec = std::getenv("BIE_BATCH_CHUNK");
    int64_t chunk = ec ? std::max<int64_t>(kFarTileSources, std::atoll(ec)) : cand.front().second;
    chunk = (chunk + kFarTileSources - 1) / kFarTileSources * kFarTileSources;
    cand.assign(1, {v, chunk});
  }
  std::unique_ptr<Config> best;
  float best_ms = 1e30f;
  cudaEvent_t e0, e1;
  BIE_CUDA(cudaEventCreate(&e0));
  BIE_CUDA(cudaEventCreate(&e1));
  DBuf<double> xin, yout;
  const size_t len = size_t(nodes) * nd * (cplx ? 2 : 1);
  BIE_CUDA(xin.alloc(len));
  BIE_CUDA(yout.alloc(len));
  BIE_CUDA(cudaMemsetAsync(xin.p, 0, len * sizeof(double), st));
  for (const auto& cv : cand) {
    auto c = std::make_unique<Config>();
    int ier = build_config(precision, nd, cv.first, cv.second, *c, st);
    if (ier) return ier;
    void* refs[2] = {xin.p, yout.p};
    BIE_CUDA(cudaMemcpyAsync(c->refs.p, refs, sizeof(refs), cudaMemcpyHostToDevice, st));
    BIE_CUDA(dev::launch_batch_matvec(c->args, st));  // warm
    BIE_CUDA(cudaEventRecord(e0, st));
    BIE_CUDA(dev::launch_batch_matvec(c->args, st));
    BIE_CUDA(cudaEventRecord(e1, st));
    BIE_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
      best = std::move(c);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  out = std::move(best);
  return kOk;
}

bool BatchPlan::far_choice(int precision, int nd, int* variant, int64_t* chunk) const {
  auto it = cfg_.find({precision, nd});
  if (it == cfg_.end()) return false;
  *variant = it->second->variant;
  *chunk = it->second->chunk;
  return true;
}

int BatchPlan::apply(int precision, int nd, const double* x, double* y, cudaStream_t st) {
  if (plans.empty() || nodes == 0) {
    set_last_error("batch not finalised");
    return kErrArg;
  }
  if (nd < 1 || nd > 256 || (precision != 0 && precision != 1)) return kErrArg;
  auto key = std::make_pair(precision, nd);
  auto it = cfg_.find(key);
  if (it == cfg_.end()) {
    std::unique_ptr<Config> c;
    int ier = tune(precision, nd, st, c);
    if (ier) return ier;
    it = cfg_.emplace(key, std::move(c)).first;
  }
  Config& c = *it->second;
  // the launches read the vectors through c.refs (pageable copy: staged
  // before cudaMemcpyAsync returns, so `refs` may go out of scope)
  void* refs[2] = {const_cast<double*>(x), y};
  BIE_CUDA(cudaMemcpyAsync(c.refs.p, refs, sizeof(refs), cudaMemcpyHostToDevice, st));
  if (!use_graph) {
    BIE_CUDA(dev::launch_batch_matvec(c.args, st));
    return kOk;
  }
  if (!c.graph) {
    // record on a private stream (the caller's may be the legacy default
    // stream, which cannot be captured); the graph then replays on `st`
    cudaGraph_t g = nullptr;
    cudaStream_t cap = nullptr;
    BIE_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaError_t be = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    const cudaError_t le = be == cudaSuccess ? dev::launch_batch_matvec(c.args, cap) : be;
    const cudaError_t ce = be == cudaSuccess ? cudaStreamEndCapture(cap, &g) : be;
    cudaStreamDestroy(cap);
    if (le != cudaSuccess || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      set_last_error(std::string("batch matvec capture: ") +
                     cudaGetErrorString(le != cudaSuccess ? le : ce));
      return kErrCuda;
    }
    const cudaError_t ie = cudaGraphInstantiate(&c.graph, g, 0);
    cudaGraphDestroy(g);
    BIE_CUDA(ie);
  }
  BIE_CUDA(cudaGraphLaunch(c.graph, st));
  dev::note_launches(3);
  return kOk;
}

}  // namespace bie
