// bie_farfield_dev_noalloc: the far-field sum of bie_farfield_dev without
// any device allocation.
//
// Who needs it: callers that must not (or cannot) call cudaMalloc at the
// point where they evaluate the far field -- a code whose device memory is
// owned by its own pool (a framework allocator, or a budget fixed when the
// job starts), a caller on a path where a cudaMalloc/cudaFree would stall
// other streams (cudaFree synchronises the device), or a caller running
// under a memory cap where a late allocation can fail mid-solve.  Their
// inputs and outputs are already device buffers they own; what
// bie_farfield_dev would allocate is only its scratch (the packed
// source strengths and the per-chunk partial sums).  This variant takes that
// scratch from one fixed array compiled into the library instead.
//
// Limits and sharing rules:
//  * the scratch is kNoAllocScratchBytes (48 MiB) of device memory that every
//    GPU which loads this code keeps until the process exits;
//  * it always evaluates the direct sum (FP64 or FP32 pair sums, as iprec
//    says): BIE_FAR_METHOD and BIE_TREE_PAIRS, which switch
//    bie_farfield_dev to the hierarchical sum for large calls, are ignored;
//  * ns <= kNoAllocMaxSources (1,048,576) sources, and at most 1,048,576
//    targets for Helmholtz (kind 1) or 2,097,152 for Laplace (kind 0): one
//    chunk of partial sums (one complex or real value per target) must fit
//    in the 16 MiB left after the strengths; larger calls are rejected with
//    BIE_ERR_ARG and a message;
//  * all calls share the one array: two calls whose work overlaps on the GPU
//    (different streams, or different host threads on the same device) race
//    on it and give wrong results -- order them on one stream or serialise
//    them;
//  * the first call on each device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; make
//    that first call before any stream capture begins on that device.  The
//    cached address belongs to the device's primary context: after
//    cudaDeviceReset (or anything else that destroys that context) it is
//    stale, and the process must not call this entry point on that device
//    again;
//  * nothing in the scratch needs to start at zero: each call writes every
//    strength and every partial sum it later reads, so the contents left by
//    the previous call are never used.
#include <algorithm>
#include <exception>
#include <mutex>
#include <new>
#include <string>

#include "../../../include/fmm3dbie_b200.h"
#include "device.cuh"
#include "plan.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(48) << 20;
constexpr int64_t kNoAllocMaxSources = int64_t(1) << 20;
// strengths: up to 4 doubles per source; the rest holds partial sums
constexpr size_t kStrengthBytes = size_t(kNoAllocMaxSources) * 4 * sizeof(double);
constexpr size_t kPartialBytes = kNoAllocScratchBytes - kStrengthBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (host code must
// not use the symbol itself as a pointer).
int scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices) {
    bie::set_last_error("device ordinal out of range for the no-alloc scratch table");
    return BIE_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      bie::set_last_error(std::string("cudaGetSymbolAddress(no-alloc scratch): ") +
                          cudaGetErrorString(e));
      return BIE_ERR_CUDA;
    }
    g_addr[device] = p;
  }
  *out = g_addr[device];
  return BIE_OK;
}

}  // namespace

namespace {

int farfield_noalloc(int64_t kind, const double* zk, int64_t ns, const double* src_dev,
                     const double* nrm_dev, const double* charge_dev, const double* dipstr_dev,
                     int64_t nt, const double* targ_dev, double thresh, int64_t iprec,
                     double* pot_dev, void* stream) {
  if ((kind != 0 && kind != 1) || (iprec != 0 && iprec != 1) || ns < 0 || nt < 0) {
    bie::set_last_error("bie_farfield_dev_noalloc: bad kind/iprec/sizes");
    return BIE_ERR_ARG;
  }
  if (ns > kNoAllocMaxSources) {
    bie::set_last_error("bie_farfield_dev_noalloc: ns = " + std::to_string(ns) +
                        " exceeds the fixed scratch limit of " +
                        std::to_string(kNoAllocMaxSources) + " sources");
    return BIE_ERR_ARG;
  }
  const int c = kind == 1 ? 2 : 1;
  const int64_t per_chunk = nt * c * int64_t(sizeof(double));
  if (nt > 0 && per_chunk > int64_t(kPartialBytes)) {
    bie::set_last_error("bie_farfield_dev_noalloc: nt = " + std::to_string(nt) +
                        " exceeds the fixed scratch limit of " +
                        std::to_string(kPartialBytes / (c * sizeof(double))) + " targets");
    return BIE_ERR_ARG;
  }
  if (nt == 0) return BIE_OK;
  int device = 0, sms = 148;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) {
    bie::set_last_error(cudaGetErrorString(e));
    return BIE_ERR_CUDA;
  }
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) {
    bie::set_last_error(cudaGetErrorString(e));
    return BIE_ERR_CUDA;
  }
  void* base = nullptr;
  int ier = scratch_address(device, &base);
  if (ier) return ier;
  unsigned char* scratch = static_cast<unsigned char*>(base);
  double* partial = reinterpret_cast<double*>(scratch + kStrengthBytes);
  // as many source chunks as the far kernel wants, capped by the scratch
  int nch = bie::dev::far_nchunks(nt, std::max<int64_t>(ns, 1), int(kind), int(iprec), 1, sms);
  nch = int(std::max<int64_t>(1, std::min<int64_t>(nch, int64_t(kPartialBytes) / per_chunk)));

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
  bie::dev::MatvecArgs a;
  a.precision = int(iprec);
  a.nd = 1;
  a.nchunks = nch;
  a.strengths = scratch;
  a.partial = partial;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  e = bie::dev::launch_pack_strengths(int(kind), int(iprec), ns, charge_dev, dipstr_dev, scratch, st);
  if (e == cudaSuccess) e = bie::dev::launch_far(g, kp, a, st);
  if (e == cudaSuccess) e = bie::dev::launch_reduce_partials(int(kind), partial, nch, nt, pot_dev, st);
  if (e != cudaSuccess) {
    bie::set_last_error(cudaGetErrorString(e));
    return BIE_ERR_CUDA;
  }
  return BIE_OK;
}

}  // namespace

// The C-ABI entry: no exception (a failed string or lock operation) leaves
// through it; those become an error status like every other failure.
extern "C" int bie_farfield_dev_noalloc(int64_t kind, const double* zk, int64_t ns,
                                        const double* src_dev, const double* nrm_dev,
                                        const double* charge_dev, const double* dipstr_dev,
                                        int64_t nt, const double* targ_dev, double thresh,
                                        int64_t iprec, double* pot_dev, void* stream) {
  try {
    return farfield_noalloc(kind, zk, ns, src_dev, nrm_dev, charge_dev, dipstr_dev, nt, targ_dev,
                            thresh, iprec, pot_dev, stream);
  } catch (const std::bad_alloc&) {
    bie::set_last_error("bie_farfield_dev_noalloc: host allocation failed");
    return BIE_ERR_NOMEM;
  } catch (const std::exception& ex) {
    bie::set_last_error(ex.what());
    return BIE_ERR_ARG;
  } catch (...) {
    return BIE_ERR_ARG;
  }
}
