// Device setup: near lists, far-field orders, oversampled geometry (see
// setup_gpu.h).  Each follows its host counterpart in host/setup.cpp step
// by step; only the loops over targets, patches and nodes become threads.
#include "setup_gpu.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../host/basis.h"
#include "basis_dev.cuh"
#include "plan.h"

namespace bie {
namespace {

constexpr double kSgOver4Pi = 0.07957747154594767;
// far_field_routs.f90's list of far orders {1, 2, 3, 4, 6, 8, 10, 12, 14, 16}
__host__ __device__ constexpr int far_order_at(int i) { return i < 4 ? i + 1 : 2 * i - 2; }
constexpr int kSgProbes = 25;
constexpr int kSgChunk = 32;
constexpr int kSgThreads = 128;

template <class T>
cudaError_t upload(DBuf<T>& d, const T* h, size_t n, cudaStream_t st) {
  cudaError_t e = d.alloc(std::max<size_t>(n, 1));
  if (e != cudaSuccess || n == 0) return e;
  return cudaMemcpyAsync(d.p, h, n * sizeof(T), cudaMemcpyHostToDevice, st);
}

int cuda_fail(const char* where, cudaError_t e) {
  set_last_error(std::string(where) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? kErrNoMem : kErrCuda;
}

// ---- findnear ---------------------------------------------------------------

struct NearGrid {
  double lo[3], h;
  int64_t dims[3];
};

// |c - t|^2 <= r^2 with every product and sum rounded separately, as the
// host near list decides it.
__device__ __forceinline__ bool within_radius(const double* c, const double* t, double r) {
  const double a = c[0] - t[0], b = c[1] - t[1], e = c[2] - t[2];
  const double s = __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(e, e));
  return s <= __dmul_rn(r, r);
}

// One thread per target: the patches of the 27 cells around the target's
// cell that contain it in their near sphere.  Pass 1 counts, pass 2 writes
// the 1-based patch indices at the row offset and sorts the row.
template <bool FILL>
__global__ void near_kernel(NearGrid g, const double* __restrict__ cms,
                            const double* __restrict__ rads, const int64_t* __restrict__ cstart,
                            const int64_t* __restrict__ cidx, const double* __restrict__ targ,
                            int64_t nt, int* cnt, const int64_t* off, int64_t* col) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  const double t[3] = {targ[3 * i], targ[3 * i + 1], targ[3 * i + 2]};
  int64_t c[3];
  for (int k = 0; k < 3; ++k) c[k] = int64_t(floor((t[k] - g.lo[k]) / g.h));
  const int64_t base = FILL ? off[i] : 0;
  int n = 0;
  for (int64_t dz = -1; dz <= 1; ++dz)
    for (int64_t dy = -1; dy <= 1; ++dy)
      for (int64_t dx = -1; dx <= 1; ++dx) {
        const int64_t x = c[0] + dx, y = c[1] + dy, z = c[2] + dz;
        if (x < 0 || y < 0 || z < 0 || x >= g.dims[0] || y >= g.dims[1] || z >= g.dims[2])
          continue;
        const int64_t cell = (z * g.dims[1] + y) * g.dims[0] + x;
        for (int64_t q = cstart[cell]; q < cstart[cell + 1]; ++q) {
          const int64_t j = cidx[q];
          if (within_radius(cms + 3 * j, t, rads[j])) {
            if (FILL) col[base + n] = j + 1;
            ++n;
          }
        }
      }
  if constexpr (!FILL) {
    cnt[i] = n;
  } else {
    for (int a = 1; a < n; ++a) {
      const int64_t v = col[base + a];
      int b = a - 1;
      while (b >= 0 && col[base + b] > v) {
        col[base + b + 1] = col[base + b];
        --b;
      }
      col[base + b + 1] = v;
    }
  }
}

// ---- get_far_order ------------------------------------------------------------

struct FarArgs {
  double eps, zr, zi;
  int ikerorder, np_max;
  const double* coefs;
  const int64_t* pstart;
  const int* pcls;    // 0 triangle, 1 Legendre quad, 2 Chebyshev quad
  const int* pord;    // patch order
  const int* pown;    // arena offset of the patch order's nodes
  const double* probes;  // 25 x 3 per patch
  const double* arena;
  const int* ord_off;  // [cls * 10 + order index]: nodes (2 nf) then weights (nf)
  const int* ord_nf;
  double* scratch;  // per patch: two 25 x np complex integral tables
  int64_t* nfars;
};

__device__ __forceinline__ int cls_iptype(int cls) { return cls == 0 ? 1 : (cls == 1 ? 11 : 12); }

// h3d_slp / h3d_dlp (helm_kernels.f90:18,48) at target t of the source s
// (xyz, normal at s[9..11]), k = zr + i zi.
__device__ __forceinline__ void far_kernel_val(const FarArgs& a, const double* s, const double* t,
                                               double& re, double& im) {
  const double dx = t[0] - s[0], dy = t[1] - s[1], dz = t[2] - s[2];
  const double r = sqrt(dx * dx + dy * dy + dz * dz);
  double sn, cs;
  sincos(a.zr * r, &sn, &cs);
  const double m = exp(-a.zi * r) * kSgOver4Pi;
  const double er = cs * m, ei = sn * m;  // e^{ikr} / 4pi
  if (a.ikerorder == -1) {
    re = er / r;
    im = ei / r;
    return;
  }
  const double d = dx * s[9] + dy * s[10] + dz * s[11];
  const double f = d / (r * r * r);
  const double omr = 1.0 + a.zi * r, omi = -a.zr * r;  // 1 - ikr
  re = f * (omr * er - omi * ei);
  im = f * (omr * ei + omi * er);
}

// Integrals v(it, l) = sum_j K(y_j, t_it) w_j |J_j| P_l(y_j) over the far
// nodes of order index oi; v is 25 x np complex (interleaved), it-major.
__device__ void far_integrals(const FarArgs& a, int64_t p, int oi, const double* probes,
                              double* Psh, double* val, double* v) {
  const int tid = threadIdx.x;
  const int cls = a.pcls[p], ip = cls_iptype(cls), no = a.pord[p];
  const int np = npols_dev(ip, no);
  const double* c = a.coefs + 9 * a.pstart[p];
  const int nf = a.ord_nf[cls * 10 + oi];
  const double* uvs = a.arena + a.ord_off[cls * 10 + oi];
  const double* w = uvs + 2 * nf;
  for (int i = tid; i < kSgProbes * np; i += blockDim.x) v[2 * i] = v[2 * i + 1] = 0.0;
  __syncthreads();
  for (int j0 = 0; j0 < nf; j0 += kSgChunk) {
    const int jn = min(kSgChunk, nf - j0);
    if (tid < jn) {
      const int j = j0 + tid;
      double g[9];
      basis_geom<true>(ip, no, uvs[2 * j], uvs[2 * j + 1], c, Psh + tid, kSgChunk, g);
      const double n0 = g[4] * g[8] - g[5] * g[7];
      const double n1 = g[5] * g[6] - g[3] * g[8];
      const double n2 = g[3] * g[7] - g[4] * g[6];
      const double rr = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
      const double src[12] = {g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7], g[8],
                              n0 / rr, n1 / rr, n2 / rr};
      const double qw = w[j] * rr;
      for (int it = 0; it < kSgProbes; ++it) {
        double kr, ki;
        far_kernel_val(a, src, probes + 3 * it, kr, ki);
        val[2 * (tid * kSgProbes + it)] = kr * qw;
        val[2 * (tid * kSgProbes + it) + 1] = ki * qw;
      }
    }
    __syncthreads();
    for (int i = tid; i < kSgProbes * np; i += blockDim.x) {
      const int it = i / np, l = i - it * np;
      double sr = 0.0, si = 0.0;
      for (int jj = 0; jj < jn; ++jj) {
        const double pv = Psh[l * kSgChunk + jj];
        sr = fma(val[2 * (jj * kSgProbes + it)], pv, sr);
        si = fma(val[2 * (jj * kSgProbes + it) + 1], pv, si);
      }
      v[2 * i] += sr;
      v[2 * i + 1] += si;
    }
    __syncthreads();
  }
}

// One block per patch: the tolerance eps (min |du x dv|^2)^(1/4), then the
// integrals at successive orders until two agree to it
// (host/setup.cpp far_order, far_field_routs.f90:177-330).
__global__ void __launch_bounds__(kSgThreads) far_order_kernel(FarArgs a) {
  extern __shared__ __align__(16) double sg_smem[];
  __shared__ double red[kSgThreads];
  __shared__ double probes[3 * kSgProbes];
  const int tid = threadIdx.x;
  const int64_t p = blockIdx.x;
  const int cls = a.pcls[p], ip = cls_iptype(cls), no = a.pord[p];
  const int np = npols_dev(ip, no);
  const double* c = a.coefs + 9 * a.pstart[p];
  double* Psh = sg_smem;
  double* val = Psh + size_t(kSgChunk) * a.np_max;
  for (int i = tid; i < 3 * kSgProbes; i += blockDim.x) probes[i] = a.probes[75 * p + i];
  double rmin = 1e300;
  for (int j = tid; j < np; j += blockDim.x) {
    const double* uv = a.arena + a.pown[p] + 2 * j;
    double g[9];
    basis_geom<false>(ip, no, uv[0], uv[1], c, nullptr, 0, g);
    const double n0 = g[4] * g[8] - g[5] * g[7];
    const double n1 = g[5] * g[6] - g[3] * g[8];
    const double n2 = g[3] * g[7] - g[4] * g[6];
    rmin = fmin(rmin, n0 * n0 + n1 * n1 + n2 * n2);
  }
  red[tid] = rmin;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (tid < o) red[tid] = fmin(red[tid], red[tid + o]);
    __syncthreads();
  }
  const double epsp = pow(red[0], 0.25) * a.eps;
  __syncthreads();
  double* vcomp = a.scratch + size_t(p) * 4 * kSgProbes * a.np_max;
  double* vref = vcomp + 2 * kSgProbes * a.np_max;
  far_integrals(a, p, 0, probes, Psh, val, vcomp);
  int nnn = 1;
  for (; nnn < 10; ++nnn) {
    far_integrals(a, p, nnn, probes, Psh, val, vref);
    double e = 0.0;
    if (tid < kSgProbes) {
      double e2 = 0.0;
      for (int l = 0; l < np; ++l) {
        const double dr = vref[2 * (tid * np + l)] - vcomp[2 * (tid * np + l)];
        const double di = vref[2 * (tid * np + l) + 1] - vcomp[2 * (tid * np + l) + 1];
        e2 += dr * dr + di * di;
      }
      e = sqrt(e2);
    }
    red[tid] = e;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (tid < o) red[tid] = fmax(red[tid], red[tid + o]);
      __syncthreads();
    }
    const bool done = red[0] < epsp;
    __syncthreads();
    if (done) break;
    double* t = vcomp;
    vcomp = vref;
    vref = t;
  }
  if (tid == 0) a.nfars[p] = nnn == 10 ? far_order_at(9) : far_order_at(nnn - 1);
}

// ---- oversample_geom ------------------------------------------------------------

struct OverArgs {
  const double* coefs;
  const double* srcvals;
  const int64_t* pstart;
  const int64_t* pso;  // first oversampled node, 0-based
  const int* pip;
  const int* pno;
  const int* pnf;      // far order
  const int* ptab;     // arena offset of the far nodes (2 nf), then nclash and the clash pairs
  const double* arena;
  double* srcover;
};

__global__ void __launch_bounds__(kSgThreads) oversample_kernel(OverArgs a) {
  const int64_t p = blockIdx.x;
  const int ip = a.pip[p], no = a.pno[p], nfar = a.pnf[p];
  const int np = npols_dev(ip, no), nf = npols_dev(ip, nfar);
  const int64_t st = a.pstart[p], so = a.pso[p];
  if (nfar == no) {
    for (int i = threadIdx.x; i < 12 * np; i += blockDim.x)
      a.srcover[12 * so + i] = a.srcvals[12 * st + i];
    return;
  }
  const double* uvs = a.arena + a.ptab[p];
  const double* c = a.coefs + 9 * st;
  for (int j = threadIdx.x; j < nf; j += blockDim.x) {
    double g[9];
    basis_geom<false>(ip, no, uvs[2 * j], uvs[2 * j + 1], c, nullptr, 0, g);
    double* o = a.srcover + 12 * (so + j);
    for (int k = 0; k < 9; ++k) o[k] = g[k];
    const double n0 = g[4] * g[8] - g[5] * g[7];
    const double n1 = g[5] * g[6] - g[3] * g[8];
    const double n2 = g[3] * g[7] - g[4] * g[6];
    const double r = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    o[9] = n0 / r;
    o[10] = n1 / r;
    o[11] = n2 / r;
  }
  __syncthreads();
  // nodes shared by the two orders keep the given values (get_clashing_indices)
  const double* cl = uvs + 2 * nf;
  const int nclash = int(cl[0]);
  for (int q = threadIdx.x; q < nclash; q += blockDim.x) {
    const int ic = int(cl[1 + 2 * q]), icf = int(cl[2 + 2 * q]);
    for (int k = 0; k < 12; ++k) a.srcover[12 * (so + icf) + k] = a.srcvals[12 * (st + ic) + k];
  }
}

}  // namespace

int findnear_gpu(int64_t npatches, const double* cms, const double* rads, int ndt, int64_t nt,
                 const double* targs, std::vector<int64_t>& row_ptr,
                 std::vector<int64_t>& col_ind, cudaStream_t st) {
  row_ptr.assign(size_t(std::max<int64_t>(nt, 0)) + 1, 1);
  col_ind.clear();
  if (nt <= 0 || npatches <= 0) return kOk;
  // the host's grid: cells of size >= the largest radius over the centroids'
  // bounding box, grown until there are at most 8 npatches + 64 cells
  NearGrid g;
  double rmax = 0, hi[3] = {-1e300, -1e300, -1e300};
  for (int k = 0; k < 3; ++k) g.lo[k] = 1e300;
  for (int64_t j = 0; j < npatches; ++j) {
    rmax = std::max(rmax, rads[j]);
    for (int k = 0; k < 3; ++k) {
      g.lo[k] = std::min(g.lo[k], cms[3 * j + k]);
      hi[k] = std::max(hi[k], cms[3 * j + k]);
    }
  }
  g.h = std::max(rmax, 1e-300);
  for (int k = 0; k < 3; ++k) g.dims[k] = std::max<int64_t>(1, int64_t((hi[k] - g.lo[k]) / g.h) + 1);
  while (g.dims[0] * g.dims[1] * g.dims[2] > 8 * npatches + 64) {
    g.h *= 1.5;
    for (int k = 0; k < 3; ++k)
      g.dims[k] = std::max<int64_t>(1, int64_t((hi[k] - g.lo[k]) / g.h) + 1);
  }
  const int64_t ncell = g.dims[0] * g.dims[1] * g.dims[2];
  std::vector<int64_t> cstart(ncell + 1, 0), cidx(npatches), cellid(npatches);
  for (int64_t j = 0; j < npatches; ++j) {
    int64_t c[3];
    for (int k = 0; k < 3; ++k) {
      c[k] = int64_t(std::floor((cms[3 * j + k] - g.lo[k]) / g.h));
      c[k] = std::min(std::max<int64_t>(c[k], 0), g.dims[k] - 1);
    }
    cellid[j] = (c[2] * g.dims[1] + c[1]) * g.dims[0] + c[0];
    cstart[cellid[j] + 1]++;
  }
  for (int64_t i = 0; i < ncell; ++i) cstart[i + 1] += cstart[i];
  {
    std::vector<int64_t> fill(cstart.begin(), cstart.end() - 1);
    for (int64_t j = 0; j < npatches; ++j) cidx[fill[cellid[j]]++] = j;
  }
  std::vector<double> t3(3 * size_t(nt));
  for (int64_t i = 0; i < nt; ++i)
    for (int k = 0; k < 3; ++k) t3[3 * i + k] = targs[size_t(ndt) * i + k];
  DBuf<double> d_cms, d_rads, d_targ;
  DBuf<int64_t> d_cstart, d_cidx, d_off, d_col;
  DBuf<int> d_cnt;
  cudaError_t e;
  if ((e = upload(d_cms, cms, 3 * size_t(npatches), st)) != cudaSuccess ||
      (e = upload(d_rads, rads, size_t(npatches), st)) != cudaSuccess ||
      (e = upload(d_targ, t3.data(), t3.size(), st)) != cudaSuccess ||
      (e = upload(d_cstart, cstart.data(), cstart.size(), st)) != cudaSuccess ||
      (e = upload(d_cidx, cidx.data(), cidx.size(), st)) != cudaSuccess ||
      (e = d_cnt.alloc(size_t(nt))) != cudaSuccess)
    return cuda_fail("findnear_gpu", e);
  const unsigned blocks = unsigned((nt + 255) / 256);
  near_kernel<false><<<blocks, 256, 0, st>>>(g, d_cms.p, d_rads.p, d_cstart.p, d_cidx.p, d_targ.p,
                                             nt, d_cnt.p, nullptr, nullptr);
  std::vector<int> cnt(nt);
  if ((e = cudaMemcpyAsync(cnt.data(), d_cnt.p, nt * sizeof(int), cudaMemcpyDeviceToHost, st)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cuda_fail("findnear_gpu", e);
  std::vector<int64_t> off(nt);
  for (int64_t i = 0; i < nt; ++i) {
    off[i] = row_ptr[i] - 1;
    row_ptr[i + 1] = row_ptr[i] + cnt[i];
  }
  const int64_t nnz = row_ptr[nt] - 1;
  col_ind.resize(size_t(nnz));
  if (nnz == 0) return kOk;
  if ((e = upload(d_off, off.data(), off.size(), st)) != cudaSuccess ||
      (e = d_col.alloc(size_t(nnz))) != cudaSuccess)
    return cuda_fail("findnear_gpu", e);
  near_kernel<true><<<blocks, 256, 0, st>>>(g, d_cms.p, d_rads.p, d_cstart.p, d_cidx.p, d_targ.p,
                                            nt, nullptr, d_off.p, d_col.p);
  dev::note_launches(2);
  if ((e = cudaMemcpyAsync(col_ind.data(), d_col.p, nnz * sizeof(int64_t), cudaMemcpyDeviceToHost,
                           st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess)
    return cuda_fail("findnear_gpu", e);
  return kOk;
}

int far_order_gpu(double eps, const Surf& s, const double* cms, const double* rads, int ndt,
                  int64_t nt, const double* targs, int ikerorder, cdouble zk, int64_t nnz,
                  const int64_t* row_ptr, const int64_t* col_ind, double rfac, int64_t* nfars,
                  int64_t* ixyzso, cudaStream_t st) {
  const int64_t npat = s.npatches;
  // node tables: per class and order of the list, and the patches' own orders
  std::vector<double> arena;
  std::vector<int> ord_off(30, 0), ord_nf(30, 0);
  const int cls_ip[3] = {1, 11, 12};
  bool used[3] = {false, false, false};
  std::vector<int> pcls(npat), pord(npat), pown(npat);
  std::vector<int64_t> pstart(npat);
  std::map<std::pair<int, int>, int> own;
  int np_max = 0;
  for (int64_t p = 0; p < npat; ++p) {
    const int ip = int(s.iptype[p]), no = int(s.norders[p]);
    const int cls = ip == 1 ? 0 : (ip == 11 ? 1 : 2);
    if (!valid_patch(ip, no) || npols_of(ip, no) != s.npols(p)) {
      set_last_error("far_order_gpu: patch " + std::to_string(p + 1) + " has an invalid type/order");
      return kErrArg;
    }
    used[cls] = true;
    pcls[p] = cls;
    pord[p] = no;
    pstart[p] = s.start(p);
    np_max = std::max(np_max, int(s.npols(p)));
    auto key = std::make_pair(ip, no);
    auto f = own.find(key);
    if (f == own.end()) {
      std::vector<double> uv(2 * npols_of(ip, no));
      if (disc_nodes(ip, no, uv.data())) {
        set_last_error("far_order_gpu: no node table for a patch type");
        return kErrTables;
      }
      f = own.emplace(key, int(arena.size())).first;
      arena.insert(arena.end(), uv.begin(), uv.end());
    }
    pown[p] = f->second;
  }
  if (np_max > 256) {
    set_last_error("far_order_gpu: patches with more than 256 basis functions");
    return kErrArg;
  }
  for (int cls = 0; cls < 3; ++cls) {
    if (!used[cls]) continue;
    for (int oi = 0; oi < 10; ++oi) {
      const int ip = cls_ip[cls], nf = npols_of(ip, far_order_at(oi));
      std::vector<double> uv(2 * nf), w(nf);
      if (disc_nodes(ip, far_order_at(oi), uv.data()) || disc_wts(ip, far_order_at(oi), w.data())) {
        set_last_error("far_order_gpu: no node table for a far order");
        return kErrTables;
      }
      ord_off[cls * 10 + oi] = int(arena.size());
      ord_nf[cls * 10 + oi] = nf;
      arena.insert(arena.end(), uv.begin(), uv.end());
      arena.insert(arena.end(), w.begin(), w.end());
    }
  }
  // probe targets per patch, exactly as far_order chooses them
  std::vector<int64_t> col_ptr(npat + 1), row_ind(nnz), iper(nnz);
  rsc_to_csc(npat, nt, nnz, row_ptr, col_ind, col_ptr.data(), row_ind.data(), iper.data());
  std::vector<double> probes(75 * size_t(npat));
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t p = 0; p < npat; ++p) {
    const double* cm = cms + 3 * p;
    const double rad0 = rfac * rads[p];
    const int64_t ntp = col_ptr[p + 1] - col_ptr[p];
    std::vector<std::pair<double, int64_t>> dd(ntp);
    for (int64_t q = 0; q < ntp; ++q) {
      const double* t = targs + size_t(ndt) * (row_ind[col_ptr[p] - 1 + q] - 1);
      dd[q] = {(t[0] - cm[0]) * (t[0] - cm[0]) + (t[1] - cm[1]) * (t[1] - cm[1]) +
                   (t[2] - cm[2]) * (t[2] - cm[2]),
               q};
    }
    std::stable_sort(dd.begin(), dd.end(),
                     [](const auto& a, const auto& b) { return a.first < b.first; });
    const int i0 = int(std::min<int64_t>(10, ntp / 2));
    double* tt = probes.data() + 75 * p;
    for (int i = 0; i < i0; ++i) {
      const double* t = targs + size_t(ndt) * (row_ind[col_ptr[p] - 1 + dd[ntp - 1 - i].second] - 1);
      for (int k = 0; k < 3; ++k) tt[3 * i + k] = t[k];
    }
    for (int i = i0; i < kSgProbes; ++i) {
      const double ph = hkrand(1001 + i + 1) * 2 * M_PI;
      const double th = hkrand(3042 + i + 1) * M_PI;
      tt[3 * i + 0] = cm[0] + rad0 * std::sin(th) * std::cos(ph);
      tt[3 * i + 1] = cm[1] + rad0 * std::sin(th) * std::sin(ph);
      tt[3 * i + 2] = cm[2] + rad0 * std::cos(th);
    }
    if (ntp < 0) bad = 1;
  }
  if (bad) {
    set_last_error("far_order_gpu: inconsistent near list");
    return kErrArg;
  }
  DBuf<double> d_coefs, d_probes, d_arena, d_scratch;
  DBuf<int64_t> d_pstart, d_nfars;
  DBuf<int> d_cls, d_ord, d_own, d_ooff, d_onf;
  cudaError_t e;
  if ((e = upload(d_coefs, s.srccoefs, 9 * size_t(s.npts), st)) != cudaSuccess ||
      (e = upload(d_probes, probes.data(), probes.size(), st)) != cudaSuccess ||
      (e = upload(d_arena, arena.data(), arena.size(), st)) != cudaSuccess ||
      (e = upload(d_pstart, pstart.data(), pstart.size(), st)) != cudaSuccess ||
      (e = upload(d_cls, pcls.data(), pcls.size(), st)) != cudaSuccess ||
      (e = upload(d_ord, pord.data(), pord.size(), st)) != cudaSuccess ||
      (e = upload(d_own, pown.data(), pown.size(), st)) != cudaSuccess ||
      (e = upload(d_ooff, ord_off.data(), ord_off.size(), st)) != cudaSuccess ||
      (e = upload(d_onf, ord_nf.data(), ord_nf.size(), st)) != cudaSuccess ||
      (e = d_scratch.alloc(size_t(npat) * 4 * kSgProbes * np_max)) != cudaSuccess ||
      (e = d_nfars.alloc(size_t(npat))) != cudaSuccess)
    return cuda_fail("far_order_gpu", e);
  fill_basis_constants(st);
  FarArgs a;
  a.eps = eps;
  a.zr = zk.real();
  a.zi = zk.imag();
  a.ikerorder = ikerorder;
  a.np_max = np_max;
  a.coefs = d_coefs.p;
  a.pstart = d_pstart.p;
  a.pcls = d_cls.p;
  a.pord = d_ord.p;
  a.pown = d_own.p;
  a.probes = d_probes.p;
  a.arena = d_arena.p;
  a.ord_off = d_ooff.p;
  a.ord_nf = d_onf.p;
  a.scratch = d_scratch.p;
  a.nfars = d_nfars.p;
  const size_t smem = sizeof(double) * (size_t(kSgChunk) * np_max + 2 * kSgChunk * kSgProbes);
  if ((e = cudaFuncSetAttribute(far_order_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(smem))) != cudaSuccess)
    return cuda_fail("far_order_gpu", e);
  far_order_kernel<<<unsigned(npat), kSgThreads, smem, st>>>(a);
  dev::note_launches(1);
  if ((e = cudaMemcpyAsync(nfars, d_nfars.p, npat * sizeof(int64_t), cudaMemcpyDeviceToHost,
                           st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess)
    return cuda_fail("far_order_gpu", e);
  int err = 0;
  ixyzso[0] = 1;
  for (int64_t p = 0; p < npat; ++p) {
    const int nf = npols_of(int(s.iptype[p]), int(nfars[p]));
    if (nf > 289) err = 1;
    ixyzso[p + 1] = ixyzso[p] + nf;
  }
  return err ? kErrArg : kOk;
}

int oversample_geom_gpu(const Surf& s, const int64_t* nfars, const int64_t* ixyzso,
                        int64_t nptso, double* srcover, cudaStream_t st) {
  const int64_t npat = s.npatches;
  std::vector<double> arena;
  std::map<std::array<int, 3>, int> tab;
  std::vector<int> pip(npat), pno(npat), pnf(npat), ptab(npat);
  std::vector<int64_t> pstart(npat), pso(npat);
  for (int64_t p = 0; p < npat; ++p) {
    const int ip = int(s.iptype[p]), no = int(s.norders[p]), nfar = int(nfars[p]);
    const int nf = npols_of(ip, nfar);
    if (!valid_patch(ip, nfar) || nf != ixyzso[p + 1] - ixyzso[p] ||
        npols_of(ip, no) != s.npols(p) || ixyzso[p + 1] - 1 > nptso) {
      set_last_error("oversample_geom_gpu: patch " + std::to_string(p + 1) +
                     " has inconsistent orders or offsets");
      return kErrArg;
    }
    pip[p] = ip;
    pno[p] = no;
    pnf[p] = nfar;
    pstart[p] = s.start(p);
    pso[p] = ixyzso[p] - 1;
    const std::array<int, 3> key{ip, no, nfar};
    auto f = tab.find(key);
    if (f == tab.end()) {
      std::vector<double> uv(2 * nf);
      if (disc_nodes(ip, nfar, uv.data())) {
        set_last_error("oversample_geom_gpu: no node table for a far order");
        return kErrTables;
      }
      std::vector<int> ic(std::max(nf, npols_of(ip, no))), icf(ic.size());
      const int nclash = nfar == no ? 0 : clashing_indices(ip, no, nfar, ic.data(), icf.data());
      f = tab.emplace(key, int(arena.size())).first;
      arena.insert(arena.end(), uv.begin(), uv.end());
      arena.push_back(double(nclash));
      for (int q = 0; q < nclash; ++q) {
        arena.push_back(double(ic[q]));
        arena.push_back(double(icf[q]));
      }
    }
    ptab[p] = f->second;
  }
  DBuf<double> d_coefs, d_vals, d_arena, d_over;
  DBuf<int64_t> d_pstart, d_pso;
  DBuf<int> d_ip, d_no, d_nf, d_tab;
  cudaError_t e;
  if ((e = upload(d_coefs, s.srccoefs, 9 * size_t(s.npts), st)) != cudaSuccess ||
      (e = upload(d_vals, s.srcvals, 12 * size_t(s.npts), st)) != cudaSuccess ||
      (e = upload(d_arena, arena.data(), arena.size(), st)) != cudaSuccess ||
      (e = upload(d_pstart, pstart.data(), pstart.size(), st)) != cudaSuccess ||
      (e = upload(d_pso, pso.data(), pso.size(), st)) != cudaSuccess ||
      (e = upload(d_ip, pip.data(), pip.size(), st)) != cudaSuccess ||
      (e = upload(d_no, pno.data(), pno.size(), st)) != cudaSuccess ||
      (e = upload(d_nf, pnf.data(), pnf.size(), st)) != cudaSuccess ||
      (e = upload(d_tab, ptab.data(), ptab.size(), st)) != cudaSuccess ||
      (e = d_over.alloc(12 * size_t(nptso))) != cudaSuccess)
    return cuda_fail("oversample_geom_gpu", e);
  fill_basis_constants(st);
  OverArgs a;
  a.coefs = d_coefs.p;
  a.srcvals = d_vals.p;
  a.pstart = d_pstart.p;
  a.pso = d_pso.p;
  a.pip = d_ip.p;
  a.pno = d_no.p;
  a.pnf = d_nf.p;
  a.ptab = d_tab.p;
  a.arena = d_arena.p;
  a.srcover = d_over.p;
  oversample_kernel<<<unsigned(npat), kSgThreads, 0, st>>>(a);
  dev::note_launches(1);
  if ((e = cudaMemcpyAsync(srcover, d_over.p, 12 * size_t(nptso) * sizeof(double),
                           cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess)
    return cuda_fail("oversample_geom_gpu", e);
  return kOk;
}

}  // namespace bie
