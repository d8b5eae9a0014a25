// Device-side data layout and kernel entry points for the locally corrected
// combined-field matvec (Laplace and Helmholtz), sm_100a.
//
// HBM layout of one operator plan (all arrays SoA, 0-based):
//   targets       : tx,ty,tz            f64[ntarg] each
//   oversampled   : sx,sy,sz,nx,ny,nz,w f64[nptso] each (srcover, whtsover)
//   patches       : pstart[npatches+1], ostart[npatches+1] (node offsets),
//                   pclass[npatches] -> interpolation matrix of the class
//                   (iptype, norder, nfar): imat[nf x np] f64 (row-major)
//   near matrix   : row_ptr[ntarg+1] (into col/wofs), col[nnz] patch index,
//                   wofs[nnz+1] entry offsets (iquad-1), nps[nnz] first
//                   node of each near patch,
//                   W_eff[nquad] = wnear - smooth oversampled part, stored
//                   f64 (and f32 for the mixed-precision path);
//                   complex values are interleaved (re, im).
// Densities are stored point-major with nd densities per point
// (sigma[(pt*nd + m)], the reference's sigma(ndim, npts)), complex
// interleaved.  Per matvec the strength kernel writes per-source
// charge/dipole strengths (scaled by alpha, beta, w and 1/(4 pi)), the far
// kernel writes per-chunk partial potentials (scratch), and the combine
// kernel sums the partials and the near correction into pot.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bie {
namespace dev {

struct Geometry {
  int64_t ntarg = 0, nptso = 0, npatches = 0, npts = 0;
  const double* tx = nullptr;
  const double* ty = nullptr;
  const double* tz = nullptr;
  const double* sx = nullptr;
  const double* sy = nullptr;
  const double* sz = nullptr;
  const double* snx = nullptr;
  const double* sny = nullptr;
  const double* snz = nullptr;
  const double* sw = nullptr;
  const int32_t* pstart = nullptr;   // npatches+1
  const int32_t* ostart = nullptr;   // npatches+1
  const int32_t* pclass = nullptr;   // npatches
  const int64_t* cmoff = nullptr;    // per class offset into imat
  const double* imat = nullptr;
  int max_np = 0, max_nf = 0;
  // Bounding boxes (lo xyz, hi xyz) of the FP32 far kernel's target blocks
  // (kFarBlockTargets32 targets) and source tiles (kFarTileSources sources),
  // and the squared gap below which a tile may hold a pair closer than the
  // self-interaction threshold (threshold plus a margin for FP32 rounding).
  const double* tbox = nullptr;
  const double* sbox = nullptr;
  double box_margin2 = 0.0;
  // FP32 coordinate centre per target (3 doubles) of the hierarchical far
  // field; null for the direct far kernels (first target of each block)
  const double* tcen = nullptr;
};
constexpr int kFarBlockTargets32 = 512;
constexpr int kFarTileSources = 128;

struct Near {
  int64_t nnz = 0, nquad = 0;
  const int64_t* row_ptr = nullptr;  // ntarg+1
  const int32_t* col = nullptr;      // nnz
  const int64_t* wofs = nullptr;     // nnz+1
  const int32_t* nps = nullptr;      // nnz: first node of patch col[k] (pstart[col[k]])
};

// Kernel constants. kind 0: Laplace (real alpha, beta), 1: Helmholtz.
struct KParams {
  int kind = 0;
  double ar = 0, ai = 0, br = 0, bi = 0, kr = 0, ki = 0;
  double thresh = 0;
};

// precision: 0 = f64 far field, 1 = f32 far field (f64 accumulation across
// source tiles).
struct MatvecArgs {
  int precision = 0;
  int nd = 1;
  int nchunks = 1;
  const double* sigma = nullptr;  // npts*nd (x2 if complex)
  double* pot = nullptr;          // ntarg*nd (x2 if complex)
  void* strengths = nullptr;      // nptso*nd*(2 or 4) reals of the far precision
  double* partial = nullptr;      // nchunks*ntarg*nd*(1 or 2)
  const void* weff = nullptr;     // W_eff in f64 or f32
  int weff_f32 = 0;
  int far_variant = 0;            // far-kernel block shape (see far_block_targets)
  const void* ab = nullptr;       // per-source constants for the multi-density kernel
  int* tc_err = nullptr;          // set by the tensor-core far field if a completion wait timed out
  const int32_t* sdest = nullptr; // strengths: source s is stored at position sdest[s]
};

cudaError_t launch_strengths(const Geometry& g, const KParams& kp, const MatvecArgs& a,
                             cudaStream_t st);
cudaError_t launch_far(const Geometry& g, const KParams& kp, const MatvecArgs& a,
                       cudaStream_t st);
cudaError_t launch_combine(const Geometry& g, const Near& nr, const KParams& kp,
                           const MatvecArgs& a, cudaStream_t st);
// W_eff = wnear - [K(t_i, y_l) w_l]_l * imat  for every near pair.
// match32 = 0: exact FP64 kernel, weff is double* (may alias wnear);
// match32 = 1: kernel values as the FP32 far kernel computes them
// (same centring and pair functions), weff is float*.
// match32 = 2: wnear is the FP64 W_eff; weff (float*) = wnear + exact part -
// FP32-matched part (an FP32 W_eff for another far-field centring).
// Near pairs k0 .. k1 - 1 only (k1 < 0: to the last pair).
cudaError_t launch_fold(const Geometry& g, const Near& nr, const KParams& kp,
                        const double* wnear, void* weff, int match32, cudaStream_t st,
                        int64_t k0 = 0, int64_t k1 = -1);
cudaError_t launch_to_f32(const double* in, float* out, int64_t n, cudaStream_t st);
// Caller strengths (charge, dipole strength per source; complex interleaved
// when kind == 1) -> far-kernel layout in the far precision, times 1/(4 pi).
// sdest (optional): source s is stored at position sdest[s].
cudaError_t launch_pack_strengths(int kind, int precision, int64_t ns, const double* charge,
                                  const double* dipstr, void* str, cudaStream_t st,
                                  const int32_t* sdest = nullptr);
// pot[i] = sum_c partial[c][i] (complex when kind == 1).
cudaError_t launch_reduce_partials(int kind, const double* partial, int nchunks, int64_t ntarg,
                                   double* pot, cudaStream_t st);

// Number of source chunks the far kernel splits the sources into (the
// partial-potential scratch holds nchunks*ntarg*nd values).
int far_nchunks(int64_t ntarg, int64_t nptso, int kind, int precision, int nd, int num_sms);
// Far-kernel block shapes ("variants"): targets per block of a variant (512
// for every f32 variant), resident blocks per SM, and the number of source
// chunks that fills `waves` waves of resident blocks.
// md = 1 selects the multi-density kernel's shapes (nd > 1).
int far_variants();
// Tensor-core far field (variants 3 and 4 of the multi-density FP32
// Helmholtz path): densities per CTA, 0 where the variant does not apply.
int far_tc_group(int variant, int nd, int precision, int kind);
int far_tc_targets();  // targets per CTA
// Launches it, or with occ != null reports its resident CTAs per SM.
cudaError_t far_tc(int variant, const Geometry& g, const KParams& kp, const MatvecArgs& a,
                   cudaStream_t st, int* occ);
int far_block_targets(int precision, int variant, int md = 0, int nd = 1);
int far_md_group(int variant, int nd);
int far_blocks_per_sm(const KParams& kp, int precision, int variant, int md = 0, int nd = 1);
int far_chunks_for_waves(int64_t ntarg, int64_t nptso, int precision, int variant, int nd,
                         int num_sms, int blocks_per_sm, double waves, int md = 0);
// Multi-density far field: a.strengths holds sigma_over[s][nd] (far
// precision, from launch_oversample) and a.ab the per-source constants
// (from launch_source_consts).
cudaError_t launch_far_md(const Geometry& g, const KParams& kp, const MatvecArgs& a,
                          cudaStream_t st);
cudaError_t launch_oversample(const Geometry& g, const KParams& kp, const MatvecArgs& a,
                              cudaStream_t st);
// The same oversampled densities by the tensor cores (3xTF32 products, FP32
// accumulator; oversample_tc.cu): complex densities, FP32 path, nd a
// multiple of 8 up to 128, at most 128 far nodes and 64 nodes per patch
// (oversample_tc_fits); cudaErrorNotSupported otherwise.  a.tc_err receives
// a completion-wait timeout.
bool oversample_tc_fits(const Geometry& g, const KParams& kp, int precision, int nd);
cudaError_t launch_oversample_tc(const Geometry& g, const KParams& kp, const MatvecArgs& a,
                                 cudaStream_t st);
// Engine of the several-density oversampling in the plans' matvecs: 0 CUDA
// cores (default), 1 tensor cores where oversample_tc_fits (BIE_OVERSAMPLE_ENGINE).
int oversample_engine();
void set_oversample_engine(int engine);
// sdest (optional): source s is stored at position sdest[s].
cudaError_t launch_source_consts(const Geometry& g, const KParams& kp, int precision, void* ab,
                                 cudaStream_t st, const int32_t* sdest = nullptr);

// ---- GMRES helpers --------------------------------------------------------
// Vectors hold npts nodes x nd densities (point-major).  The nodes form
// nseg segments (the surfaces of a batch; one for a single plan); system
// sys = segment * nd + density is one independent linear system.  Reductions
// run over chunks: contiguous node ranges that lie inside one segment.
struct Segs {
  int nseg = 1;                         // segments
  int nchunk = 1;                       // reduction chunks
  const int64_t* chunk_lo = nullptr;    // device, nchunk: first node of each chunk
  const int64_t* chunk_hi = nullptr;    // device, nchunk: one past its last node
  const int32_t* seg_chunk0 = nullptr;  // device, nseg+1: first chunk of each segment
  const int32_t* node_seg = nullptr;    // device, npts: segment of each node (null if nseg == 1)
};
// out[2*(k*nsys + sys)] + i out[2*(k*nsys + sys)+1] = sum over sys's nodes of
// wts * conj(V_k) w, for k < m, V_k = V + k*ldv; partial needs
// 2*m*nd*nchunk doubles.
cudaError_t launch_mdot(const double* V, int64_t ldv, int m, const double* w, const double* wts,
                        int nd, int cplx, const Segs& sg, double* partial, double* out,
                        cudaStream_t st);
// w[e] -= sum_k h[k, sys(e)] V_k[e]   (h complex on device, layout as out)
cudaError_t launch_maxpy(const double* V, int64_t ldv, int m, const double* h, double* w,
                         int64_t n, int nd, int cplx, const Segs& sg, cudaStream_t st);
// y[e] = s[sys(e)] x[e], s complex on device (y may alias x)
cudaError_t launch_dscale(const double* x, double* y, const double* s, int64_t n, int nd,
                          int cplx, const Segs& sg, cudaStream_t st);
// y = a x + b y with scalar complex a = (ar, ai), b = (br, bi)
cudaError_t launch_axpby(const double* x, double* y, double ar, double ai, double br, double bi,
                         int64_t n, int cplx, cudaStream_t st);
// y[e] = a[sys(e)] x[e] + b y[e], a complex per system on device
cudaError_t launch_axpbys(const double* x, double* y, const double* a, double br, double bi,
                          int64_t n, int nd, int cplx, const Segs& sg, cudaStream_t st);
// GMRES least squares on the device, FP64, one thread per system: the
// Givens step of iteration it (Hessenberg column from the two Gram-Schmidt
// passes h1, h2 and the new vector's squared norm nrm, rotations, residual
// estimate, stopping test, scale = 1/||w|| for the systems that go on), and
// the back-substitution into the combination coefficients.  H (M+1) x M per
// system, column-major; cs, sn M, sv M+1 per system; all complex (re, im).
cudaError_t launch_gmres_givens(int it, int M, int nsys, const double* h1, const double* h2,
                                const double* nrm, const double* zid, double* H, double* cs,
                                double* sn, double* sv, const double* bnorm, const double* eps,
                                int64_t* done, int* brk, double* errs, double* scale,
                                cudaStream_t st);
cudaError_t launch_gmres_backsolve(int M, int nsys, int mused, const double* H, const double* sv,
                                   const int64_t* done, double* coef, cudaStream_t st);
// Krylov-basis coefficients (mcols per system) of each system's GMRES
// residual vector r0 - A V y.
cudaError_t launch_gmres_resvec(int M, int nsys, int mcols, const double* cs, const double* sn,
                                const double* sv, const int64_t* done, double* z,
                                cudaStream_t st);
// kx += r - rn - zid[sys] d
cudaError_t launch_kx_update(double* kx, const double* r, const double* rn, const double* d,
                             const double* zid, int64_t n, int nd, int cplx, const Segs& sg,
                             cudaStream_t st);
// y[e] = sum_k c[k, sys(e)] V_k[e]
cudaError_t launch_combo(const double* V, int64_t ldv, int m, const double* c, double* y,
                         int64_t n, int nd, int cplx, const Segs& sg, cudaStream_t st);

// ---- batched matvec: the surfaces of a batch in one launch per stage -------
// One surface as the batched kernels see it.  Vector slices of the surface
// start at node vofs (input and output: the targets are the nodes), its
// oversampled sources at sofs in the batch strength array, its far partial
// sums at pofs[precision] (doubles) with nchunks[precision] chunks of
// chunk_len[precision] sources.
struct BatchSurf {
  Geometry g;
  Near nr;
  KParams kp;
  const void* weff[2] = {nullptr, nullptr};  // W_eff: double* (f64), float* (f32)
  const void* ab[2] = {nullptr, nullptr};    // per-source (a, b) per precision
  int64_t vofs = 0, sofs = 0;
  int64_t pofs[2] = {0, 0};
  int64_t chunk_len[2] = {0, 0};
  int nchunks[2] = {0, 0};
  // device flag: 0 while every system of the surface has converged; its
  // strengths and far-field items are then skipped and its output rows zeroed
  const int* live = nullptr;
};

struct BatchArgs {
  int kind = 0, precision = 0, nd = 1, variant = 0;
  bool ck = false;                         // some surface has a complex wavenumber
  const BatchSurf* surfs = nullptr;        // device table
  const int2* patch_items = nullptr;       // (surface, patch)
  const int4* far_items = nullptr;         // (surface, target block, source chunk, density group)
  const int2* row_items = nullptr;         // (surface, group of 8 target rows)
  int npatch_items = 0, nfar_items = 0, nrow_items = 0;
  const double* const* xref = nullptr;     // device slot holding the input vector pointer
  double* const* yref = nullptr;           // device slot holding the output vector pointer
  void* str = nullptr;                     // strengths (nd == 1) or oversampled densities
  double* partial = nullptr;
  int grid_patch = 1, grid_far = 1, grid_row = 1;  // persistent grid sizes
  int max_np = 0;
  int* far_counter = nullptr;              // device work counter of the far-field launch
};
// Strengths/oversampling, far field and combine of every surface: three
// persistent launches, each walking its work list.  Reads the vector
// pointers from xref/yref when it runs (so the launches can be captured in
// a CUDA graph once and replayed for any vectors).
cudaError_t launch_batch_matvec(const BatchArgs& a, cudaStream_t st);
// Far-kernel shape used by the batch: targets per block and densities per
// block group for (precision, variant, nd); blocks per SM of the kernel.
void batch_far_shape(int precision, int variant, int nd, int* targets_per_block, int* group);
int batch_far_blocks_per_sm(int kind, int precision, int variant, int nd, bool ck);
int batch_far_variants(int precision, int nd);

// Number of kernels this library has launched in the process.
int64_t launch_count();
// Adds n launches made by kernels defined outside kernels.cu to that count.
void note_launches(int64_t n);
// FFMA throughput probe (flops = blocks*threads*iters*16*8*2).
cudaError_t launch_ffma_peak(float* out, int blocks, int threads, int iters, cudaStream_t st);
// MUFU throughput probe (ops = blocks*threads*iters*16*8 reciprocal square roots).
cudaError_t launch_mufu_peak(float* out, int blocks, int threads, int iters, cudaStream_t st);

}  // namespace dev
}  // namespace bie
