// Near-field quadrature generator on the device: the same weights as
// getnearquad (host/nearquad.h) -- the integrals of the combined-field
// kernel against the patch basis, mapped to nodal values by umat -- computed
// by one warp per (target, patch) pair.
//
// Rules, tolerances and refinement are those of the host generator: the
// collapsed Gauss rule of 8/10/12 points per direction by patch order,
// 4-way refinement of parameter-space triangles until the children's sum
// agrees with the parent to 0.1 * eps * sqrt(min_j |J_j| w_j) or level 18,
// and for a target on the patch the split at the target into triangles
// integrated with a Duffy and a sinh map (nself = clamp(ceil(2.2 digits)+4,
// 12, 40) points each way).  The two generators agree to within that
// tolerance; they are not bit-identical (refinement decisions at the
// threshold and summation order can differ).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

#include "../host/nearquad.h"
#include "../host/setup.h"

namespace bie {

// Largest patch basis (npols) the device generator takes.
constexpr int kNearQuadMaxNp = 256;

// Inputs are host arrays in the reference layout (1-based index arrays);
// wnear_dev is device memory: nquad reals (kind 0) or nquad interleaved
// complex values (kind 1).  Work runs on `st`; the call returns after the
// stream has finished.  Returns kOk, kErrArg (inconsistent input or a patch
// with more than kNearQuadMaxNp basis functions), kErrCuda, or kErrTimeout
// when a pair hit the refinement-step cap.
int getnearquad_gpu(const Surf& s, int ndt, int64_t nt, const double* targs,
                    const int64_t* ipatch_id, const double* uvs_targ, double eps, int kind,
                    cdouble zk, cdouble alpha, cdouble beta, int64_t nnz, const int64_t* row_ptr,
                    const int64_t* col_ind, const int64_t* iquad, int64_t nquad,
                    double* wnear_dev, cudaStream_t st, NearQuadStats* stats = nullptr);

}  // namespace bie
