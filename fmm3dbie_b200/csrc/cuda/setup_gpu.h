// The rest of the setup on the device: near lists (findnear), far-field
// oversampling orders (get_far_order) and oversampled geometry
// (oversample_geom), with the host versions' rules (host/setup.h) so the
// results are the same sets, the same orders and the same geometry up to
// rounding.  Inputs and outputs are host arrays in the reference layout;
// work runs on `st` and the calls return after it has finished.
#pragma once
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "../host/setup.h"

namespace bie {

// findnear: {patch j : |t_i - cms_j| <= rads_j} per target, sorted, 1-based.
int findnear_gpu(int64_t npatches, const double* cms, const double* rads, int ndt, int64_t nt,
                 const double* targs, std::vector<int64_t>& row_ptr,
                 std::vector<int64_t>& col_ind, cudaStream_t st);

// get_far_order: nfars (and ixyzso) per patch; probe targets and tolerance
// as far_order (host/setup.h).
int far_order_gpu(double eps, const Surf& s, const double* cms, const double* rads, int ndt,
                  int64_t nt, const double* targs, int ikerorder, cdouble zk, int64_t nnz,
                  const int64_t* row_ptr, const int64_t* col_ind, double rfac, int64_t* nfars,
                  int64_t* ixyzso, cudaStream_t st);

// oversample_geom: srcover(12, nptso).
int oversample_geom_gpu(const Surf& s, const int64_t* nfars, const int64_t* ixyzso,
                        int64_t nptso, double* srcover, cudaStream_t st);

}  // namespace bie
