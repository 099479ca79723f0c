// Drop-in replacement of compute_half_inverse (nukexc/nukexc_utils.hpp:198-270)
// over nkx_half_inverse: X (N x K) with X X^T the pseudo-inverse of the
// preconditioned metric, keeping singular values > lin_dep_threshold.
#pragma once

#include "nukexc_config.hpp"

namespace Nukexc {

inline DeviceView2DLeft compute_half_inverse(const DeviceView2DLeft &overlap_matrix,
                                             const double lin_dep_threshold = 1e-5) {
  const int N = (int)overlap_matrix.extent(0);
  DeviceView2DLeft full("X (all columns)", N, N);
  int K = 0;
  nkx_shim::check(nkx_half_inverse(N, overlap_matrix.data(), lin_dep_threshold, full.data(), &K, nullptr),
                  "compute_half_inverse");
  DeviceView2DLeft X("X", N, K);
  if (K > 0)
    nkx_shim::check_cuda(cudaMemcpy(X.data(), full.data(), sizeof(double) * N * K, cudaMemcpyDeviceToDevice), "copy");
  return X;
}

}  // namespace Nukexc
