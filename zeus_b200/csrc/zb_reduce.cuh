// Final reduction over runs: argmin of fval plus the status census, one
// kernel (the reference runs a CUB ArgMin, copies every Result<D> to the
// host and counts there: bfgs_common.cuh:280-319, util.hpp:151-200).
#pragma once

#include "zb_common.cuh"
#include "zb_pso.cuh"

namespace zb {

  inline constexpr int kMaxKnownDim = 256;

  struct KnownMin {
    int has;                  // 0: the origin
    double x[kMaxKnownDim];
  };

  struct Census {
    int32_t actual, claimed, surrendered, stopped, best_idx, reserved;
  };

  // One block of 1024 threads, grid-stride over the runs.
  __global__ void __launch_bounds__(1024)
    census_kernel(const double* __restrict__ fval,
                  const int32_t* __restrict__ status,
                  const double* __restrict__ x, int64_t n, int dim,
                  KnownMin km, Census* out);

  // NLL per-bin constants {ln x, ln(1-x), k, lgamma(k+1)}.
  __global__ void nll_bins_kernel(const double* __restrict__ centres,
                                  const int* __restrict__ counts, int nbins,
                                  double* __restrict__ bins);

} // namespace zb
