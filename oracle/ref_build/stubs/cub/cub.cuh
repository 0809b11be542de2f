// Stand-in for <cub/cub.cuh> in the host build of the reference.  Only the
// declaration the reference names (bfgs_common.cuh launchReduction) is given;
// the host oracle never instantiates launchReduction.
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace cub {
  struct DeviceReduce {
    template <class In, class OutV, class OutI>
    static cudaError_t ArgMin(void*, std::size_t&, In, OutV, OutI, int);
  };
}
