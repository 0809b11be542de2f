// The persistent batch kernel with 512-thread blocks.
#include "zb_batch_kernel.cuh"

namespace zb {

  int
  launch_batch_512(const BatchTable& bt, size_t smem, cudaStream_t st)
  {
    return launch_batch_kernel<512>(bt, smem, st);
  }

} // namespace zb
