// The persistent batch kernel with 384-thread blocks.
#include "zb_batch_kernel.cuh"

namespace zb {

  int
  launch_batch_384(const BatchTable& bt, size_t smem, cudaStream_t st)
  {
    return launch_batch_kernel<384>(bt, smem, st);
  }

} // namespace zb
