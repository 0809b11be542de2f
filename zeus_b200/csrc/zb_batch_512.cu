// The persistent batch kernel with 512-thread blocks.
#include "zb_batch_kernel.cuh"

namespace zb {

  int
  launch_batch_512(const BatchTable& bt, size_t smem, cudaStream_t st)
  {
    // the warp-sized bodies inlined where no row or CTA class is present
    for (int i = 0; i < bt.ncls; ++i)
      if (bt.c[i].layout == ZEUS_LAYOUT_CTA || bt.c[i].layout == ZEUS_LAYOUT_ROWS)
        return launch_batch_kernel<512, false>(bt, smem, st);
    return launch_batch_kernel<512, true>(bt, smem, st);
  }

} // namespace zb
