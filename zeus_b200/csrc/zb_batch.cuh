// Persistent batched BFGS: one launch runs every class of a batch.
//
// A class is one (objective, dimension) with its own runs, starts, outputs
// and stop-early control; classes may have per-instance data (e.g. one toy
// spectrum per 256 runs).  One block (512 or 384 threads) per SM:
//
//   phase A  first the row-layout classes (D = 32, 64, 128: H rows in
//            registers): the block splits into groups of warps (six 2-warp
//            groups for D = 32 and three 4-warp groups for D = 64 at 384
//            threads, the whole block for D = 128), each group taking runs
//            from the class queue on its own; then the block takes runs of
//            the CTA-layout classes (D > 32, H in shared memory) one at a
//            time, smallest dimension first;
//   phase B  each warp, independently, walks the tile- and thread-layout
//            classes: its tiles (or single threads) pop runs from the class
//            queue as their previous run ends, so a slot is refilled the
//            moment its run converges, stalls or fails.  A warp syncs only
//            when it moves on to the next class (its tile width may change).
//
// Most blocks run phase A, then B.  When a batch has both kinds of class,
// one block in 16 runs B first, then A: the tile/thread classes' bulk is
// small, and their few runs that iterate to MAX_ITER then overlap the CTA
// classes instead of starting after them.
//
// The per-run bodies are the standalone layouts' (tile_run, cta_run,
// thread_run), so results equal the standalone kernels' run for run.
#pragma once

#include "zb_bfgs_coop.cuh"
#include "zb_internal.h"
#include "zb_objectives.cuh"

namespace zb {

  // The kernel is built for two block sizes (one block per SM).
  inline constexpr int kBatchBlockLarge = 512;
  inline constexpr int kBatchBlockSmall = 384;

  struct BatchClass {
    int kind, dim, layout, tile;
    int64_t n;
    const double* starts;
    RunOut out;
    Control* ctl;
    const double* data;
    const int* idata;
    int ndata;
    int flags;
    const double* nll_bins;
    int64_t runs_per_instance; // 0: one instance shared by all runs
    unsigned long long* queue;
    int required;
  };

  inline constexpr int kMaxBatchClasses = 16;

  // The whole batch description travels as the kernel's parameter block
  // (about 2.6 KB): no host-to-device copy, capturable in a CUDA graph.
  struct BatchTable {
    int ncls;
    int max_iter;
    double tol;
    int flags;
    int early_b; // blocks that drain the tile/thread classes before the CTA ones
    BatchClass c[kMaxBatchClasses];
  };

  // Tile widths compiled into the batch kernel for an objective and
  // dimension: at most two rows of H and 32 doubles of it per lane (the
  // kernel is limited to 128 registers per thread by its 512-thread,
  // one-block-per-SM launch bounds); at most 4*D lanes (the lanes beyond D
  // evaluate line-search trials in parallel) except for the objectives whose
  // cooperative evaluation splits bins or matrix rows.
  __host__ __device__ constexpr unsigned
  batch_widths(int kind, int d)
  {
    unsigned m = 0;
    if (d > 32)
      return 0;
    const bool wide = kind == ZEUS_OBJ_POISSON_NLL || kind == ZEUS_OBJ_GAUSSIAN;
    for (int k = 1; k <= 5; ++k) {
      const int ts = 1 << k;
      const int r = (d + ts - 1) / ts;
      if (r <= 2 && r * d <= 32 && (wide || ts <= 4 * d))
        m |= 1u << k;
    }
    return m;
  }
  inline constexpr int kBatchThreadMaxDim = 4;
  inline constexpr int kBatchCtaMinDim = 33;
  // the row layout in a batch (zb_bfgs_rows.cuh): dimensions 32 and up
  inline constexpr int kBatchRowMinDim = 32;

  // Objective with instance `inst`'s data: instances are stored one after
  // another (Gaussian: D*D doubles; NLL: ndata centres / counts, 4*ndata
  // bin constants).
  template <class F>
  __device__ __forceinline__ F
  with_instance(F f, const BatchClass& c, int64_t inst)
  {
    if constexpr (requires { f.C; }) {
      f.C += inst * (int64_t)c.dim * c.dim;
    } else if constexpr (requires { f.bins; }) {
      f.centres += inst * c.ndata;
      f.counts += inst * c.ndata;
      f.bins += inst * 4 * (int64_t)c.ndata;
    }
    return f;
  }

  int launch_batch_512(const BatchTable& bt, size_t smem, cudaStream_t st);
  int launch_batch_384(const BatchTable& bt, size_t smem, cudaStream_t st);

  __host__ __device__ inline size_t
  batch_tile_buf_doubles(int dim, int ts)
  {
    return (size_t)(32 / ts) * tile_buf_doubles(dim, ts);
  }

} // namespace zb
