// The persistent batch kernel, a template on its block size; each of
// zb_batch_512.cu and zb_batch_384.cu instantiates one and exports its
// launcher (the host side, zb_batch.cu, picks one per batch).
#pragma once

#include "zb_batch.cuh"
#include "zb_bfgs_rows.cuh"
#include "zb_objective_visit.cuh"

namespace zb {

  namespace {

    // Device-side (kind, dim) -> functor, for the dimensions the library is
    // built for (the same sets as visit_objective).
    template <class Fn>
    __device__ __forceinline__ void
    batch_visit(const BatchClass& c, Fn&& fn)
    {
      switch (c.kind) {
        case ZEUS_OBJ_ROSENBROCK:
          switch (c.dim) {
#define ZB_CASE(D)                                                             \
  case D:                                                                      \
    fn(zeus::Rosenbrock<D>{});                                                 \
    return;
            ZB_ROSENBROCK_DIMS(ZB_CASE)
#undef ZB_CASE
          }
          return;
        case ZEUS_OBJ_RASTRIGIN:
          switch (c.dim) {
#define ZB_CASE(D)                                                             \
  case D:                                                                      \
    fn(zeus::Rastrigin<D>{});                                                  \
    return;
            ZB_RASTRIGIN_DIMS(ZB_CASE)
#undef ZB_CASE
          }
          return;
        case ZEUS_OBJ_ACKLEY:
          switch (c.dim) {
#define ZB_CASE(D)                                                             \
  case D:                                                                      \
    fn(zeus::Ackley<D>{});                                                     \
    return;
            ZB_ACKLEY_DIMS(ZB_CASE)
#undef ZB_CASE
          }
          return;
        case ZEUS_OBJ_GAUSSIAN:
          switch (c.dim) {
#define ZB_CASE(D)                                                             \
  case D: {                                                                    \
    zeus::Gaussian<D> g;                                                       \
    g.C = c.data;                                                              \
    g.symmetric = (c.flags & 1) != 0;                                          \
    fn(g);                                                                     \
    return;                                                                    \
  }
            ZB_GAUSSIAN_DIMS(ZB_CASE)
#undef ZB_CASE
          }
          return;
        case ZEUS_OBJ_POISSON_NLL:
          if (c.dim == 4) {
            zeus::PoissonNLL p;
            p.centres = c.data;
            p.counts = c.idata;
            p.bins = c.nll_bins;
            p.nbins = c.ndata;
            fn(p);
          }
          return;
      }
    }

    // The CTA, tile and thread bodies are called, not inlined, in a batch
    // with row or CTA classes: each is then compiled as a function of its
    // own, with its own register assignment and scheduling, instead of
    // sharing them with every other layout's body in the one kernel
    // (measured: a 64-D row-layout run 1.94 us an iteration inlined beside
    // the tile, thread and CTA bodies, 1.49 us alone).  The row bodies stay
    // inline in that kernel (the mixed batch 20.71 -> 20.37 ms, the 128-D
    // iteration 3.18 -> 3.10 us); the kernel for batches without row or CTA
    // classes never runs them and keeps them out of line (inlined there
    // they cost the multimodal batch 8%).
    template <class F, int D, int NW, int KS>
    __device__ __noinline__ void
    batch_row_call(const F f, double* gsm, int bar, int base, const BfgsParams prm,
                   const double* x0, int64_t run, const RunOut out, Control* ctl)
    {
      row_run<F, D, NW, true, false, KS>(f, gsm, bar, base, prm, x0, run, out, ctl);
    }

    template <bool kInline, class F, int D, int NW, int KS>
    __device__ __forceinline__ void
    batch_row_run(const F& f, double* gsm, int bar, int base, const BfgsParams& prm,
                  const double* x0, int64_t run, const RunOut& out, Control* ctl)
    {
      if constexpr (kInline)
        batch_row_call<F, D, NW, KS>(f, gsm, bar, base, prm, x0, run, out, ctl);
      else
        row_run<F, D, NW, true, false, KS>(f, gsm, bar, base, prm, x0, run, out, ctl);
    }

    template <class F, int D, int kBlock>
    __device__ __noinline__ void
    batch_cta_run(const F f, double* sm, const BfgsParams prm, const double* x0,
                  int64_t run, const RunOut out, Control* ctl)
    {
      cta_run<F, D, true, kBlock>(f, sm, prm, x0, run, out, ctl);
    }

    // The tile and thread bodies come in both forms: a batch with row or
    // CTA classes calls them (the register assignment of the row bodies
    // then does not suffer from theirs), a batch of tile/thread classes
    // alone inlines them (measured: the multimodal batch 26.1 -> 23.4 ms,
    // the dijet batch 449 -> 360 ms inlined; the mixed batch 20.3 -> 21.9 ms).
    template <class F, int D, int TS>
    __device__ __noinline__ void
    batch_tile_call(const F f, double* buf, const BfgsParams prm, const double* x0,
                    int64_t run, const RunOut out, Control* ctl)
    {
      tile_run<F, D, TS, true>(f, cg::tiled_partition<TS>(cg::this_thread_block()), buf,
                               prm, x0, run, out, ctl);
    }

    template <class F, int D>
    __device__ __noinline__ void
    batch_thread_call(const F f, const BfgsParams prm, const double* x0, int64_t run,
                      const RunOut out, Control* ctl)
    {
      thread_run<F, D, true>(f, prm, x0, run, out, ctl);
    }

    template <bool kInline, class F, int D, int TS>
    __device__ __forceinline__ void
    batch_tile_run(const F& f, double* buf, const BfgsParams& prm, const double* x0,
                   int64_t run, const RunOut& out, Control* ctl)
    {
      if constexpr (kInline)
        tile_run<F, D, TS, true>(f, cg::tiled_partition<TS>(cg::this_thread_block()),
                                 buf, prm, x0, run, out, ctl);
      else
        batch_tile_call<F, D, TS>(f, buf, prm, x0, run, out, ctl);
    }

    template <bool kInline, class F, int D>
    __device__ __forceinline__ void
    batch_thread_run(const F& f, const BfgsParams& prm, const double* x0, int64_t run,
                     const RunOut& out, Control* ctl)
    {
      if constexpr (kInline)
        thread_run<F, D, true>(f, prm, x0, run, out, ctl);
      else
        batch_thread_call<F, D>(f, prm, x0, run, out, ctl);
    }

    template <class F>
    __device__ __forceinline__ F
    instance_for(const F& f, const BatchClass& c, int64_t run)
    {
      return c.runs_per_instance > 0 ? with_instance(f, c, run / c.runs_per_instance)
                                     : f;
    }

    template <bool kInline, class F, int D, int TS>
    __device__ __forceinline__ void
    drain_tile_class(const F& f, const BatchClass& c, const BfgsParams& prm,
                     double* warp_buf)
    {
      auto tile = cg::tiled_partition<TS>(cg::this_thread_block());
      const int tin = (int)(threadIdx.x & 31) / TS;
      double* buf = warp_buf + tin * tile_buf_doubles(D, TS);
      for (;;) {
        unsigned long long r = 0;
        if (tile.thread_rank() == 0)
          r = atomicAdd(c.queue, 1ull);
        r = tile.shfl(r, 0);
        if ((int64_t)r >= c.n)
          break;
        batch_tile_run<kInline, F, D, TS>(instance_for(f, c, (int64_t)r), buf, prm,
                                 c.starts + (int64_t)r * D, (int64_t)r, c.out, c.ctl);
      }
    }

  } // namespace

  template <int kBlock, bool kInline>
  __global__ void __launch_bounds__(kBlock, 1)
    bfgs_batch_kernel(const __grid_constant__ BatchTable bt)
  {
    const int ncls = bt.ncls;
    const BatchClass* classes = bt.c;
    extern __shared__ __align__(16) double sm[];
    __shared__ unsigned long long sh_run;

    // Blocks below early_b take the tile/thread classes (phase B) before
    // the CTA ones (phase A): the former's bulk is small, and their few runs
    // that iterate to MAX_ITER then overlap the CTA classes instead of
    // starting after them.  The other blocks run A, then B, and find the
    // tile/thread queues drained or nearly so.
    const bool early = (int)blockIdx.x < bt.early_b;
    for (int pass = 0; pass < 2; ++pass) {
      if ((pass == 0) != early) {
        // phase A, row-layout classes: the block splits into groups of NW
        // warps, each taking runs from the class queue on its own.  (Split
        // groups, two 128-D runs a block with part of H in shared memory,
        // measured slower here than in their own kernel -- 19.9 against 15.8
        // ms for the 128-D class: the body spills under the batch kernel's
        // register budget, and with 222 KB of shared memory in use the spills
        // miss L1.  The batch keeps one 12-warp group for D = 128.)
        for (int ci = 0; ci < ncls; ++ci) {
          const BatchClass& c = classes[ci];
          if (c.layout != ZEUS_LAYOUT_ROWS)
            continue;
          const BfgsParams prm{c.n, bt.max_iter, c.required, bt.tol, bt.flags};
          batch_visit(c, [&](auto f) {
            using F = decltype(f);
            constexpr int D = (int)F::arity;
            constexpr int NW = row_warps(D, kBlock);
            constexpr int KS = 0;
            if constexpr (NW > 0 && D >= kBatchRowMinDim && RowLayoutObjective<F>) {
              constexpr int NT = 32 * NW;
              // the host sizes shared memory for this shape: a launch given
              // less (a host/device mismatch) runs none of the class's runs
              // rather than reach past the end of shared memory
              unsigned dyn;
              asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
              if ((size_t)(kBlock / NT) * row_smem_doubles<D, NW, KS>() * sizeof(double) > dyn)
                return;
              const int gi = (int)threadIdx.x / NT;
              double* gsm = sm + (size_t)gi * row_smem_doubles<D, NW, KS>();
              long long* slot =
                reinterpret_cast<long long*>(gsm + row_smem_doubles<D, NW, KS>() - 2);
              for (;;) {
                if ((int)threadIdx.x % NT == 0)
                  *slot = (long long)atomicAdd(c.queue, 1ull);
                asm volatile("bar.sync %0, %1;" ::"r"(1 + gi), "n"(NT) : "memory");
                const int64_t r = *slot;
                asm volatile("bar.sync %0, %1;" ::"r"(1 + gi), "n"(NT) : "memory");
                if (r >= c.n)
                  break;
                batch_row_run<kInline, F, D, NW, KS>(instance_for(f, c, r), gsm, 1 + gi,
                                                     gi * NT, prm, c.starts + r * D, r,
                                                     c.out, c.ctl);
              }
            }
          });
          __syncthreads();
        }
        // phase A, CTA-layout classes, one run per block at a time
        for (int ci = 0; ci < ncls; ++ci) {
          const BatchClass& c = classes[ci];
          if (c.layout != ZEUS_LAYOUT_CTA)
            continue;
          const BfgsParams prm{c.n, bt.max_iter, c.required, bt.tol, bt.flags};
          for (;;) {
            if (threadIdx.x == 0)
              sh_run = atomicAdd(c.queue, 1ull);
            __syncthreads();
            const int64_t r = (int64_t)sh_run;
            __syncthreads();
            if (r >= c.n)
              break;
            batch_visit(c, [&](auto f) {
              using F = decltype(f);
              constexpr int D = (int)F::arity;
              if constexpr (D >= kBatchCtaMinDim && !cta_h_global(D, kBlock) &&
                            sizeof(double) * cta_smem_doubles<F, D, true>(kBlock) <=
                              227 * 1024)
                batch_cta_run<F, D, kBlock>(instance_for(f, c, r), sm, prm,
                                            c.starts + r * D, r, c.out, c.ctl);
            });
          }
        }
        __syncthreads();
        continue;
      }
      // phase B: each warp drains the tile / thread classes; per-warp
      // buffers follow each other, sized by the host for the widest class
      size_t stride = 0;
      for (int ci = 0; ci < ncls; ++ci)
        if (classes[ci].layout == ZEUS_LAYOUT_TILE)
          stride = stride > batch_tile_buf_doubles(classes[ci].dim, classes[ci].tile)
                     ? stride
                     : batch_tile_buf_doubles(classes[ci].dim, classes[ci].tile);
      double* warp_buf = sm + (size_t)(threadIdx.x >> 5) * stride;
      for (int ci = 0; ci < ncls; ++ci) {
        const BatchClass& c = classes[ci];
        if (c.layout == ZEUS_LAYOUT_CTA || c.layout == ZEUS_LAYOUT_ROWS)
          continue;
        const BfgsParams prm{c.n, bt.max_iter, c.required, bt.tol, bt.flags};
        batch_visit(c, [&](auto f) {
          using F = decltype(f);
          constexpr int D = (int)F::arity;
          if (c.layout == ZEUS_LAYOUT_THREAD) {
            if constexpr (D <= kBatchThreadMaxDim) {
              for (;;) {
                const int64_t r = (int64_t)atomicAdd(c.queue, 1ull);
                if (r >= c.n)
                  break;
                batch_thread_run<kInline, F, D>(instance_for(f, c, r), prm,
                                                c.starts + r * D, r, c.out, c.ctl);
              }
            }
          } else if constexpr (D < kBatchCtaMinDim) {
            constexpr unsigned W = batch_widths(F::kind, D);
            switch (c.tile) {
#define ZB_TS(K)                                                               \
  case (1 << K):                                                               \
    if constexpr ((W >> K) & 1u)                                               \
      drain_tile_class<kInline, F, D, (1 << K)>(f, c, prm, warp_buf);                   \
    break;
              ZB_TS(1)
              ZB_TS(2)
              ZB_TS(3)
              ZB_TS(4)
              ZB_TS(5)
#undef ZB_TS
            }
          }
        });
        __syncwarp();
      }
      __syncthreads(); // the warp buffers are free again
    }
  }


  // Sets the shared-memory attribute, sizes the grid to the SMs and launches.
  template <int kBlock, bool kInline>
  int
  launch_batch_kernel(const BatchTable& bt, size_t smem, cudaStream_t st)
  {
    auto kern = bfgs_batch_kernel<kBlock, kInline>;
    int rc = cuda_fail(cudaFuncSetAttribute(
                         kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                       "batch shared memory attribute");
    if (rc)
      return rc;
    int per_sm = 0;
    rc = cuda_fail(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, smem),
      "batch occupancy");
    if (rc)
      return rc;
    if (per_sm < 1) {
      set_error("batch kernel does not fit on an SM (%zu bytes of shared memory)",
                smem);
      return ZEUS_E_UNSUPPORTED;
    }
    kern<<<sm_count() * per_sm, kBlock, smem, st>>>(bt);
    return cuda_fail(cudaGetLastError(), "batch BFGS launch");
  }

} // namespace zb
