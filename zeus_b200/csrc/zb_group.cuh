// Cooperative groups the BFGS layouts run one optimisation on:
//   TileGroup<TS>: TS lanes of one warp (TS = 2..32), reductions by xor
//                  butterflies, barriers __syncwarp(tile mask);
//   CtaGroup:      the whole thread block, reductions through shared memory.
// Both give the same interface (rank, size, sync, sum, bcast) so objective
// code is written once for either.  sum() returns identical bits in every
// member: butterfly partners add the same two values (addition commutes),
// and the block version has every thread add the per-warp sums in one order.
#pragma once

#include <cooperative_groups.h>

namespace zb {

  namespace cg = cooperative_groups;

  // Every group also carries `scratch`: shared memory of at least size()
  // doubles that objectives may use between two sync()s.
  template <int TS>
  struct TileGroup {
    cg::thread_block_tile<TS> t;
    double* scratch;

    __device__ TileGroup(cg::thread_block_tile<TS> tile, double* scr)
      : t(tile), scratch(scr)
    {}
    __device__ __forceinline__ int
    rank() const
    {
      return (int)t.thread_rank();
    }
    static constexpr int
    size()
    {
      return TS;
    }
    __device__ __forceinline__ void
    sync() const
    {
      t.sync();
    }
    __device__ __forceinline__ double
    sum(double v) const
    {
#pragma unroll
      for (int m = TS / 2; m > 0; m >>= 1)
        v += t.shfl_xor(v, m);
      return v;
    }
    template <int K>
    __device__ __forceinline__ void
    sum(double (&v)[K]) const
    {
#pragma unroll
      for (int m = TS / 2; m > 0; m >>= 1)
#pragma unroll
        for (int k = 0; k < K; ++k)
          v[k] += t.shfl_xor(v[k], m);
    }
    template <class T>
    __device__ __forceinline__ T
    bcast(T v, int src) const
    {
      return t.shfl(v, src);
    }
  };

  // `red` points at kCtaRedDoubles doubles of shared memory reserved for the
  // group's reductions: two buffers of 32 warps x 8 values used in turn --
  // every thread runs the same sequence of sums, so a buffer is rewritten
  // only two sums later, after the barrier of the sum in between, when every
  // thread has finished reading it: one barrier per sum -- plus one slot for
  // bcast().  The block size must be a multiple of 32.
  inline constexpr int kCtaRedDoubles = 2 * 32 * 8 + 8;

  struct CtaGroup {
    double* red;
    double* scratch;
    mutable int parity = 0;

    __device__ __forceinline__ int
    rank() const
    {
      return (int)threadIdx.x;
    }
    __device__ __forceinline__ int
    size() const
    {
      return (int)blockDim.x;
    }
    __device__ __forceinline__ void
    sync() const
    {
      __syncthreads();
    }
    template <int K>
    __device__ __forceinline__ void
    sum(double (&v)[K]) const
    {
      static_assert(K <= 8, "at most 8 simultaneous sums");
#pragma unroll
      for (int m = 16; m > 0; m >>= 1)
#pragma unroll
        for (int k = 0; k < K; ++k)
          v[k] += __shfl_xor_sync(0xffffffffu, v[k], m);
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
      const int nw = (blockDim.x + 31) >> 5;
      double* buf = red + parity * (32 * 8);
      parity ^= 1;
      if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k)
          buf[warp * 8 + k] = v[k];
      __syncthreads();
#pragma unroll
      for (int k = 0; k < K; ++k) {
        double a = 0.0;
        for (int w = 0; w < nw; ++w)
          a += buf[w * 8 + k];
        v[k] = a;
      }
    }
    __device__ __forceinline__ double
    sum(double v) const
    {
      double a[1] = {v};
      sum<1>(a);
      return a[0];
    }
    __device__ __forceinline__ double
    bcast(double v, int src) const
    {
      double* slot = red + 2 * 32 * 8;
      if ((int)threadIdx.x == src)
        slot[0] = v;
      __syncthreads();
      const double r = slot[0];
      __syncthreads();
      return r;
    }
  };

} // namespace zb
