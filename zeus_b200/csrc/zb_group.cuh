// Cooperative groups the BFGS layouts run one optimisation on:
//   TileGroup<TS>: TS lanes of one warp (TS = 2..32), reductions by xor
//                  butterflies, barriers __syncwarp(tile mask);
//   CtaGroup:      the whole thread block, reductions through shared memory.
// Both give the same interface (rank, size, sync, sum, bcast) so objective
// code is written once for either.  sum() returns identical bits in every
// member: butterfly partners add the same two values (addition commutes),
// and a value summed by one lane reaches the others by shuffles or shared
// memory, never re-added.
#pragma once

#include <cooperative_groups.h>

namespace zb {

  namespace cg = cooperative_groups;

  // Reduce-scatter of K values over the NL lanes of a warp or tile (NL a
  // power of two >= P, P = K rounded up to a power of two): at each of the
  // first log2 P xor levels a lane keeps half of its values and adds the
  // partner's copy of that half, so the level moves half as many values as
  // a plain butterfly of all K; the remaining levels add one value.  On
  // return lane l holds in v[0] the sum of value rs_index(l) over all NL
  // lanes.  `shx(x, m)` is the xor shuffle of the group.
  template <int K>
  struct ReduceScatter {
    static constexpr int P = K <= 1 ? 1 : K <= 2 ? 2 : K <= 4 ? 4 : 8;
    static_assert(K <= 8, "at most 8 values");

    template <int NL>
    __device__ static __forceinline__ int
    index(int lane)
    {
      int idx = 0;
#pragma unroll
      for (int h = P / 2, m = NL / 2; h > 0; h >>= 1, m >>= 1)
        if (lane & m)
          idx += h;
      return idx;
    }
    // the lowest lane holding value k
    template <int NL>
    __device__ static __forceinline__ int
    owner(int k)
    {
      int lane = 0;
#pragma unroll
      for (int h = P / 2, m = NL / 2; h > 0; h >>= 1, m >>= 1)
        if (k & h)
          lane += m;
      return lane;
    }
    template <int NL, class Shx>
    __device__ static __forceinline__ double
    run(const double (&in)[K], int lane, Shx shx)
    {
      static_assert(NL >= P, "group narrower than the value count");
      double v[P];
#pragma unroll
      for (int k = 0; k < P; ++k)
        v[k] = k < K ? in[k] : 0.0;
      int m = NL / 2;
#pragma unroll
      for (int h = P / 2; h > 0; h >>= 1, m >>= 1) {
        const bool up = (lane & m) != 0;
#pragma unroll
        for (int j = 0; j < h; ++j) {
          const double send = up ? v[j] : v[j + h];
          const double keep = up ? v[j + h] : v[j];
          v[j] = keep + shx(send, m);
        }
      }
#pragma unroll
      for (; m > 0; m >>= 1)
        v[0] += shx(v[0], m);
      return v[0];
    }
  };

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
      using RS = ReduceScatter<K>;
      if constexpr (K >= 3 && TS >= RS::P) {
        // reduce-scatter, then every lane fetches each total from its owner
        const int lane = (int)t.thread_rank();
        const double mine = RS::template run<TS>(
          v, lane, [&](double x, int m) { return t.shfl_xor(x, m); });
#pragma unroll
        for (int k = 0; k < K; ++k)
          v[k] = t.shfl(mine, RS::template owner<TS>(k));
      } else {
#pragma unroll
        for (int m = TS / 2; m > 0; m >>= 1)
#pragma unroll
          for (int k = 0; k < K; ++k)
            v[k] += t.shfl_xor(v[k], m);
      }
    }
    template <class T>
    __device__ __forceinline__ T
    bcast(T v, int src) const
    {
      return t.shfl(v, src);
    }
  };

  // `red` points at kCtaRedDoubles doubles of shared memory reserved for the
  // group's reductions: two buffers of 8 values x 32 warps used in turn
  // (every thread runs the same sequence of sums, so a buffer is rewritten
  // only two sums later, after the barriers of the sum in between, when
  // every thread has finished with it), 8 totals and one slot for bcast().
  // A sum: each warp reduce-scatters its values and writes its partials;
  // barrier; warp 0 reduce-scatters the per-warp partials and writes the
  // totals; barrier; every thread reads the totals.  (Redundant per-warp
  // second stages cost more in shuffle throughput than the second barrier.)
  // The block size must be a multiple of 32.
  inline constexpr int kCtaRedDoubles = 2 * 32 * 8 + 8 + 8;

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
      using RS = ReduceScatter<K>;
      const auto shx = [](double x, int m) {
        return __shfl_xor_sync(0xffffffffu, x, m);
      };
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
      const int nw = (blockDim.x + 31) >> 5;
      double* buf = red + parity * (32 * 8);
      double* tot = red + 2 * 32 * 8;
      parity ^= 1;
      const int idx = RS::template index<32>(lane);
      const bool owner = (lane & (32 / RS::P - 1)) == 0 && idx < K;
      const double mine = RS::template run<32>(v, lane, shx);
      if (owner)
        buf[idx * 32 + warp] = mine;
      __syncthreads();
      if (warp == 0) {
        double w[K];
#pragma unroll
        for (int k = 0; k < K; ++k)
          w[k] = lane < nw ? buf[k * 32 + lane] : 0.0;
        const double t = RS::template run<32>(w, lane, shx);
        if (owner)
          tot[idx] = t;
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < K; ++k)
        v[k] = tot[k];
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
      double* slot = red + 2 * 32 * 8 + 8;
      if ((int)threadIdx.x == src)
        slot[0] = v;
      __syncthreads();
      const double r = slot[0];
      __syncthreads();
      return r;
    }
  };

  // A group of NT threads (NT a multiple of 32, starting at a warp
  // boundary `base`) inside a larger block, synchronised by the named
  // barrier `bar` (1..15; 0 is __syncthreads), so that several groups of a
  // block run independent optimisations.  Same interface as CtaGroup;
  // `red` holds row_red_doubles(NT / 32) doubles of shared memory.  A sum
  // takes one barrier: each warp reduce-scatters its values and writes its
  // partials (two buffers used in turn, as in CtaGroup), and after the
  // barrier every lane adds up its value's partials itself, in warp order.
  __host__ __device__ constexpr int
  row_red_doubles(int nw)
  {
    return 2 * 8 * nw + 8 + 8;
  }

  template <int NT>
  struct RowGroup {
    static_assert(NT % 32 == 0 && NT <= 1024, "a whole number of warps");
    static constexpr int NW = NT / 32;
    int base;
    int bar;
    double* red;
    double* scratch;
    mutable int parity = 0;

    __device__ __forceinline__ int
    rank() const
    {
      return (int)threadIdx.x - base;
    }
    static constexpr int
    size()
    {
      return NT;
    }
    __device__ __forceinline__ void
    sync() const
    {
      if constexpr (NT == 32)
        __syncwarp();
      else
        asm volatile("bar.sync %0, %1;" ::"r"(bar), "n"(NT) : "memory");
    }
    // AW: only warps below AW hold non-zero values (the others' partials
    // are neither written nor read)
    template <int K, int AW = NW>
    __device__ __forceinline__ void
    sum(double (&v)[K]) const
    {
      using RS = ReduceScatter<K>;
      static_assert(AW >= 1 && AW <= NW, "active warps");
      const auto shx = [](double x, int m) {
        return __shfl_xor_sync(0xffffffffu, x, m);
      };
      const int t = rank(), lane = t & 31, warp = t >> 5;
      double* buf = red + parity * (8 * NW);
      double* tot = red + 2 * 8 * NW;
      parity ^= 1;
      const int idx = RS::template index<32>(lane);
      const bool owner = (lane & (32 / RS::P - 1)) == 0 && idx < K;
      const double mine = RS::template run<32>(v, lane, shx);
      (void)tot;
      if constexpr (NW == 1) {
#pragma unroll
        for (int k = 0; k < K; ++k)
          v[k] = __shfl_sync(0xffffffffu, mine, RS::template owner<32>(k));
        return;
      } else {
        // one barrier: every lane sums its value's per-warp partials in warp
        // order (the same bits in every warp), then the totals go round the
        // warp by shuffles
        if (owner && warp < AW)
          buf[idx * NW + warp] = mine;
        sync();
        double tt = 0.0;
        if (idx < K) {
          const double* b = buf + idx * NW;
          double a0 = b[0], a1 = AW > 1 ? b[1] : 0.0;
#pragma unroll
          for (int w = 2; w + 1 < AW; w += 2) {
            a0 += b[w];
            a1 += b[w + 1];
          }
          if constexpr (AW > 2 && AW % 2 == 1)
            a0 += b[AW - 1];
          tt = a0 + a1;
        }
#pragma unroll
        for (int k = 0; k < K; ++k)
          v[k] = __shfl_sync(0xffffffffu, tt, RS::template owner<32>(k));
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
      double* slot = red + 2 * 8 * NW + 8;
      if (rank() == src)
        slot[0] = v;
      sync();
      const double r = slot[0];
      sync();
      return r;
    }
  };

} // namespace zb
