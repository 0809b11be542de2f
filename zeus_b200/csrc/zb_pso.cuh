// PSO swarm seeding (the reference's pso.cuh:17-155), one particle per
// thread, positions/velocities row-major [particle][dim] in HBM.
//
// Differences from the reference, by design:
//  * random numbers come from the stateless Philox generator (zb_philox.cuh)
//    instead of a per-particle cuRAND state;
//  * gBest is resolved deterministically at the end of each launch: every
//    block reduces its (f, index) minimum, the last block to finish (a
//    threadfence + counter handshake) reduces the block minima, ties going
//    to the lowest index, and updates gBest if strictly better.  The
//    reference races on gBestX inside the iteration (pso.cuh:63-67,
//    149-153); here every particle of iteration t sees the gBest of t-1;
//  * nothing returns to the host between iterations (the reference syncs and
//    copies gBest back every iteration, pso.cuh:326-333), so the whole loop
//    can be captured into one CUDA graph.
// Coefficients w, c1, c2 and the update v <- w v + c1 r1 (pb - x) +
// c2 r2 (gb - x), x <- x + v are the reference's (pso.cuh:104-119, 302).
//
// For D >= kPsoCoopMinDim a warp moves one particle (lane l takes
// coordinates l, l+32, ...) and evaluates f cooperatively: one thread per
// particle would serialise O(D^2) work per particle (the 150-D Gaussian)
// over a handful of SMs.  Positions and velocities are the same bits either
// way; f differs from the one-thread sum at rounding level.
#pragma once

#include "zb_bfgs_coop.cuh"
#include "zb_common.cuh"
#include "zb_philox.cuh"
#include "zb_sobol.cuh"

namespace zb {

  struct PsoWork {
    double* X;                     // n*D positions
    double* V;                     // n*D velocities
    unsigned long long* part_key;  // per-block minimum key
    int* part_idx;                 // per-block argmin
    unsigned int* counter;         // blocks finished in this launch
    double* gbest;                 // {f, x[D]}
    const uint32_t* sobol = nullptr; // Sobol' directions: initial positions
  };

  inline constexpr int kPsoBlock = 256;
  inline constexpr int kPsoCoopMinDim = 33;

  // Blocks of one PSO launch (one per-block minimum slot each).
  __host__ __device__ inline int64_t
  pso_blocks(int64_t n, int dim)
  {
    const int per = dim >= kPsoCoopMinDim ? kPsoBlock / 32 : kPsoBlock;
    return (n + per - 1) / per;
  }

  // Block-wide lexicographic min of (key, idx); result valid in thread 0.
  __device__ __forceinline__ void
  block_argmin(unsigned long long& key, int& idx)
  {
    __shared__ unsigned long long wk[32];
    __shared__ int wi[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long k2 = __shfl_down_sync(0xffffffffu, key, o);
      const int i2 = __shfl_down_sync(0xffffffffu, idx, o);
      if (k2 < key || (k2 == key && i2 < idx)) {
        key = k2;
        idx = i2;
      }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
      wk[warp] = key;
      wi[warp] = idx;
    }
    __syncthreads();
    if (warp == 0) {
      const int nw = (blockDim.x + 31) >> 5;
      key = lane < nw ? wk[lane] : ~0ull;
      idx = lane < nw ? wi[lane] : 0x7fffffff;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long k2 = __shfl_down_sync(0xffffffffu, key, o);
        const int i2 = __shfl_down_sync(0xffffffffu, idx, o);
        if (k2 < key || (k2 == key && i2 < idx)) {
          key = k2;
          idx = i2;
        }
      }
    }
  }

  // Block minima -> last block -> gBest update (strictly better only).
  template <int D>
  __device__ __forceinline__ void
  pso_publish(const PsoWork& w, const double* pos, unsigned long long key,
              int idx)
  {
    block_argmin(key, idx);
    __shared__ bool last;
    if (threadIdx.x == 0) {
      w.part_key[blockIdx.x] = key;
      w.part_idx[blockIdx.x] = idx;
      __threadfence();
      last = atomicAdd(w.counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last)
      return;
    __threadfence();
    unsigned long long k = ~0ull;
    int i = 0x7fffffff;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
      const unsigned long long kb =
        *reinterpret_cast<volatile unsigned long long*>(&w.part_key[b]);
      const int ib = *reinterpret_cast<volatile int*>(&w.part_idx[b]);
      if (kb < k || (kb == k && ib < i)) {
        k = kb;
        i = ib;
      }
    }
    block_argmin(k, i);
    __shared__ int take;
    if (threadIdx.x == 0) {
      take = -1;
      if (k != ~0ull) {
        // decode the key back to the value it came from
        const unsigned long long b =
          (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
        const double f = __longlong_as_double((long long)b);
        if (f < w.gbest[0]) {
          w.gbest[0] = f;
          take = i;
        }
      }
      *w.counter = 0u; // ready for the next launch
    }
    __syncthreads();
    if (take >= 0)
      for (int d = threadIdx.x; d < D; d += blockDim.x)
        w.gbest[1 + d] =
          *reinterpret_cast<const volatile double*>(&pos[(size_t)take * D + d]);
  }

  template <class F, int D>
  __global__ void __launch_bounds__(kPsoBlock)
    pso_init_kernel(F f, int64_t n, double lower, double upper, uint64_t seed,
                    PsoWork w, double* __restrict__ pbx,
                    double* __restrict__ pbf)
  {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long key = ~0ull;
    int kidx = 0x7fffffff;
    if (i < n) {
      const double vr = (upper - lower) * 0.1;
      std::array<double, D> xa;
#pragma unroll 1
      for (int d = 0; d < D; ++d) {
        const double ux = position01(w.sobol, seed, kTagPsoX, (uint64_t)i, (uint32_t)d);
        const double uv = uniform01(seed, kTagPsoV, (uint64_t)i, (uint32_t)d);
        const double rx = lower + (upper - lower) * ux;
        const double rv = -vr + (vr - -vr) * uv;
        w.X[i * D + d] = rx;
        w.V[i * D + d] = rv;
        pbx[i * D + d] = rx;
        xa[d] = rx;
      }
      const double fv = f(xa);
      pbf[i] = fv;
      key = order_key(fv);
      kidx = (int)i;
    }
    pso_publish<D>(w, w.X, key, kidx);
  }

  template <class F, int D>
  __global__ void __launch_bounds__(kPsoBlock)
    pso_iter_kernel(F f, int64_t n, double wi, double c1, double c2,
                    uint64_t seed, int t, PsoWork w,
                    double* __restrict__ pbx, double* __restrict__ pbf)
  {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long key = ~0ull;
    int kidx = 0x7fffffff;
    if (i < n) {
      const uint32_t tag = kTagPsoIter + (uint32_t)t;
      std::array<double, D> xa;
#pragma unroll 1
      for (int d = 0; d < D; ++d) {
        const double r1 = uniform01(seed, tag, (uint64_t)i, 2u * d);
        const double r2 = uniform01(seed, tag, (uint64_t)i, 2u * d + 1u);
        const double xi = w.X[i * D + d];
        const double vi = w.V[i * D + d];
        const double pb = pbx[i * D + d];
        const double gb = w.gbest[1 + d];
        const double nv = wi * vi + c1 * r1 * (pb - xi) + c2 * r2 * (gb - xi);
        const double nx = xi + nv;
        w.V[i * D + d] = nv;
        w.X[i * D + d] = nx;
        xa[d] = nx;
      }
      const double fv = f(xa);
      if (fv < pbf[i]) {
        pbf[i] = fv;
#pragma unroll 1
        for (int d = 0; d < D; ++d)
          pbx[i * D + d] = xa[d];
      }
      key = order_key(fv);
      kidx = (int)i;
    }
    pso_publish<D>(w, w.X, key, kidx);
  }

  // Warp-per-particle forms (D >= kPsoCoopMinDim): particle i is warp i of
  // the grid; the same random counters and update expressions as above.
  template <class F, int D>
  __global__ void __launch_bounds__(kPsoBlock)
    pso_init_coop_kernel(F f, int64_t n, double lower, double upper,
                         uint64_t seed, PsoWork w, double* __restrict__ pbx,
                         double* __restrict__ pbf)
  {
    __shared__ double scr[kPsoBlock];
    const int lane = threadIdx.x & 31;
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    unsigned long long key = ~0ull;
    int kidx = 0x7fffffff;
    if (i < n) { // warp-uniform
      const double vr = (upper - lower) * 0.1;
      for (int d = lane; d < D; d += 32) {
        const double ux = position01(w.sobol, seed, kTagPsoX, (uint64_t)i, (uint32_t)d);
        const double uv = uniform01(seed, kTagPsoV, (uint64_t)i, (uint32_t)d);
        const double rx = lower + (upper - lower) * ux;
        const double rv = -vr + (vr - -vr) * uv;
        w.X[i * D + d] = rx;
        w.V[i * D + d] = rv;
        pbx[i * D + d] = rx;
      }
      __syncwarp();
      const TileGroup<32> grp(cg::tiled_partition<32>(cg::this_thread_block()),
                              scr + (threadIdx.x & ~31));
      const double fv = coop_value<F, D>(f, grp, w.X + i * D);
      if (lane == 0) {
        pbf[i] = fv;
        key = order_key(fv);
        kidx = (int)i;
      }
    }
    pso_publish<D>(w, w.X, key, kidx);
  }

  template <class F, int D>
  __global__ void __launch_bounds__(kPsoBlock)
    pso_iter_coop_kernel(F f, int64_t n, double wi, double c1, double c2,
                         uint64_t seed, int t, PsoWork w,
                         double* __restrict__ pbx, double* __restrict__ pbf)
  {
    __shared__ double scr[kPsoBlock];
    const int lane = threadIdx.x & 31;
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    unsigned long long key = ~0ull;
    int kidx = 0x7fffffff;
    if (i < n) { // warp-uniform
      const uint32_t tag = kTagPsoIter + (uint32_t)t;
      for (int d = lane; d < D; d += 32) {
        const double r1 = uniform01(seed, tag, (uint64_t)i, 2u * d);
        const double r2 = uniform01(seed, tag, (uint64_t)i, 2u * d + 1u);
        const double xi = w.X[i * D + d];
        const double vi = w.V[i * D + d];
        const double pb = pbx[i * D + d];
        const double gb = w.gbest[1 + d];
        const double nv = wi * vi + c1 * r1 * (pb - xi) + c2 * r2 * (gb - xi);
        w.V[i * D + d] = nv;
        w.X[i * D + d] = xi + nv;
      }
      __syncwarp();
      const TileGroup<32> grp(cg::tiled_partition<32>(cg::this_thread_block()),
                              scr + (threadIdx.x & ~31));
      const double fv = coop_value<F, D>(f, grp, w.X + i * D);
      const bool better = fv < pbf[i];
      if (better)
        for (int d = lane; d < D; d += 32) // coordinates this lane wrote
          pbx[i * D + d] = w.X[i * D + d];
      __syncwarp(); // every lane has read pbf[i]
      if (lane == 0) {
        if (better)
          pbf[i] = fv;
        key = order_key(fv);
        kidx = (int)i;
      }
    }
    pso_publish<D>(w, w.X, key, kidx);
  }

  // gBest = {+inf, 0...}, counter = 0: the state before pso_init_kernel.
  template <int D>
  __global__ void
  pso_reset_kernel(PsoWork w)
  {
    if (threadIdx.x == 0) {
      w.gbest[0] = __longlong_as_double(0x7ff0000000000000ll);
      *w.counter = 0u;
    }
    for (int d = threadIdx.x; d < D; d += blockDim.x)
      w.gbest[1 + d] = 0.0;
  }

} // namespace zb
