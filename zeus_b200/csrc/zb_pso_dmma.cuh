// PSO for the Gaussian quadratic form on the FP64 tensor cores (DMMA).
//
// f(x) = 0.5 x^T C x is the one objective here whose work is a dense
// contraction shared by every particle: with the particles' positions as
// the rows of X, the swarm needs Y = X C^T and f_i = 0.5 X_i . Y_i.  A block
// takes 8 particles; its warps split their 8 x D block of Y by 8-column
// tiles and form them with mma.sync.m8n8k4.f64 (8 x 8 x 4 per instruction,
// FP64 in and out): the 8 x 4 A fragments are rows of X, the 4 x 8 B
// fragments columns of C^T (rows of C), read straight from L1/L2 (C is
// shared by the whole swarm).
// Positions, velocities and the random counters are the one-particle
// kernels' (zb_pso.cuh); only f's summation order differs.
#pragma once

#include "zb_objectives.cuh"
#include "zb_pso.cuh"

namespace zb {

  inline constexpr int kPsoDmmaParticles = 8; // per block
  // the block's positions are staged in static shared memory (8 x D doubles)
  inline constexpr int kPsoDmmaMaxDim = 512;

  // This warp's share of f for the block's 8 particles, whose positions are
  // the rows of Xs (shared memory, 8 x D; rows past the swarm are zeros):
  // the 8-column tiles jt = jt0, jt0 + jstep, ... of Y = X C^T, each dotted
  // with the same columns of X.  Returns in lane 4r the partial sum of row
  // r.  Fragment layouts of m8n8k4.f64 (PTX ISA, "Matrix fragments for
  // mma.m8n8k4 with .f64"): A[lane/4][lane%4], B[lane%4][lane/4],
  // D[lane/4][2*(lane%4) + {0, 1}].  The MMAs are not volatile, so the
  // compiler may issue the loads of C several k steps ahead of their use.
  template <int D>
  __device__ __forceinline__ double
  gauss_f8_dmma_part(const double* __restrict__ C, const double* __restrict__ Xs,
                     int lane, int jt0, int jstep)
  {
    const int r = lane >> 2, c4 = lane & 3;
    const double* xr = Xs + r * D;
    double acc = 0.0;
    for (int jt = jt0; jt < (D + 7) / 8; jt += jstep) {
      // two accumulator tiles (even and odd k steps): half the chain of
      // dependent MMAs
      double e0 = 0.0, e1 = 0.0, o0 = 0.0, o1 = 0.0;
      const int jb = jt * 8 + r; // the B column (a row of C) this lane loads
      const bool bv = jb < D;
      const double* cb = C + (size_t)(bv ? jb : 0) * D;
      // the B operands of up to 40 k steps (D = 150: the whole tile) are
      // loaded before their MMAs: that many independent loads in flight
      // instead of one L2 round trip a step
      constexpr int KT = (D + 3) / 4;
      constexpr int KC = KT < 40 ? KT : 40;
      for (int k0 = 0; k0 < KT; k0 += KC) {
        double bk[KC];
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) {
          const int k = (k0 + kk) * 4 + c4;
          bk[kk] = (bv && k < D) ? cb[k] : 0.0;
        }
#pragma unroll
        for (int kk = 0; kk < KC; kk += 2) {
          const int k = (k0 + kk) * 4 + c4, k2 = k + 4;
          const double a = k < D ? xr[k] : 0.0;
          const double a2 = (kk + 1 < KC && k2 < D) ? xr[k2] : 0.0;
          const double b2 = kk + 1 < KC ? bk[kk + 1] : 0.0;
          asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 "
              "{%0, %1}, {%2}, {%3}, {%0, %1};"
              : "+d"(e0), "+d"(e1)
              : "d"(a), "d"(bk[kk]));
          asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 "
              "{%0, %1}, {%2}, {%3}, {%0, %1};"
              : "+d"(o0), "+d"(o1)
              : "d"(a2), "d"(b2));
        }
      }
      const double d0 = e0 + o0, d1 = e1 + o1;
      const int j0 = jt * 8 + c4 * 2;
      if (j0 < D)
        acc = fma(xr[j0], d0, acc);
      if (j0 + 1 < D)
        acc = fma(xr[j0 + 1], d1, acc);
    }
    // the four lanes of a row hold its partial sums
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    return acc;
  }

  // f of the block's 8 particles (rows of Xs): every warp takes every 8th
  // column tile; thread t < 8 returns particle t's value.  `part` is 8 x 8
  // doubles of shared memory.
  template <int D>
  __device__ __forceinline__ double
  gauss_f8_dmma(const double* __restrict__ C, const double* __restrict__ Xs,
                double* part)
  {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    const double a = gauss_f8_dmma_part<D>(C, Xs, lane, warp, nw);
    if ((lane & 3) == 0)
      part[warp * 8 + (lane >> 2)] = a;
    __syncthreads();
    double f = 0.0;
    if (threadIdx.x < kPsoDmmaParticles)
      for (int w = 0; w < nw; ++w)
        f += part[w * 8 + threadIdx.x];
    return 0.5 * f;
  }

  __host__ __device__ inline int64_t
  pso_dmma_blocks(int64_t n)
  {
    return (n + kPsoDmmaParticles - 1) / kPsoDmmaParticles;
  }

  template <int D>
  __global__ void __launch_bounds__(kPsoBlock)
    pso_init_dmma_kernel(zeus::Gaussian<D> f, int64_t n, double lower, double upper,
                         uint64_t seed, PsoWork w, double* __restrict__ pbx,
                         double* __restrict__ pbf)
  {
    static_assert(D <= kPsoDmmaMaxDim, "positions staged in static shared memory");
    __shared__ double part[(kPsoBlock / 32) * 8];
    __shared__ double Xs[kPsoDmmaParticles * D];
    const int t = threadIdx.x;
    const int64_t i0 = (int64_t)blockIdx.x * kPsoDmmaParticles;
    const int64_t cnt = n - i0 < kPsoDmmaParticles ? n - i0 : kPsoDmmaParticles;
    const double vr = (upper - lower) * 0.1;
    for (int e = (int)cnt * D + t; e < kPsoDmmaParticles * D; e += blockDim.x)
      Xs[e] = 0.0;
    for (int e = t; e < cnt * D; e += blockDim.x) {
      const int64_t i = i0 + e / D;
      const int d = e % D;
      const double ux = position01(w.sobol, seed, kTagPsoX, (uint64_t)i, (uint32_t)d);
      const double uv = uniform01(seed, kTagPsoV, (uint64_t)i, (uint32_t)d);
      const double rx = lower + (upper - lower) * ux;
      const double rv = -vr + (vr - -vr) * uv;
      w.X[i * D + d] = rx;
      w.V[i * D + d] = rv;
      pbx[i * D + d] = rx;
      Xs[e] = rx;
    }
    __syncthreads();
    const double fv = gauss_f8_dmma<D>(f.C, Xs, part);
    unsigned long long key = ~0ull;
    int kidx = 0x7fffffff;
    if (t < cnt) {
      pbf[i0 + t] = fv;
      key = order_key(fv);
      kidx = (int)(i0 + t);
    }
    pso_publish<D>(w, w.X, key, kidx);
  }

  template <int D>
  __global__ void __launch_bounds__(kPsoBlock)
    pso_iter_dmma_kernel(zeus::Gaussian<D> f, int64_t n, double wi, double c1, double c2,
                         uint64_t seed, int t, PsoWork w, double* __restrict__ pbx,
                         double* __restrict__ pbf)
  {
    static_assert(D <= kPsoDmmaMaxDim, "positions staged in static shared memory");
    __shared__ double part[(kPsoBlock / 32) * 8];
    __shared__ double Xs[kPsoDmmaParticles * D];
    __shared__ int better[kPsoDmmaParticles];
    const int tid = threadIdx.x;
    const int64_t i0 = (int64_t)blockIdx.x * kPsoDmmaParticles;
    const int64_t cnt = n - i0 < kPsoDmmaParticles ? n - i0 : kPsoDmmaParticles;
    const uint32_t tag = kTagPsoIter + (uint32_t)t;
    for (int e = (int)cnt * D + tid; e < kPsoDmmaParticles * D; e += blockDim.x)
      Xs[e] = 0.0;
    for (int e = tid; e < cnt * D; e += blockDim.x) {
      const int64_t i = i0 + e / D;
      const int d = e % D;
      const double r1 = uniform01(seed, tag, (uint64_t)i, 2u * d);
      const double r2 = uniform01(seed, tag, (uint64_t)i, 2u * d + 1u);
      const double xi = w.X[i * D + d];
      const double vi = w.V[i * D + d];
      const double pb = pbx[i * D + d];
      const double gb = w.gbest[1 + d];
      const double nv = wi * vi + c1 * r1 * (pb - xi) + c2 * r2 * (gb - xi);
      w.V[i * D + d] = nv;
      w.X[i * D + d] = xi + nv;
      Xs[e] = xi + nv;
    }
    __syncthreads();
    const double fv = gauss_f8_dmma<D>(f.C, Xs, part);
    unsigned long long key = ~0ull;
    int kidx = 0x7fffffff;
    if (tid < kPsoDmmaParticles) {
      const bool b = tid < cnt && fv < pbf[i0 + tid];
      better[tid] = b;
      if (b)
        pbf[i0 + tid] = fv;
      if (tid < cnt) {
        key = order_key(fv);
        kidx = (int)(i0 + tid);
      }
    }
    __syncthreads();
    for (int e = tid; e < cnt * D; e += blockDim.x) {
      const int64_t i = i0 + e / D;
      if (better[e / D])
        pbx[i * D + e % D] = Xs[e];
    }
    pso_publish<D>(w, w.X, key, kidx);
  }

} // namespace zb
