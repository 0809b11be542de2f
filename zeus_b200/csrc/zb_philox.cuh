// Counter-based random numbers for start points and PSO.
//
// Philox4x32-10 as published by Salmon, Moraes, Dror and Shaw, "Parallel
// random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of two 32x32->64
// multiplies (0xD2511F53, 0xCD9E8D57) with Weyl key increments (0x9E3779B9,
// 0xBB67AE85).  Stateless: the value for (seed, stream tag, run, index) is a
// pure function, so no per-run generator state is kept in HBM (the
// reference stores a cuRAND state per run, bfgs_common.cuh:14-43).
#pragma once

#include <cstdint>

namespace zb {

  enum : uint32_t {
    kTagStarts = 1u,   // BFGS uniform starts
    kTagPsoX = 2u,     // PSO initial positions
    kTagPsoV = 3u,     // PSO initial velocities
    kTagPsoIter = 16u  // + t: PSO iteration t, r1 at 2d, r2 at 2d+1
  };

  __host__ __device__ inline void
  philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                uint32_t k0, uint32_t k1, uint32_t out[4])
  {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
      const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
      const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
      const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
      const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
      const uint32_t n0 = hi1 ^ c1 ^ k0;
      const uint32_t n2 = hi0 ^ c3 ^ k1;
      c0 = n0;
      c1 = lo1;
      c2 = n2;
      c3 = lo0;
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
  }

  // Uniform double in [0, 1) with 53 random bits.  Counter = (run lo,
  // index/2, tag, run hi), key = seed; one Philox block serves two indices.
  __host__ __device__ inline double
  uniform01(uint64_t seed, uint32_t tag, uint64_t run, uint32_t index)
  {
    uint32_t o[4];
    philox4x32_10((uint32_t)run, index >> 1, tag, (uint32_t)(run >> 32),
                  (uint32_t)seed, (uint32_t)(seed >> 32), o);
    const int w = (int)(index & 1u) * 2;
    const uint64_t bits = ((uint64_t)o[w] << 32) | o[w + 1];
    return (double)(bits >> 11) * (1.0 / 9007199254740992.0);
  }

} // namespace zb
