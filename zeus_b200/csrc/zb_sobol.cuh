// Quasi-random start positions: Sobol' points, digitally shifted by the seed.
//
// The reference offers PRNGType::SOBOL (traits.hpp:67-71), a cuRAND Sobol32
// state per run (bfgs_common.cuh:46-81, src/utils.cu:41-49) that feeds the
// PSO's positions and its other draws.  Here the Sobol' point set itself is
// the start design: run i takes point i of the D-dimensional sequence,
// coordinate d its dimension d, so the starts of any 2^m consecutive runs
// are stratified in every coordinate.  Velocities and the PSO's r1/r2 stay
// on Philox (a low-discrepancy sequence reused across iterations correlates
// the swarm's moves).
//
// Construction (Sobol' 1967; recurrence as in Bratley and Fox, ACM TOMS 14
// (1988) 88-100): dimension 0 is the van der Corput sequence in base 2,
// dimension j >= 1 uses the j-th primitive polynomial over GF(2) in order
// of degree, then value, with initial direction numbers m_1..m_s (odd,
// m_k < 2^k) drawn from a fixed splitmix64 stream.  The table is built on
// the host (zb_sobol.cu) and kept in device memory: dirs[d * 32 + k] is the
// direction number v_{k+1} of dimension d as a 32-bit binary fraction.
// Point n in natural order is the XOR of v_{k+1} over the set bits k of n;
// the digital shift XORs in 32 Philox bits per dimension.
#pragma once

#include <cstdint>

#include "zb_philox.cuh"

namespace zb {

  inline constexpr int kSobolMaxDim = 1024; // the largest dimension built
  inline constexpr int kSobolBits = 32;
  enum : uint32_t { kTagSobolShift = 4u };

  __host__ __device__ inline int
  ctz32(uint32_t m)
  {
#ifdef __CUDA_ARCH__
    return __ffs((int)m) - 1;
#else
    return __builtin_ctz(m);
#endif
  }

  // 32 random bits per (seed, dimension): the digital shift.
  __host__ __device__ inline uint32_t
  sobol_shift(uint64_t seed, uint32_t d)
  {
    uint32_t o[4];
    philox4x32_10(d, 0u, kTagSobolShift, 0u, (uint32_t)seed,
                  (uint32_t)(seed >> 32), o);
    return o[0];
  }

  // Point `run` (low 32 bits), coordinate d, shifted, as the midpoint of its
  // 2^-32 cell: a double in (0, 1).
  __host__ __device__ inline double
  sobol01(const uint32_t* __restrict__ dirs, uint64_t seed, uint64_t run,
          uint32_t d)
  {
    uint32_t x = sobol_shift(seed, d);
    const uint32_t* v = dirs + (size_t)d * kSobolBits;
    for (uint32_t m = (uint32_t)run; m; m &= m - 1u)
      x ^= v[ctz32(m)];
    return ((double)x + 0.5) * (1.0 / 4294967296.0);
  }

  // A run's position coordinate in [0, 1): Sobol' when a direction table is
  // given, else the Philox uniform of stream `tag`.
  __host__ __device__ inline double
  position01(const uint32_t* sobol, uint64_t seed, uint32_t tag, uint64_t run,
             uint32_t d)
  {
    return sobol ? sobol01(sobol, seed, run, d) : uniform01(seed, tag, run, d);
  }

  // Host table for dimensions [0, ndim), dirs[d * 32 + k] (zb_sobol.cu).
  void sobol_table(int ndim, uint32_t* dirs);
  // The table for all kSobolMaxDim dimensions in the current device's
  // memory; built and copied on the first call per device (synchronous).
  int sobol_table_device(const uint32_t** out);

} // namespace zb
