// Execution-space shim that lets the reference's header-only CUDA BFGS
// (include/bfgs_sequential.cuh, include/utils.cuh, include/duals.cuh and the
// objective headers under examples/) compile as ordinary host code.
//
// Test infrastructure only: the library built from this shim
// (oracle/_ref/libzeus_ref.so) is the reference's own algorithm run on the
// CPU.  It pins the C restatement in oracle/zeus_oracle.c and serves as the
// timed CPU baseline.  Nothing in the product links it.
//
// What the shim does (the TU is compiled by nvcc, which parses the
// reference's <<<>>> launches in its uninstantiated host templates):
//   * after the CUDA headers are in, redefines __device__ as __host__, so
//     every reference helper becomes a host-only function and no device code
//     is generated for it.  __global__ stays real until the driver has
//     included utils.cuh and bfgs_common.cuh (whose non-template
//     initializeSobolStates launches a kernel declared there); the driver then
//     redefines __global__ as __host__ so the BFGS kernel template is an
//     ordinary host function;
//   * provides the built-in index variables as thread-local host variables so
//     a host thread can play "run idx" (idx = blockIdx.x*blockDim.x+threadIdx.x);
//   * maps the device atomics the reference uses on its BFGSContext to GCC
//     __atomic builtins, clock64() to 0 (cycle counters are not used) and
//     asm("trap;") to abort().
#pragma once

#include <algorithm>
#include <array>
#include <atomic>
#include <cassert>
#include <cmath>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <string_view>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include <cuda_runtime.h>
#include <curand_kernel.h> // the stub in stubs/, found first on the path
#include <cub/cub.cuh>     // the stub in stubs/

#undef __device__
#define __device__ __host__

using std::isfinite;
using std::isinf;
using std::isnan;

struct zref_index3 {
  unsigned int x, y, z;
};
extern thread_local zref_index3 zref_blockIdx;
extern thread_local zref_index3 zref_threadIdx;
extern thread_local zref_index3 zref_blockDim;
#define blockIdx zref_blockIdx
#define threadIdx zref_threadIdx
#define blockDim zref_blockDim

#define atomicAdd zref_atomicAdd
#define atomicExch zref_atomicExch
#define atomicCAS zref_atomicCAS
#define __threadfence zref_threadfence
#define clock64 zref_clock64
#define __longlong_as_double zref_longlong_as_double
#define __double_as_longlong zref_double_as_longlong

inline int
atomicAdd(int* p, int v)
{
  return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST);
}
inline int
atomicExch(int* p, int v)
{
  return __atomic_exchange_n(p, v, __ATOMIC_SEQ_CST);
}
inline unsigned long long
atomicCAS(unsigned long long* p, unsigned long long expected,
          unsigned long long desired)
{
  __atomic_compare_exchange_n(p, &expected, desired, false, __ATOMIC_SEQ_CST,
                              __ATOMIC_SEQ_CST);
  return expected;
}
inline void
__threadfence()
{
  __atomic_thread_fence(__ATOMIC_SEQ_CST);
}
inline long long
clock64()
{
  return 0;
}
inline double
__longlong_as_double(unsigned long long b)
{
  double d;
  std::memcpy(&d, &b, sizeof d);
  return d;
}
inline unsigned long long
__double_as_longlong(double d)
{
  unsigned long long b;
  std::memcpy(&b, &d, sizeof b);
  return b;
}

// device_matrix.cuh traps on heap exhaustion with asm("trap;")
#define asm(...) ::abort()
