// PSO seeding that allocates nothing.
//
// Some callers cannot allocate device memory at the point where they seed a
// swarm: code running inside a region whose allocator belongs to another
// framework (a host application that hands the library only its own
// buffers), real-time loops that forbid allocation after start-up, or hosts
// whose allocation calls would implicitly synchronize a device they are
// pipelining.  zeus_pso_device needs a caller-provided workspace for the
// swarm state (positions, velocities, per-block minima and the launch
// counter); this entry point keeps that state in one fixed array compiled
// into the library instead, so the caller passes only its inputs and
// outputs.
//
// The array is kNoAllocScratchBytes (8 MiB) of device memory that every GPU
// which loads the library keeps until the process exits.  Every call shares
// it: the last call's contents stay there, the kernels clear what must start
// at zero (the launch counter and gBest) at the beginning of each call, and
// two calls that overlap on the GPU (different streams, or other threads)
// race on it and corrupt each other -- callers must serialize them.
#include <mutex>

#include "zb_internal.h"
#include "zb_pso.cuh"

namespace zb {

  namespace {

    constexpr size_t kNoAllocScratchBytes = 8u << 20;

    static __device__ __align__(256) unsigned char
      g_noalloc_scratch[kNoAllocScratchBytes];

    // The array's device address, looked up once per device with that
    // device current (the symbol's host-side name is not a device address).
    void*
    scratch_address(int* rc)
    {
      static std::mutex mu;
      static void* addr[64] = {};
      int dev = 0;
      cudaError_t e = cudaGetDevice(&dev);
      if (e != cudaSuccess) {
        *rc = cuda_fail(e, "zeus_pso_device_noalloc: cudaGetDevice");
        return nullptr;
      }
      if (dev < 0 || dev >= 64) {
        set_error("zeus_pso_device_noalloc: device index %d out of range", dev);
        *rc = ZEUS_E_INVALID;
        return nullptr;
      }
      std::lock_guard<std::mutex> lk(mu);
      if (!addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
          *rc = cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                          "zeus_pso_device_noalloc: cudaGetSymbolAddress");
          return nullptr;
        }
        addr[dev] = p;
      }
      *rc = ZEUS_OK;
      return addr[dev];
    }

  } // namespace

} // namespace zb

using namespace zb;

extern "C" {

int
zeus_pso_device_noalloc(const zeus_problem* problem, uint64_t seed, int64_t n,
                        double lower, double upper, int32_t iters, double w,
                        double c1, double c2, double* d_pbest_x,
                        double* d_pbest_f, double* d_gbest, void* stream)
{
  if (!problem || n < 0 || iters < 0 ||
      (n > 0 && (!d_pbest_x || !d_pbest_f || !d_gbest))) {
    set_error("zeus_pso_device_noalloc: bad arguments");
    return ZEUS_E_INVALID;
  }
  if (!pso_supported(problem->kind, problem->dim)) {
    set_error("zeus_pso_device_noalloc: objective kind %d with dim %d is not built",
              problem->kind, problem->dim);
    return ZEUS_E_UNSUPPORTED;
  }
  if (n == 0)
    return ZEUS_OK;
  if (n > 0x7fffffffLL) {
    set_error("zeus_pso_device_noalloc: n must fit in int32");
    return ZEUS_E_INVALID;
  }
  const size_t need = pso_workspace_bytes(n, problem->dim);
  if (need > kNoAllocScratchBytes) {
    set_error("zeus_pso_device_noalloc: %lld particles of dimension %d need %zu "
              "bytes of swarm state; the fixed array holds %zu (use "
              "zeus_pso_device with a workspace)",
              (long long)n, problem->dim, need, kNoAllocScratchBytes);
    return ZEUS_E_WORKSPACE;
  }
  int rc = ZEUS_OK;
  void* scratch = scratch_address(&rc);
  if (!scratch)
    return rc;
  Objective o{problem->kind, problem->dim,   problem->data, problem->idata,
              problem->ndata, problem->flags, nullptr};
  return launch_pso(o, seed, n, lower, upper, iters, w, c1, c2, d_pbest_x,
                    d_pbest_f, d_gbest, scratch, kNoAllocScratchBytes,
                    (cudaStream_t)stream);
}

} // extern "C"
