// The reference's own sequential BFGS kernel (include/bfgs_sequential.cuh:
// 16-234, bfgs::sequential::optimize) compiled for sm_100a and launched on the
// GPU with injected starts -- the reference's integration-test entry
// (test/bfgs_tests.cu:297-317: pso_array set, SaveTrajectories on) -- so that
// the library's exact mode can be compared with the reference's arithmetic on
// the same device libm (cos, exp, log, pow, lgamma of CUDA's math library).
//
// Test infrastructure only: built from the reference sources where they lie
// (oracle/Makefile, target ref-gpu) into oracle/_ref/libzeus_ref_gpu.so; the
// product never links it.  Compiled with -fmad=false, as the library's exact
// mode is, so that both keep the reference's operation order without
// contraction (the reference's own build contracts with nvcc's default).
//
// The kernel allocates its two D x D matrices from the device heap
// (include/device_matrix.cuh:45-50, a trap when malloc fails), so the entry
// point sizes the heap for every run before the launch and refuses the call
// when the heap cannot hold them.
#include <cuda_runtime.h>

#include "duals.cuh"
#include "utils.cuh"
#include "pso.cuh"
#include "traits.hpp"
#include "bfgs_common.cuh"
#include "bfgs_sequential.cuh"
#include "rosenbrock.hpp"
#include "rastrigin.hpp"
#include "ackley.hpp"
#include "simulation/fitting/LogLikelihood.h"

#include <cstdint>
#include <cstdio>
#include <vector>

// the reference's digamma (src/duals.cu:10-39), compiled into this TU
#include "duals.cu"

namespace {

  // heap per run: two D x D doubles plus the allocator's own overhead, with
  // a factor of four to spare
  constexpr std::size_t kHeapSlack = 4;
  constexpr std::size_t kHeapFloor = std::size_t(64) << 20;
  constexpr std::size_t kStackBytes = 64 * 1024; // util::setStackSize's value

  struct Outputs {
    double* fval;
    int* status;
    int* iter;
    double* gnorm;
    double* x_out;
    double* traj_x;
    double* traj_f;
    double* traj_g;
    signed char* traj_status;
  };

  int
  fail(cudaError_t e, const char* what)
  {
    if (e == cudaSuccess)
      return 0;
    std::fprintf(stderr, "zrefg: %s: %s\n", what, cudaGetErrorString(e));
    return -2;
  }

  template <class T>
  struct DevBuf {
    T* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    int
    alloc(std::size_t n)
    {
      return fail(cudaMalloc(&p, sizeof(T) * (n ? n : 1)), "cudaMalloc");
    }
  };

  int
  size_device_heap(int n, std::size_t dim)
  {
    const std::size_t need =
      kHeapSlack * (std::size_t)n * 2 * dim * dim * sizeof(double);
    const std::size_t want = need > kHeapFloor ? need : kHeapFloor;
    std::size_t have = 0;
    if (fail(cudaDeviceGetLimit(&have, cudaLimitMallocHeapSize), "heap limit"))
      return -2;
    if (have < want)
      cudaDeviceSetLimit(cudaLimitMallocHeapSize, want);
    if (fail(cudaDeviceGetLimit(&have, cudaLimitMallocHeapSize), "heap limit") ||
        have < need) {
      std::fprintf(stderr, "zrefg: device heap of %zu bytes, %zu needed\n", have,
                   need);
      return -3;
    }
    std::size_t stack = 0;
    cudaDeviceGetLimit(&stack, cudaLimitStackSize);
    if (stack < kStackBytes &&
        fail(cudaDeviceSetLimit(cudaLimitStackSize, kStackBytes), "stack limit"))
      return -2;
    return 0;
  }

  template <class F, std::size_t D>
  int
  run(const F& f, const double* starts, int n, double lower, double upper,
      int max_iter, int required, double tol, const Outputs& o)
  {
    if (n <= 0)
      return 0;
    int rc = size_device_heap(n, D);
    if (rc)
      return rc;
    const bool traj = o.traj_x && o.traj_f && o.traj_g && o.traj_status;
    const std::size_t nt = traj ? (std::size_t)max_iter * n : 0;
    DevBuf<double> d_starts, d_dev_results, d_tx, d_tf, d_tg;
    DevBuf<int8_t> d_ts;
    DevBuf<zeus::Result<D>> d_res;
    DevBuf<curandStateXORWOW_t> d_states;
    DevBuf<util::BFGSContext> d_ctx;
    if ((rc = d_starts.alloc((std::size_t)n * D)) || (rc = d_dev_results.alloc(n)) ||
        (rc = d_res.alloc(n)) || (rc = d_states.alloc(n)) || (rc = d_ctx.alloc(1)))
      return rc;
    if (traj && ((rc = d_tx.alloc(nt * D)) || (rc = d_tf.alloc(nt)) ||
                 (rc = d_tg.alloc(nt)) || (rc = d_ts.alloc(nt))))
      return rc;
    if ((rc = fail(cudaMemcpy(d_starts.p, starts, sizeof(double) * n * D,
                              cudaMemcpyHostToDevice), "starts in")) ||
        (rc = fail(cudaMemset(d_ctx.p, 0, sizeof(util::BFGSContext)), "context")) ||
        (rc = fail(cudaMemset(d_states.p, 0, sizeof(curandStateXORWOW_t) * n),
                   "states")))
      return rc;
    if (traj &&
        ((rc = fail(cudaMemcpy(d_tx.p, o.traj_x, sizeof(double) * nt * D,
                               cudaMemcpyHostToDevice), "trajectory prefill")) ||
         (rc = fail(cudaMemcpy(d_tf.p, o.traj_f, sizeof(double) * nt,
                               cudaMemcpyHostToDevice), "trajectory prefill")) ||
         (rc = fail(cudaMemcpy(d_tg.p, o.traj_g, sizeof(double) * nt,
                               cudaMemcpyHostToDevice), "trajectory prefill")) ||
         (rc = fail(cudaMemcpy(d_ts.p, o.traj_status, nt, cudaMemcpyHostToDevice),
                    "trajectory prefill"))))
      return rc;
    constexpr unsigned kBlock = 128;
    const unsigned grid = (unsigned)((n + kBlock - 1) / kBlock);
    if (traj)
      bfgs::sequential::optimize<F, D, kBlock, true, curandStateXORWOW_t>
        <<<grid, kBlock>>>(f, lower, upper, d_starts.p,
                           util::NonNull{d_dev_results.p}, d_tx.p, d_tf.p, d_tg.p,
                           d_ts.p, n, max_iter, required, tol, 0,
                           util::NonNull{d_res.p}, util::NonNull{d_states.p},
                           util::NonNull{d_ctx.p});
    else
      bfgs::sequential::optimize<F, D, kBlock, false, curandStateXORWOW_t>
        <<<grid, kBlock>>>(f, lower, upper, d_starts.p,
                           util::NonNull{d_dev_results.p}, nullptr, nullptr,
                           nullptr, nullptr, n, max_iter, required, tol, 0,
                           util::NonNull{d_res.p}, util::NonNull{d_states.p},
                           util::NonNull{d_ctx.p});
    if ((rc = fail(cudaGetLastError(), "launch")) ||
        (rc = fail(cudaDeviceSynchronize(), "kernel")))
      return rc;
    std::vector<zeus::Result<D>> res(n);
    if ((rc = fail(cudaMemcpy(res.data(), d_res.p, sizeof(zeus::Result<D>) * n,
                              cudaMemcpyDeviceToHost), "results out")))
      return rc;
    if (traj &&
        ((rc = fail(cudaMemcpy(o.traj_x, d_tx.p, sizeof(double) * nt * D,
                               cudaMemcpyDeviceToHost), "trajectory out")) ||
         (rc = fail(cudaMemcpy(o.traj_f, d_tf.p, sizeof(double) * nt,
                               cudaMemcpyDeviceToHost), "trajectory out")) ||
         (rc = fail(cudaMemcpy(o.traj_g, d_tg.p, sizeof(double) * nt,
                               cudaMemcpyDeviceToHost), "trajectory out")) ||
         (rc = fail(cudaMemcpy(o.traj_status, d_ts.p, nt, cudaMemcpyDeviceToHost),
                    "trajectory out"))))
      return rc;
    for (int i = 0; i < n; ++i) {
      if (o.fval)
        o.fval[i] = res[i].fval;
      if (o.status)
        o.status[i] = res[i].status;
      if (o.iter)
        o.iter[i] = res[i].iter;
      if (o.gnorm)
        o.gnorm[i] = res[i].gradientNorm;
      if (o.x_out)
        for (std::size_t d = 0; d < D; ++d)
          o.x_out[(std::size_t)i * D + d] = res[i].coordinates[d];
    }
    return 0;
  }

} // namespace

extern "C" {

/// Objective kinds shared with oracle/zeus_oracle.h.
enum { ZREFG_ROSENBROCK = 0, ZREFG_RASTRIGIN = 1, ZREFG_ACKLEY = 2,
       ZREFG_POISSON_NLL = 4 };

/// The reference's sequential BFGS on the GPU for n injected starts
/// (row-major, starts[i*dim+d]); the same signature as the host build's
/// zref_bfgs (nthreads is unused).  Trajectory buffers use the reference
/// layout [iter][dim][run] / [iter][run] (bfgs_sequential.cuh:100-109) and
/// must be NaN / -1 prefilled by the caller.  Returns 0; -1 for a (kind,
/// dim) not instantiated here; -2 for a CUDA error; -3 when the device heap
/// cannot hold every run's matrices.
int
zrefg_bfgs(int kind, int dim, const double* data, const int* idata, int ndata,
           const double* starts, int n, double lower, double upper, int max_iter,
           int required, double tol, double* fval, int* status, int* iter,
           double* gnorm, double* x_out, double* traj_x, double* traj_f,
           double* traj_g, signed char* traj_status, int /*nthreads*/)
{
  const Outputs o{fval, status, iter, gnorm, x_out, traj_x, traj_f, traj_g,
                  traj_status};
#define ZREFG_CASE(KIND, D, OBJ)                                               \
  if (kind == KIND && dim == D)                                                \
    return run<OBJ, D>(OBJ{}, starts, n, lower, upper, max_iter, required, tol, \
                       o);
  ZREFG_CASE(ZREFG_ROSENBROCK, 2, util::Rosenbrock<2>)
  ZREFG_CASE(ZREFG_ROSENBROCK, 8, util::Rosenbrock<8>)
  ZREFG_CASE(ZREFG_RASTRIGIN, 2, util::Rastrigin<2>)
  ZREFG_CASE(ZREFG_RASTRIGIN, 10, util::Rastrigin<10>)
  ZREFG_CASE(ZREFG_ACKLEY, 2, util::Ackley<2>)
  ZREFG_CASE(ZREFG_ACKLEY, 30, util::Ackley<30>)
#undef ZREFG_CASE
  if (kind == ZREFG_POISSON_NLL && dim == 4 && data && idata && ndata > 0) {
    std::vector<int> counts(idata, idata + ndata);
    std::vector<double> centres(data, data + ndata);
    LogLikelihood ll(counts, centres);
    return run<LogLikelihood, 4>(ll, starts, n, lower, upper, max_iter, required,
                                 tol, o);
  }
  return -1;
}

} // extern "C"
