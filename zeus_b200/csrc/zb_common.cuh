// Shared device-side types and helpers for the BFGS / PSO kernels.
#pragma once

#include <array>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <type_traits>

#include "zb_dual.cuh"

namespace zb {

  // Status codes of the reference's Result::status (util.hpp:39-44).
  enum : int {
    kUnset = -1,
    kSurrender = 0,
    kConverged = 1,
    kStopped = 2,
    kNonFinite = 5
  };

  // Line-search constants (utils.cuh:389-395) and the update skip threshold
  // (utils.cuh:254-255).
  inline constexpr double kArmijoC1 = 0.1;
  inline constexpr int kLineSearchTrials = 20;
  inline constexpr double kMinCurvature = 1e-14;

  // 2^-k for 0 <= k <= 1022, built from its exponent bits (the line-search
  // step sizes alpha_k, exact).
  __host__ __device__ __forceinline__ double
  pow2neg(int k)
  {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)(1023 - k) << 52);
#else
    union {
      unsigned long long u;
      double d;
    } b;
    b.u = (unsigned long long)(1023 - k) << 52;
    return b.d;
#endif
  }

  struct BfgsParams {
    int64_t n;
    int max_iter;
    int required;
    double tol;
    int flags; // ZEUS_FLAG_* (include/zeus_b200.h)
  };

  inline constexpr int kFlagNoFixedPoint = 1;

  // Device view of zeus_run_outputs (include/zeus_b200.h).
  struct RunOut {
    double* fval;
    int32_t* status;
    int32_t* iter;
    double* gnorm;
    double* x;
    int64_t* counters; // [run][3]: iterations, f evaluations, gradients
    double* traj_x;
    double* traj_f;
    double* traj_g;
    int8_t* traj_status;
    int64_t* cycles; // [run][3]: gradient, update, whole-run clock64 cycles
  };

  // Per-run cycle counts, the reference's AD / BFGS / total timers
  // (bfgs_sequential.cuh:93-97, 150-155, 166-174, 229-232), sampled only
  // when the caller asked for them (RunOut::cycles non-null): clock64 spans
  // of the gradient evaluations, of the inverse-Hessian update (with the
  // new search direction where a layout fuses the two) and of the whole
  // run, as the leader of the run's group (its rank 0) sees them.  The
  // spans accumulate in the run's three output slots themselves (minus the
  // clock at a span's start, plus it at its end), so the timer holds no
  // registers across the loop.  Kernels instantiate it only when the
  // caller asks for cycles (CycleTimer<false> is empty): even off, the
  // timer's branches and stores cost the fused layouts several percent.
  template <bool On = true>
  struct CycleTimer {
    const RunOut& out;
    int64_t run;
    bool lead;
    __device__ __forceinline__
    CycleTimer(const RunOut& o, int64_t r, bool leader)
      : out(o), run(r), lead(leader)
    {
      if (out.cycles && lead) {
        out.cycles[3 * run + 0] = 0;
        out.cycles[3 * run + 1] = 0;
        out.cycles[3 * run + 2] = -(int64_t)clock64();
      }
    }
    __device__ __forceinline__ void
    start(int k) const
    {
      if (out.cycles && lead)
        out.cycles[3 * run + k] -= (int64_t)clock64();
    }
    __device__ __forceinline__ void
    stop(int k) const
    {
      if (out.cycles && lead)
        out.cycles[3 * run + k] += (int64_t)clock64();
    }
    __device__ __forceinline__ void
    start_grad() const
    {
      start(0);
    }
    __device__ __forceinline__ void
    stop_grad() const
    {
      stop(0);
    }
    __device__ __forceinline__ void
    start_update() const
    {
      start(1);
    }
    __device__ __forceinline__ void
    stop_update() const
    {
      stop(1);
    }
    // the whole run's span; after the run's last timed phase
    __device__ __forceinline__ void
    finish() const
    {
      stop(2);
    }
  };
  template <>
  struct CycleTimer<false> {
    __device__ __forceinline__ CycleTimer(const RunOut&, int64_t, bool) {}
    __device__ __forceinline__ void start_grad() const {}
    __device__ __forceinline__ void stop_grad() const {}
    __device__ __forceinline__ void start_update() const {}
    __device__ __forceinline__ void stop_update() const {}
    __device__ __forceinline__ void finish() const {}
  };



  // {stop flag, converged count}: the reference's BFGSContext
  // (context.hpp:7-10), device-global.
  struct Control {
    int stop;
    int converged;
  };

  template <class F>
  concept HasValue = requires(const F& f, const double* x) {
    { f.value(x) } -> std::convertible_to<double>;
  };
  template <class F>
  concept HasAdjoint = requires(const F& f, const double* x, double* g) {
    { f.adjoint(x, g) } -> std::convertible_to<double>;
  };

  // Relaxed read of the stop flag, issued once per BFGS iteration like the
  // reference's atomicAdd(&stopFlag, 0) (bfgs_common.cuh:127).
  __device__ __forceinline__ int
  load_stop(const Control* c)
  {
    return *reinterpret_cast<const volatile int*>(&c->stop);
  }

  // Marks one more converged run; raises the stop flag at `required`
  // (bfgs_common.cuh:184-193).
  __device__ __forceinline__ void
  note_converged(Control* c, int required)
  {
    const int old = atomicAdd(&c->converged, 1);
    if (old + 1 == required) {
      atomicExch(&c->stop, 1);
      __threadfence();
    }
  }

  // fval as an unsigned key ordered like the doubles; NaN maps above +inf so
  // it never wins a min.
  __device__ __forceinline__ unsigned long long
  order_key(double f)
  {
    if (f != f)
      return ~0ull;
    unsigned long long b = (unsigned long long)__double_as_longlong(f);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
  }

} // namespace zb
