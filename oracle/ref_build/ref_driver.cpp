// Host driver around the reference's own sequential BFGS kernel body
// (include/bfgs_sequential.cuh:16-234, bfgs::sequential::optimize), compiled
// for the CPU through ref_shim.h.  Each host thread plays one CUDA thread: it
// sets blockIdx.x = run index and calls optimize() as a plain function, with
// the start points injected through pso_array (the same entry the reference's
// own integration tests use, test/bfgs_tests.cu:605-622).
//
// Test infrastructure only (the pin for oracle/zeus_oracle.c and the timed CPU
// baseline).  The exported entry point has the same signature as the C
// restatement's zor_bfgs() so the two can be compared call for call.
#include "ref_shim.h"

// The reference's own include order (bfgs_sequential.cuh:5-9): bfgs_common.cuh
// relies on pso.cuh's `using namespace zeus`.
#include "duals.cuh"
#include "utils.cuh"
#include "pso.cuh"
#include "traits.hpp"
#include "bfgs_common.cuh"
#undef __global__
#define __global__ __host__
#include "bfgs_sequential.cuh"
#include "rosenbrock.hpp"
#include "rastrigin.hpp"
#include "ackley.hpp"
#include "gaussian.hpp"
#include "simulation/fitting/LogLikelihood.h"

#include <memory>
#include <omp.h>

thread_local zref_index3 zref_blockIdx{0, 0, 0};
thread_local zref_index3 zref_threadIdx{0, 0, 0};
thread_local zref_index3 zref_blockDim{1, 1, 1};

namespace {

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

  template <class F, std::size_t D>
  int
  run(const F& f, const double* starts, int n, double lower, double upper,
      int max_iter, int required, double tol, const Outputs& o, int nthreads)
  {
    util::BFGSContext ctx{0, 0};
    std::vector<double> dev_results(n > 0 ? n : 1);
    std::vector<zeus::Result<D>> res(n > 0 ? n : 1);
    std::vector<curandStateXORWOW_t> states(n > 0 ? n : 1);
    const bool traj = o.traj_x && o.traj_f && o.traj_g && o.traj_status;
    if (nthreads <= 0)
      nthreads = omp_get_max_threads();
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int i = 0; i < n; ++i) {
      zref_blockIdx.x = (unsigned)i;
      zref_threadIdx.x = 0;
      zref_blockDim.x = 1;
      if (traj) {
        bfgs::sequential::optimize<F, D, 128, true, curandStateXORWOW_t>(
          f, lower, upper, starts, util::NonNull{dev_results.data()},
          o.traj_x, o.traj_f, o.traj_g,
          reinterpret_cast<int8_t*>(o.traj_status), n, max_iter, required,
          tol, 0, util::NonNull{res.data()}, util::NonNull{states.data()},
          util::NonNull{&ctx});
      } else {
        bfgs::sequential::optimize<F, D, 128, false, curandStateXORWOW_t>(
          f, lower, upper, starts, util::NonNull{dev_results.data()}, nullptr,
          nullptr, nullptr, nullptr, n, max_iter, required, tol, 0,
          util::NonNull{res.data()}, util::NonNull{states.data()},
          util::NonNull{&ctx});
      }
    }
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

  template <std::size_t D>
  int
  gaussian(const double* C, const double* starts, int n, double lo, double hi,
           int max_iter, int req, double tol, const Outputs& o, int nt)
  {
    auto Ch = std::make_unique<std::array<std::array<double, D>, D>>();
    for (std::size_t i = 0; i < D; ++i)
      for (std::size_t j = 0; j < D; ++j)
        (*Ch)[i][j] = C[i * D + j];
    Gaussian<D> g(*Ch);
    return run<Gaussian<D>, D>(g, starts, n, lo, hi, max_iter, req, tol, o,
                               nt);
  }

} // namespace

/// f(x) = x^2, the 1-D quadratic of test/bfgs_tests.cu:55-62.
struct ZrefQuadratic1 {
  static constexpr std::size_t arity = 1;
  double
  operator()(const std::array<double, 1>& v) const
  {
    return v[0] * v[0];
  }
};

extern "C" {

/// Objective kinds shared with oracle/zeus_oracle.h.
enum { ZREF_ROSENBROCK = 0, ZREF_RASTRIGIN = 1, ZREF_ACKLEY = 2,
       ZREF_GAUSSIAN = 3, ZREF_POISSON_NLL = 4 };

/// Runs the reference's sequential BFGS for n injected starts (row-major,
/// starts[i*dim+d]).  Trajectory buffers use the reference layout
/// [iter][dim][run] / [iter][run] (bfgs_sequential.cuh:100-109) and must be
/// NaN/-1 prefilled by the caller.  Returns 0, or -1 for an (kind, dim) that
/// is not instantiated here.
int
zref_bfgs(int kind, int dim, const double* data, const int* idata, int ndata,
          const double* starts, int n, double lower, double upper,
          int max_iter, int required, double tol, double* fval, int* status,
          int* iter, double* gnorm, double* x_out, double* traj_x,
          double* traj_f, double* traj_g, signed char* traj_status,
          int nthreads)
{
  Outputs o{fval, status, iter, gnorm, x_out, traj_x, traj_f, traj_g,
            traj_status};
#define ZREF_CASE(KIND, D, OBJ)                                                \
  if (kind == KIND && dim == D)                                                \
    return run<OBJ, D>(OBJ{}, starts, n, lower, upper, max_iter, required,     \
                       tol, o, nthreads);
  ZREF_CASE(ZREF_ROSENBROCK, 2, util::Rosenbrock<2>)
  ZREF_CASE(ZREF_ROSENBROCK, 4, util::Rosenbrock<4>)
  ZREF_CASE(ZREF_ROSENBROCK, 8, util::Rosenbrock<8>)
  ZREF_CASE(ZREF_ROSENBROCK, 10, util::Rosenbrock<10>)
  ZREF_CASE(ZREF_ROSENBROCK, 16, util::Rosenbrock<16>)
  ZREF_CASE(ZREF_ROSENBROCK, 32, util::Rosenbrock<32>)
  ZREF_CASE(ZREF_ROSENBROCK, 64, util::Rosenbrock<64>)
  ZREF_CASE(ZREF_ROSENBROCK, 128, util::Rosenbrock<128>)
  ZREF_CASE(ZREF_RASTRIGIN, 2, util::Rastrigin<2>)
  ZREF_CASE(ZREF_RASTRIGIN, 10, util::Rastrigin<10>)
  ZREF_CASE(ZREF_RASTRIGIN, 16, util::Rastrigin<16>)
  ZREF_CASE(ZREF_ACKLEY, 2, util::Ackley<2>)
  ZREF_CASE(ZREF_ACKLEY, 10, util::Ackley<10>)
  ZREF_CASE(ZREF_ACKLEY, 30, util::Ackley<30>)
#undef ZREF_CASE
  if (kind == ZREF_GAUSSIAN) {
    if (dim == 2)
      return gaussian<2>(data, starts, n, lower, upper, max_iter, required,
                         tol, o, nthreads);
    if (dim == 8)
      return gaussian<8>(data, starts, n, lower, upper, max_iter, required,
                         tol, o, nthreads);
    if (dim == 32)
      return gaussian<32>(data, starts, n, lower, upper, max_iter, required,
                          tol, o, nthreads);
    if (dim == 150)
      return gaussian<150>(data, starts, n, lower, upper, max_iter, required,
                           tol, o, nthreads);
  }
  if (kind == ZREF_POISSON_NLL && dim == 4) {
    std::vector<int> counts(idata, idata + ndata);
    std::vector<double> centres(data, data + ndata);
    LogLikelihood ll(counts, centres);
    return run<LogLikelihood, 4>(ll, starts, n, lower, upper, max_iter,
                                 required, tol, o, nthreads);
  }
  return -1;
}

/// Reference line search (include/utils.cuh:376-412) on the 1-D quadratic
/// x^2 of test/bfgs_tests.cu:55-62, for the known-answer check alpha = 0.5.
double
zref_linesearch_quadratic(double f0, double x, double p, double g)
{
  return util::lineSearch<ZrefQuadratic1, 1>(f0, &x, &p, &g, ZrefQuadratic1{});
}

/// Reference O(D^4) BFGS update (include/utils.cuh:312-340) for dim <= 8.
int
zref_bfgs_update(int dim, double* H, const double* s, const double* y,
                 double sTy)
{
  switch (dim) {
    case 1: util::bfgsUpdate<1>(H, s, y, sTy); return 0;
    case 2: util::bfgsUpdate<2>(H, s, y, sTy); return 0;
    case 3: util::bfgsUpdate<3>(H, s, y, sTy); return 0;
    case 4: util::bfgsUpdate<4>(H, s, y, sTy); return 0;
    case 8: util::bfgsUpdate<8>(H, s, y, sTy); return 0;
    default: return -1;
  }
}

/// Reference digamma (src/duals.cu:10-39).
double
zref_digamma(double x)
{
  return dual::digamma(x);
}

/// Reference forward-mode gradient (include/duals.cuh:241-266) of the
/// built-in objectives at one point.  Returns f(x) and writes grad.
double
zref_value_grad(int kind, int dim, const double* x, double* grad)
{
#define ZREF_VG(KIND, D, OBJ)                                                  \
  if (kind == KIND && dim == D) {                                              \
    OBJ f;                                                                     \
    std::array<double, D> xa, ga;                                              \
    for (int i = 0; i < D; ++i)                                                \
      xa[i] = x[i];                                                            \
    dual::calculateGradientUsingAD(f, xa, ga);                                 \
    for (int i = 0; i < D; ++i)                                                \
      grad[i] = ga[i];                                                         \
    return f(xa);                                                              \
  }
  ZREF_VG(ZREF_ROSENBROCK, 2, util::Rosenbrock<2>)
  ZREF_VG(ZREF_ROSENBROCK, 4, util::Rosenbrock<4>)
  ZREF_VG(ZREF_ROSENBROCK, 8, util::Rosenbrock<8>)
  ZREF_VG(ZREF_ROSENBROCK, 10, util::Rosenbrock<10>)
  ZREF_VG(ZREF_ROSENBROCK, 16, util::Rosenbrock<16>)
  ZREF_VG(ZREF_ROSENBROCK, 32, util::Rosenbrock<32>)
  ZREF_VG(ZREF_ROSENBROCK, 64, util::Rosenbrock<64>)
  ZREF_VG(ZREF_ROSENBROCK, 128, util::Rosenbrock<128>)
  ZREF_VG(ZREF_ROSENBROCK, 256, util::Rosenbrock<256>)
  ZREF_VG(ZREF_RASTRIGIN, 2, util::Rastrigin<2>)
  ZREF_VG(ZREF_RASTRIGIN, 10, util::Rastrigin<10>)
  ZREF_VG(ZREF_RASTRIGIN, 16, util::Rastrigin<16>)
  ZREF_VG(ZREF_ACKLEY, 2, util::Ackley<2>)
  ZREF_VG(ZREF_ACKLEY, 10, util::Ackley<10>)
  ZREF_VG(ZREF_ACKLEY, 30, util::Ackley<30>)
#undef ZREF_VG
  return std::numeric_limits<double>::quiet_NaN();
}

/// zref_value_grad for the objectives that carry data: the Gaussian
/// (examples/gaussian.hpp, C row-major dim*dim) and the Poisson NLL
/// (simulation/fitting/LogLikelihood.h, ndata centres and counts).
double
zref_value_grad_data(int kind, int dim, const double* data, const int* idata,
                     int ndata, const double* x, double* grad)
{
  const auto eval = [&](const auto& f, auto dimc) -> double {
    constexpr std::size_t D = decltype(dimc)::value;
    std::array<double, D> xa, ga;
    for (std::size_t i = 0; i < D; ++i)
      xa[i] = x[i];
    dual::calculateGradientUsingAD(f, xa, ga);
    for (std::size_t i = 0; i < D; ++i)
      grad[i] = ga[i];
    return f(xa);
  };
  const auto gaussian_vg = [&](auto dimc) -> double {
    constexpr std::size_t D = decltype(dimc)::value;
    auto Ch = std::make_unique<std::array<std::array<double, D>, D>>();
    for (std::size_t i = 0; i < D; ++i)
      for (std::size_t j = 0; j < D; ++j)
        (*Ch)[i][j] = data[i * D + j];
    Gaussian<D> g(*Ch);
    return eval(g, dimc);
  };
  if (kind == ZREF_GAUSSIAN) {
    if (dim == 2)
      return gaussian_vg(std::integral_constant<std::size_t, 2>{});
    if (dim == 8)
      return gaussian_vg(std::integral_constant<std::size_t, 8>{});
    if (dim == 32)
      return gaussian_vg(std::integral_constant<std::size_t, 32>{});
    if (dim == 150)
      return gaussian_vg(std::integral_constant<std::size_t, 150>{});
  }
  if (kind == ZREF_POISSON_NLL && dim == 4) {
    std::vector<int> counts(idata, idata + ndata);
    std::vector<double> centres(data, data + ndata);
    LogLikelihood ll(counts, centres);
    return eval(ll, std::integral_constant<std::size_t, 4>{});
  }
  return std::numeric_limits<double>::quiet_NaN();
}

} // extern "C"
