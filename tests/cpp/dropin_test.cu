// Uses the C++ drop-in (include/zeus.cuh) the way code written for the
// reference does: zeus::Zeus on user functors templated over
// T in {double, dual::DualNumber}, objective data in Matrix<T>.
// Prints one JSON object per case; tests/test_gpu_dropin.py checks them.
#include <array>
#include <cmath>
#include <cstdio>

#include "zeus.cuh"

// written like examples/rosenbrock.hpp: static arity + templated operator()
struct MyRosenbrock {
  static constexpr std::size_t arity = 2;
  template <class T>
  __host__ __device__ T
  operator()(const std::array<T, 2>& x) const
  {
    T a = T(1.0) - x[0];
    T b = x[1] - x[0] * x[0];
    return a * a + T(100.0) * b * b;
  }
};

// dimension from a Functor<N> template (traits.hpp:24-34)
template <std::size_t N>
struct Sphere {
  template <class T>
  __host__ __device__ T
  operator()(const std::array<T, N>& x) const
  {
    T s = T(0.0);
    for (std::size_t i = 0; i < N; ++i)
      s = s + (x[i] - T(0.5)) * (x[i] - T(0.5));
    return s;
  }
};

// objective data in a Matrix, like examples/gaussian.hpp
template <std::size_t N>
class MyGaussian {
  Matrix<double> C;

public:
  static constexpr std::size_t arity = N;
  explicit MyGaussian(const std::array<double, N * N>& c) : C(N, N) { C.set(c); }
  template <class T>
  __host__ __device__ T
  operator()(const std::array<T, N>& x) const
  {
    const double* Cp = C.data();
    T q = T(0);
    for (std::size_t i = 0; i < N; ++i)
      for (std::size_t j = 0; j < N; ++j)
        q += x[i] * T(Cp[i * N + j]) * x[j];
    return T(0.5) * q;
  }
};

// with a hand-written gradient: used instead of the dual passes
struct AdjointQuad {
  static constexpr std::size_t arity = 4;
  template <class T>
  __host__ __device__ T
  operator()(const std::array<T, 4>& x) const
  {
    T s = T(0.0);
    for (int i = 0; i < 4; ++i)
      s = s + T(double(i + 1)) * x[i] * x[i];
    return s;
  }
  __host__ __device__ double
  adjoint(const double* x, double* g) const
  {
    double s = 0.0;
    for (int i = 0; i < 4; ++i) {
      s += (i + 1) * x[i] * x[i];
      g[i] = 2.0 * (i + 1) * x[i];
    }
    return s;
  }
};

template <std::size_t D>
void
emit(const char* name, const zeus::Result<D>& r)
{
  std::printf("{\"case\": \"%s\", \"status\": %d, \"fval\": %.17g, \"gnorm\": %.17g, "
              "\"iter\": %d, \"idx\": %d, \"claimed\": %d, \"stopped\": %d, "
              "\"surrendered\": %d, \"ad\": [%.17g, %.17g, %.17g, %.17g, %.17g, %.17g], "
              "\"bfgs\": [%.17g, %.17g, %.17g, %.17g, %.17g, %.17g], \"x\": [",
              name, r.status, r.fval, r.gradientNorm, r.iter, r.idx, r.c.claimed,
              r.c.stopped, r.c.surrendered, r.ad.ms_per_call, r.ad.calls_per_thread_mean,
              r.ad.fraction_of_kernel, r.ad.block95, r.ad.serialized,
              r.ad.fraction_of_thread, r.bfgs.ms_per_call, r.bfgs.calls_per_thread_mean,
              r.bfgs.fraction_of_kernel, r.bfgs.block95, r.bfgs.serialized,
              r.bfgs.fraction_of_thread);
  for (std::size_t i = 0; i < D; ++i)
    std::printf("%s%.17g", i ? ", " : "", r.coordinates[i]);
  std::printf("]}\n");
}

int
main(int argc, char** argv)
{
  emit("rosenbrock", zeus::Zeus(MyRosenbrock{}, -5.0, 5.0, 1024, 10000, 10, 100,
                                "rosenbrock", 1e-8, 42, 0));
  emit("sphere16", zeus::Zeus(Sphere<16>{}, -5.0, 5.0, 256, 2000, 5, 1000, "sphere",
                              1e-8, 7, 0));
  std::array<double, 64> c{};
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j)
      c[i * 8 + j] = (i == j) ? 4.5 : 0.5;
  MyGaussian<8> g(c);
  emit("gaussian8", zeus::Zeus(g, -5.0, 5.0, 512, 1000, 10, 1000, "gaussian", 1e-8, 3, 0));
  emit("adjoint4", zeus::Zeus(AdjointQuad{}, -3.0, 3.0, 300, 500, -1, 1000, "quad", 1e-8,
                              5, 0));
  emit("sphere40", zeus::Zeus(Sphere<40>{}, -5.0, 5.0, 64, 2000, 0, 1000, "sphere",
                              1e-8, 9, 0));
  emit("empty", zeus::Zeus(MyRosenbrock{}, -5.0, 5.0, 0, 100, 10, 10, "rosenbrock", 1e-8,
                           42, 0));
  // past D = 160: the CTA layout keeps H in global memory
  emit("sphere200", zeus::Zeus(Sphere<200>{}, -5.0, 5.0, 40, 500, 0, 1000, "sphere",
                               1e-8, 13, 0));
  // Sobol' initial swarm
  emit("sphere16_sobol", zeus::Zeus(Sphere<16>{}, -5.0, 5.0, 256, 2000, 5, 1000,
                                    "sphere", 1e-8, 7, 0, true, zeus::PRNGType::SOBOL));
  if (argc > 1) // trajectory file: exact mode, every iteration recorded
    emit("traj", zeus::Zeus(MyRosenbrock{}, -5.0, 5.0, 6, 40, -1, 1000, "rosenbrock",
                            1e-8, 42, 0, true, zeus::PRNGType::XORWOW, argv[1]));
  if (argc > 2) // the same with Sobol' starts (step 0 of each run is its start)
    emit("traj_sobol", zeus::Zeus(MyRosenbrock{}, -5.0, 5.0, 6, 40, -1, 1000,
                                  "rosenbrock", 1e-8, 42, 0, true, zeus::PRNGType::SOBOL,
                                  argv[2]));
  return 0;
}
