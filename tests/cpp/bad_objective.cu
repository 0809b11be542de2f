// Must NOT compile: the objective has no DualNumber overload, so it fails the
// ZeusObjective concept (the reference's test/bad_objectives.cu).
#include <array>

#include "zeus.cuh"

struct DoubleOnly {
  static constexpr std::size_t arity = 2;
  __host__ __device__ double
  operator()(const std::array<double, 2>& x) const
  {
    return x[0] * x[0] + x[1] * x[1];
  }
};

int
main()
{
  auto r = zeus::Zeus(DoubleOnly{}, -1.0, 1.0, 8, 10, 1, 1, "bad", 1e-8, 1, 0);
  return r.status;
}
