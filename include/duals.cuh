// duals.cuh -- forward-mode dual numbers under the reference's header name
// (include/duals.cuh): objective headers written for the reference
// (examples/rosenbrock.hpp:2, rastrigin.hpp:2, ackley.hpp:2) include
// "duals.cuh" and call dual::DualNumber, dual::cos, dual::exp, ... through
// ADL.  The type and its math come from the library's zb_dual.cuh; this
// header adds the reference's stand-alone gradient helper.
#pragma once

#include <array>
#include <cstddef>

#include "traits.hpp"
#include "zb_dual.cuh"

namespace dual {

  // The reference's dual::calculateGradientUsingAD (duals.cuh:241-266): one
  // forward pass per coordinate, seeding that coordinate's derivative.
  template <typename Function, std::size_t DIM>
    requires zeus::ZeusObjective<Function, DIM>
  __host__ __device__ void
  calculateGradientUsingAD(Function const& f, const std::array<double, DIM>& x_arr,
                           std::array<double, DIM>& grad)
  {
    std::array<DualNumber, DIM> xd;
    for (std::size_t i = 0; i < DIM; ++i)
      xd[i] = DualNumber(x_arr[i], 0.0);
    for (std::size_t i = 0; i < DIM; ++i) {
      xd[i].dual = 1.0;
      grad[i] = f(xd).dual;
      xd[i].dual = 0.0;
    }
  }

} // namespace dual
