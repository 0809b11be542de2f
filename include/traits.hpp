// traits.hpp -- the reference's compile-time objective traits
// (include/traits.hpp:16-71), under its header name so that objective code
// written for the reference (optimization_utils.hpp includes
// "../include/traits.hpp") finds them here: FnTraits (arity from a static
// `arity` member or a Functor<N> template; user code specialises it, e.g.
// LogLikelihood.h:77-82), the CallableWithArray / ZeusObjective concepts and
// PRNGType.  The names, template parameters and enumerators have to be the
// reference's for that code to compile unchanged.
#pragma once

#include <array>
#include <concepts>
#include <cstddef>
#include <type_traits>

namespace dual {
  struct DualNumber;
}

namespace zeus {

  template <typename...>
  using VoidT = void;

  template <typename F, typename = void>
  struct FnTraits {
    static constexpr std::size_t arity = 0;
  };
  template <typename F>
  struct FnTraits<F, VoidT<decltype(F::arity)>> {
    static constexpr std::size_t arity = F::arity;
  };
  template <template <std::size_t> class Functor, std::size_t N>
  struct FnTraits<Functor<N>> {
    static constexpr std::size_t arity = N;
  };

  template <typename F, typename T, std::size_t DIM>
  concept CallableWithArray = requires(F f, std::array<T, DIM> arr) {
    { f(arr) } -> std::convertible_to<T>;
  };
  template <typename F, std::size_t DIM>
  concept ZeusObjective = CallableWithArray<F, double, DIM> &&
                          CallableWithArray<F, dual::DualNumber, DIM>;

  enum class PRNGType { XORWOW, PHILOX, SOBOL };

} // namespace zeus
