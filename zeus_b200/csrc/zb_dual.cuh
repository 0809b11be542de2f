// Forward-mode dual numbers for objective callables.
//
// User objectives written for the reference are templates over
// T in {double, dual::DualNumber} (traits.hpp:38-64) and call dual::cos,
// dual::exp, ... through ADL, so the type keeps the reference's name,
// members (real, dual) and operator set (duals.cuh:14-239).  Each operation
// applies the textbook derivative rule in the same arithmetic order as the
// reference, which the exact mode relies on for bit-identical gradients.
#pragma once

#include <cmath>
#include <limits>

namespace dual {

  struct DualNumber {
    double real;
    double dual;

    __host__ __device__ constexpr DualNumber(double r = 0.0, double d = 0.0)
      : real(r), dual(d)
    {}
    __host__ __device__ constexpr DualNumber
    operator-() const
    {
      return DualNumber(-real, -dual);
    }
    __host__ __device__ constexpr DualNumber&
    operator+=(const DualNumber& o)
    {
      real += o.real;
      dual += o.dual;
      return *this;
    }
    __host__ __device__ constexpr DualNumber&
    operator-=(const DualNumber& o)
    {
      real -= o.real;
      dual -= o.dual;
      return *this;
    }
    __host__ __device__ constexpr DualNumber
    operator+(const DualNumber& o) const
    {
      return DualNumber(real + o.real, dual + o.dual);
    }
    __host__ __device__ constexpr DualNumber
    operator-(const DualNumber& o) const
    {
      return DualNumber(real - o.real, dual - o.dual);
    }
    // (a + a'e)(b + b'e) = ab + (a'b + ab')e
    __host__ __device__ constexpr DualNumber
    operator*(const DualNumber& o) const
    {
      return DualNumber(real * o.real, dual * o.real + real * o.dual);
    }
    // quotient rule, denominator b^2
    __host__ __device__ constexpr DualNumber
    operator/(const DualNumber& o) const
    {
      const double den = o.real * o.real;
      return DualNumber(real / o.real, (dual * o.real - real * o.dual) / den);
    }
    __host__ __device__ friend constexpr DualNumber
    operator-(double l, const DualNumber& r)
    {
      return DualNumber(l - r.real, -r.dual);
    }
    __host__ __device__ friend constexpr DualNumber
    operator*(double l, const DualNumber& r)
    {
      return DualNumber(l * r.real, l * r.dual);
    }
  };

  __host__ __device__ constexpr inline bool
  operator==(const DualNumber& a, const DualNumber& b)
  {
    return a.real == b.real && a.dual == b.dual;
  }
  __host__ __device__ constexpr inline bool
  operator!=(const DualNumber& a, const DualNumber& b)
  {
    return !(a == b);
  }

  // |x|: the derivative is undefined at 0 and reported as NaN.
  __host__ __device__ constexpr inline DualNumber
  abs(const DualNumber& a)
  {
    if (a.real == 0.0)
      return DualNumber(0.0, std::numeric_limits<double>::quiet_NaN());
    return (a.real < 0.0) ? DualNumber(-a.real, -a.dual) : a;
  }
  __host__ __device__ inline DualNumber
  sin(const DualNumber& x)
  {
    return DualNumber(::sin(x.real), x.dual * ::cos(x.real));
  }
  __host__ __device__ inline DualNumber
  cos(const DualNumber& x)
  {
    return DualNumber(::cos(x.real), -x.dual * ::sin(x.real));
  }
  __host__ __device__ inline DualNumber
  exp(const DualNumber& x)
  {
    const double e = ::exp(x.real);
    return DualNumber(e, x.dual * e);
  }
  __host__ __device__ inline DualNumber
  sqrt(const DualNumber& x)
  {
    const double r = ::sqrt(x.real);
    return DualNumber(r, x.dual / (2.0 * r));
  }
  __host__ __device__ inline DualNumber
  atan2(const DualNumber& y, const DualNumber& x)
  {
    const double den = x.real * x.real + y.real * y.real;
    return DualNumber(::atan2(y.real, x.real),
                      (x.real * y.dual - y.real * x.dual) / den);
  }
  __host__ __device__ inline DualNumber
  log(const DualNumber& x)
  {
    return DualNumber(::log(x.real), x.dual / x.real);
  }
  // b^e with both varying: d(b^e) = b^e (e' ln b + e b'/b)
  __host__ __device__ inline DualNumber
  pow(const DualNumber& b, const DualNumber& e)
  {
    const double br = b.real, er = e.real;
    const double pr = ::pow(br, er);
    return DualNumber(pr, pr * (e.dual * ::log(br) + er * b.dual / br));
  }
  // b^e with constant e; at b = 0 the derivative uses e b^(e-1) directly.
  __host__ __device__ inline DualNumber
  pow(const DualNumber& b, double e)
  {
    const double br = b.real;
    const double pr = ::pow(br, e);
    if (br == 0.0)
      return DualNumber(pr, e * ::pow(br, e - 1.0) * b.dual);
    return DualNumber(pr, e * pr / br * b.dual);
  }
  __host__ __device__ constexpr inline double
  pi()
  {
    return 3.14159265358979323846;
  }

  // psi(x) = d/dx ln Gamma(x): poles at 0, -1, -2, ...; reflection
  // psi(x) = psi(1-x) - pi cot(pi x) below 1/2; upward recurrence
  // psi(x) = psi(x+1) - 1/x to x >= 8; then the asymptotic (Stirling)
  // series ln x - 1/(2x) - sum_k B_2k / (2k x^2k) through B_12.
  __host__ __device__ inline double
  digamma(double x)
  {
    if (x <= 0.0 && x == ::floor(x))
      return std::numeric_limits<double>::infinity();
    double refl = 0.0;
    if (x < 0.5) {
      refl = -pi() / ::tan(pi() * x);
      x = 1.0 - x;
    }
    double acc = 0.0;
    while (x < 8.0) {
      acc -= 1.0 / x;
      x += 1.0;
    }
    const double inv = 1.0 / x;
    const double z = inv * inv;
    const double series =
      z * (-1.0 / 12.0 +
           z * (1.0 / 120.0 +
                z * (-1.0 / 252.0 +
                     z * (1.0 / 240.0 +
                          z * (-1.0 / 132.0 + z * (691.0 / 32760.0))))));
    const double v = acc + ::log(x) - 0.5 * inv + series;
    return refl == 0.0 ? v : v + refl;
  }

  __host__ __device__ inline DualNumber
  lgamma(const DualNumber& x)
  {
    return DualNumber(::lgamma(x.real), x.dual * digamma(x.real));
  }

} // namespace dual
