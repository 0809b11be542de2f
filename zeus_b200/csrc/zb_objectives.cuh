// Built-in objectives: the reference's benchmark functions
// (examples/rosenbrock.hpp:6-41, rastrigin.hpp:6-38, ackley.hpp:10-50,
// gaussian.hpp:8-34, simulation/fitting/LogLikelihood.h:12-82).
//
// Each objective has three entry points:
//  * operator()(std::array<T, D>) for T = double and dual::DualNumber, with
//    the reference's expression order (the `if constexpr` branches exist
//    because the reference writes its double and dual bodies differently);
//    exact mode and dual gradients use only this;
//  * value(x): the same function in FMA-friendly form (fast mode);
//  * adjoint(x, g): value and hand-derived reverse-mode gradient in one
//    sweep (fast mode, ZEUS_GRAD_ADJOINT).
// Objective data (Gaussian C, NLL bins) is held as device pointers: the
// functor is trivially copyable, so it can sit in kernel parameters, CUDA
// graphs and persistent kernels without the host-side deep copies the
// reference's Matrix members imply (matrix.hpp:65-89).
#pragma once

#include <array>
#include <cmath>
#include <cstddef>
#include <type_traits>

#include "zb_dual.cuh"

namespace zeus {

  inline constexpr double kTwoPi = 2.0 * 3.14159265358979323846;

  namespace detail {
    // Member `grp.rank()` of a cooperating group visits i = rank, rank +
    // size, ... < N.  For a group whose size is a compile-time constant (a
    // tile) the loop is unrolled, so its loads issue together instead of
    // one iteration's loads waiting on the previous iteration's arithmetic.
    template <int N, class G, class Fn>
    __device__ __forceinline__ void
    coop_for(const G& grp, Fn&& fn)
    {
      if constexpr (requires { std::integral_constant<int, G::size()>{}; }) {
        constexpr int S = G::size();
#pragma unroll
        for (int k = 0; k < (N + S - 1) / S; ++k) {
          const int i = grp.rank() + k * S;
          if (i < N)
            fn(i);
        }
      } else {
        for (int i = grp.rank(); i < N; i += grp.size())
          fn(i);
      }
    }
  } // namespace detail

  template <std::size_t D>
  struct Rosenbrock {
    static constexpr std::size_t arity = D;
    static constexpr int kind = 0;

    template <class T>
    __host__ __device__ T
    operator()(const std::array<T, D>& x) const
    {
      if constexpr (std::is_same_v<T, double>) {
        double sum = 0.0;
        for (std::size_t i = 0; i + 1 < D; ++i) {
          const double t1 = 1.0 - x[i];
          const double t2 = x[i + 1] - x[i] * x[i];
          sum += t1 * t1 + 100.0 * t2 * t2;
        }
        return sum;
      } else {
        T sum(0.0, 0.0);
        for (std::size_t i = 0; i + 1 < D; ++i) {
          const T t1 = T(1.0, 0.0) - x[i];
          const T t2 = x[i + 1] - x[i] * x[i];
          sum = sum + t1 * t1 + T(100.0, 0.0) * t2 * t2;
        }
        return sum;
      }
    }

    __host__ __device__ double
    value(const double* x) const
    {
      double sum = 0.0;
#pragma unroll 4
      for (std::size_t i = 0; i + 1 < D; ++i) {
        const double t1 = 1.0 - x[i];
        const double t2 = fma(-x[i], x[i], x[i + 1]);
        sum = fma(100.0 * t2, t2, fma(t1, t1, sum));
      }
      return sum;
    }

    // f(x + a p) by one thread from interleaved {x_i, p_i} (16-byte loads);
    // coordinate i of the trial point is fma(a, p_i, x_i), the same bits as
    // a materialised trial point
    // (four partial sums: the chain of dependent FMAs is a quarter as long)
    __device__ double
    value_line(const double2* xp, double a) const
    {
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      double xi = fma(a, xp[0].y, xp[0].x);
#pragma unroll 8
      for (std::size_t i = 0; i + 1 < D; ++i) {
        const double2 q = xp[i + 1];
        const double xj = fma(a, q.y, q.x);
        const double t1 = 1.0 - xi;
        const double t2 = fma(-xi, xi, xj);
        acc[i & 3] = fma(100.0 * t2, t2, fma(t1, t1, acc[i & 3]));
        xi = xj;
      }
      return (acc[0] + acc[1]) + (acc[2] + acc[3]);
    }

    // d/dx_i: -2(1-x_i) - 400 x_i (x_{i+1}-x_i^2) + 200 (x_i - x_{i-1}^2)
    __host__ __device__ double
    adjoint(const double* x, double* g) const
    {
      double sum = 0.0, carry = 0.0;
#pragma unroll 4
      for (std::size_t i = 0; i + 1 < D; ++i) {
        const double t1 = 1.0 - x[i];
        const double t2 = fma(-x[i], x[i], x[i + 1]);
        sum = fma(100.0 * t2, t2, fma(t1, t1, sum));
        g[i] = carry - 2.0 * t1 - 400.0 * x[i] * t2;
        carry = 200.0 * t2;
      }
      g[D - 1] = carry;
      return sum;
    }

    // Cooperative forms: member k takes terms / coordinates k, k+size, ...
    // (for a group of compile-time size, alternating between two partial
    // sums: the chain of dependent FMAs is half as long)
    template <class G>
    __device__ double
    value_coop(const G& grp, const double* x) const
    {
      if constexpr (requires { std::integral_constant<int, G::size()>{}; }) {
        constexpr int S = G::size();
        double acc[2] = {0.0, 0.0};
#pragma unroll
        for (int k = 0; k < ((int)D - 1 + S - 1) / S; ++k) {
          const int i = grp.rank() + k * S;
          if (i < (int)D - 1) {
            const double t1 = 1.0 - x[i];
            const double t2 = fma(-x[i], x[i], x[i + 1]);
            acc[k & 1] = fma(100.0 * t2, t2, fma(t1, t1, acc[k & 1]));
          }
        }
        return grp.sum(acc[0] + acc[1]);
      } else {
        double part = 0.0;
        detail::coop_for<(int)D - 1>(grp, [&](int i) {
          const double t1 = 1.0 - x[i];
          const double t2 = fma(-x[i], x[i], x[i + 1]);
          part = fma(100.0 * t2, t2, fma(t1, t1, part));
        });
        return grp.sum(part);
      }
    }
    template <class G>
    __device__ double
    adjoint_coop(const G& grp, const double* x, double* g) const
    {
      double part = 0.0;
      detail::coop_for<(int)D>(grp, [&](int i) {
        double gi = 0.0;
        if (i + 1 < (int)D) {
          const double t1 = 1.0 - x[i];
          const double t2 = fma(-x[i], x[i], x[i + 1]);
          part = fma(100.0 * t2, t2, fma(t1, t1, part));
          gi = -2.0 * t1 - 400.0 * x[i] * t2;
        }
        if (i > 0)
          gi = fma(200.0, fma(-x[i - 1], x[i - 1], x[i]), gi);
        g[i] = gi;
      });
      return grp.sum(part);
    }
    // the gradient alone (no reduction): each member writes its coordinates
    template <class G>
    __device__ void
    gradient_coop(const G& grp, const double* x, double* g) const
    {
      detail::coop_for<(int)D>(grp, [&](int i) {
        double gi = 0.0;
        if (i + 1 < (int)D) {
          const double t1 = 1.0 - x[i];
          const double t2 = fma(-x[i], x[i], x[i + 1]);
          gi = -2.0 * t1 - 400.0 * x[i] * t2;
        }
        if (i > 0)
          gi = fma(200.0, fma(-x[i - 1], x[i - 1], x[i]), gi);
        g[i] = gi;
      });
    }

    // Line forms: coordinate i of x + a p is fma(a, p_i, x_i), read from
    // {x_i, p_i} pairs stored at slot (i % R) * 32 + i / R (D = 32 R; R = 1
    // is natural order), so trial points need not be stored.  Member m of
    // an S-lane group takes the terms whose first coordinate sits at slots
    // m, m + S, ...: consecutive members read consecutive slots for both of
    // a term's coordinates.  Two accumulators, as in value_coop.
    template <int S, int R>
    __device__ __forceinline__ double
    value_line_part(const double2* xp, double a, int m) const
    {
      static_assert((int)D == 32 * R, "one slot per lane and row");
      double acc[2] = {0.0, 0.0};
#pragma unroll
      for (int k = 0; k < ((int)D + S - 1) / S; ++k) {
        const int p = m + k * S;
        const int i = (p % 32) * R + p / 32;
        if (p < (int)D && i < (int)D - 1) {
          const int pn = R == 1 ? p + 1 : p / 32 < R - 1 ? p + 32 : p % 32 + 1;
          const double2 u = xp[p], w = xp[pn];
          const double xi = fma(a, u.y, u.x), xj = fma(a, w.y, w.x);
          const double t1 = 1.0 - xi;
          const double t2 = fma(-xi, xi, xj);
          acc[k & 1] = fma(100.0 * t2, t2, fma(t1, t1, acc[k & 1]));
        }
      }
      return acc[0] + acc[1];
    }
    // d/dx_i at x + a p, same storage (explicit FMAs: every call site
    // rounds alike)
    template <int R>
    __device__ __forceinline__ double
    gradient_line_entry(const double2* xp, double a, int i) const
    {
      const auto slot = [](int j) { return (j % R) * 32 + j / R; };
      const double2 c = xp[slot(i)];
      const double xi = fma(a, c.y, c.x);
      double gi = 0.0;
      if (i + 1 < (int)D) {
        const double2 n = xp[slot(i + 1)];
        const double t1 = 1.0 - xi;
        const double t2 = fma(-xi, xi, fma(a, n.y, n.x));
        gi = fma(-400.0 * xi, t2, -2.0 * t1);
      }
      if (i > 0) {
        const double2 q = xp[slot(i - 1)];
        const double xh = fma(a, q.y, q.x);
        gi = fma(200.0, fma(-xh, xh, xi), gi);
      }
      return gi;
    }
  };

  template <std::size_t D>
  struct Rastrigin {
    static constexpr std::size_t arity = D;
    static constexpr int kind = 1;

    template <class T>
    __host__ __device__ T
    operator()(const std::array<T, D>& x) const
    {
      if constexpr (std::is_same_v<T, double>) {
        double sum = 10.0 * D;
        for (std::size_t i = 0; i < D; ++i)
          sum += x[i] * x[i] - 10.0 * ::cos(kTwoPi * x[i]);
        return sum;
      } else {
        T sum(10.0 * D, 0.0);
        for (std::size_t i = 0; i < D; ++i)
          sum = sum + (x[i] * x[i] -
                       T(10.0, 0.0) * dual::cos(x[i] * T(kTwoPi, 0.0)));
        return sum;
      }
    }

    __device__ double
    value_line(const double2* xp, double a) const
    {
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
      for (std::size_t i = 0; i < D; ++i) {
        const double2 q = xp[i];
        const double xi = fma(a, q.y, q.x);
        acc[i & 3] += fma(xi, xi, -10.0 * ::cospi(2.0 * xi));
      }
      return 10.0 * D + ((acc[0] + acc[1]) + (acc[2] + acc[3]));
    }

    __host__ __device__ double
    value(const double* x) const
    {
      double sum = 10.0 * D;
      for (std::size_t i = 0; i < D; ++i)
        sum += fma(x[i], x[i], -10.0 * ::cospi(2.0 * x[i]));
      return sum;
    }

    // d/dx_i: 2 x_i + 20 pi sin(2 pi x_i)
    __host__ __device__ double
    adjoint(const double* x, double* g) const
    {
      double sum = 10.0 * D;
      for (std::size_t i = 0; i < D; ++i) {
        double s, c;
        ::sincospi(2.0 * x[i], &s, &c);
        sum += fma(x[i], x[i], -10.0 * c);
        g[i] = fma(10.0 * kTwoPi, s, 2.0 * x[i]);
      }
      return sum;
    }

    template <class G>
    __device__ double
    value_coop(const G& grp, const double* x) const
    {
      double part = 0.0;
      detail::coop_for<(int)D>(grp, [&](int i) {
        part += fma(x[i], x[i], -10.0 * ::cospi(2.0 * x[i]));
      });
      return 10.0 * D + grp.sum(part);
    }
    template <class G>
    __device__ double
    adjoint_coop(const G& grp, const double* x, double* g) const
    {
      double part = 0.0;
      detail::coop_for<(int)D>(grp, [&](int i) {
        double s, c;
        ::sincospi(2.0 * x[i], &s, &c);
        part += fma(x[i], x[i], -10.0 * c);
        g[i] = fma(10.0 * kTwoPi, s, 2.0 * x[i]);
      });
      return 10.0 * D + grp.sum(part);
    }
    template <class G>
    __device__ void
    gradient_coop(const G& grp, const double* x, double* g) const
    {
      detail::coop_for<(int)D>(grp, [&](int i) {
        double s, c;
        ::sincospi(2.0 * x[i], &s, &c);
        g[i] = fma(10.0 * kTwoPi, s, 2.0 * x[i]);
      });
    }
  };

  template <std::size_t D>
  struct Ackley {
    static constexpr std::size_t arity = D;
    static constexpr int kind = 2;

    template <class T>
    __host__ __device__ T
    operator()(const std::array<T, D>& x) const
    {
      if constexpr (std::is_same_v<T, double>) {
        double sum_sq = 0.0, sum_cos = 0.0;
        for (std::size_t i = 0; i < D; ++i) {
          sum_sq += x[i] * x[i];
          sum_cos += ::cos(kTwoPi * x[i]);
        }
        const double term1 = -20.0 * ::exp(-0.2 * ::sqrt(sum_sq / D));
        const double term2 = -::exp(sum_cos / D);
        return term1 + term2 + 20.0 + ::exp(1.0);
      } else {
        T sum_sq = 0.0, sum_cos = 0.0;
        for (std::size_t i = 0; i < D; ++i) {
          sum_sq += dual::pow(x[i], 2.0);
          sum_cos += dual::cos(kTwoPi * x[i]);
        }
        const T term1 =
          T(-20.0) * dual::exp(-0.2 * dual::sqrt(sum_sq / T(double(D))));
        const T term2 = T(0.0) - dual::exp(sum_cos / T(double(D)));
        return term1 + term2 + T(20.0) + dual::exp(T(1.0));
      }
    }

    __device__ double
    value_line(const double2* xp, double a) const
    {
      double s2[2] = {0.0, 0.0}, c2[2] = {0.0, 0.0};
#pragma unroll 8
      for (std::size_t i = 0; i < D; ++i) {
        const double2 q = xp[i];
        const double xi = fma(a, q.y, q.x);
        s2[i & 1] = fma(xi, xi, s2[i & 1]);
        c2[i & 1] += ::cospi(2.0 * xi);
      }
      const double ss = s2[0] + s2[1], sc = c2[0] + c2[1];
      constexpr double inv = 1.0 / double(D);
      return -20.0 * ::exp(-0.2 * ::sqrt(ss * inv)) - ::exp(sc * inv) + 20.0 +
             2.718281828459045;
    }

    __host__ __device__ double
    value(const double* x) const
    {
      double ss = 0.0, sc = 0.0;
      for (std::size_t i = 0; i < D; ++i) {
        ss = fma(x[i], x[i], ss);
        sc += ::cospi(2.0 * x[i]);
      }
      constexpr double inv = 1.0 / double(D);
      return -20.0 * ::exp(-0.2 * ::sqrt(ss * inv)) - ::exp(sc * inv) + 20.0 +
             2.718281828459045;
    }

    // d/dx_i: 4 e^{-0.2 r} x_i / (D r) + (2 pi / D) e^{C/D} sin(2 pi x_i),
    // r = sqrt(sum x^2 / D); NaN at r = 0 like the dual form.
    __host__ __device__ double
    adjoint(const double* x, double* g) const
    {
      double ss = 0.0, sc = 0.0;
      for (std::size_t i = 0; i < D; ++i) {
        double s, c;
        ::sincospi(2.0 * x[i], &s, &c);
        ss = fma(x[i], x[i], ss);
        sc += c;
        g[i] = s;
      }
      constexpr double inv = 1.0 / double(D);
      const double r = ::sqrt(ss * inv);
      const double e1 = ::exp(-0.2 * r), e2 = ::exp(sc * inv);
      const double a = 4.0 * e1 * inv / r, b = kTwoPi * e2 * inv;
      for (std::size_t i = 0; i < D; ++i)
        g[i] = fma(a, x[i], b * g[i]);
      return -20.0 * e1 - e2 + 20.0 + 2.718281828459045;
    }

    template <class G>
    __device__ double
    value_coop(const G& grp, const double* x) const
    {
      double v[2] = {0.0, 0.0};
      detail::coop_for<(int)D>(grp, [&](int i) {
        v[0] = fma(x[i], x[i], v[0]);
        v[1] += ::cospi(2.0 * x[i]);
      });
      grp.template sum<2>(v);
      constexpr double inv = 1.0 / double(D);
      return -20.0 * ::exp(-0.2 * ::sqrt(v[0] * inv)) - ::exp(v[1] * inv) + 20.0 +
             2.718281828459045;
    }
    template <class G>
    __device__ double
    adjoint_coop(const G& grp, const double* x, double* g) const
    {
      double v[2] = {0.0, 0.0};
      detail::coop_for<(int)D>(grp, [&](int i) {
        double s, c;
        ::sincospi(2.0 * x[i], &s, &c);
        v[0] = fma(x[i], x[i], v[0]);
        v[1] += c;
        g[i] = s; // the same member finishes g[i] below
      });
      grp.template sum<2>(v);
      constexpr double inv = 1.0 / double(D);
      const double r = ::sqrt(v[0] * inv);
      const double e1 = ::exp(-0.2 * r), e2 = ::exp(v[1] * inv);
      const double a = 4.0 * e1 * inv / r, b = kTwoPi * e2 * inv;
      detail::coop_for<(int)D>(grp, [&](int i) { g[i] = fma(a, x[i], b * g[i]); });
      return -20.0 * e1 - e2 + 20.0 + 2.718281828459045;
    }
  };

  // 0.5 x^T C x with C a dense D x D row-major device matrix.
  template <std::size_t D>
  struct Gaussian {
    static constexpr std::size_t arity = D;
    static constexpr int kind = 3;
    const double* C = nullptr; // device pointer, D*D
    bool symmetric = true;     // checked on the host when built from data

    template <class T>
    __host__ __device__ T
    operator()(const std::array<T, D>& x) const
    {
      const double* Cp = C;
      T q = T(0);
      for (std::size_t i = 0; i < D; ++i)
        for (std::size_t j = 0; j < D; ++j)
          q += x[i] * T(Cp[i * D + j]) * x[j];
      return T(0.5) * q;
    }

    __host__ __device__ double
    value(const double* x) const
    {
      double q = 0.0;
      for (std::size_t i = 0; i < D; ++i) {
        double r = 0.0;
        for (std::size_t j = 0; j < D; ++j)
          r = fma(C[i * D + j], x[j], r);
        q = fma(x[i], r, q);
      }
      return 0.5 * q;
    }

    // grad = (C + C^T) x / 2 (= C x when C is symmetric)
    __host__ __device__ double
    adjoint(const double* x, double* g) const
    {
      double q = 0.0;
      for (std::size_t i = 0; i < D; ++i) {
        double r = 0.0;
        for (std::size_t j = 0; j < D; ++j)
          r = fma(C[i * D + j], x[j], r);
        g[i] = r;
        q = fma(x[i], r, q);
      }
      if (!symmetric) {
        for (std::size_t i = 0; i < D; ++i) {
          double c = 0.0;
          for (std::size_t j = 0; j < D; ++j)
            c = fma(C[j * D + i], x[j], c);
          g[i] = 0.5 * (g[i] + c);
        }
      }
      return 0.5 * q;
    }

    // r = C^T x, split over Q = size/D segments of j so that every member
    // works; member t owns column i = t % D and segment t / D.  Reads of C
    // are coalesced (consecutive members, consecutive i).  The partial sums
    // meet in grp.scratch (size() doubles).  x^T C^T x = x^T C x, so f comes
    // from C^T x even when C is not symmetric.
    template <class G>
    __device__ void
    ctx_coop(const G& grp, const double* x, const double* M, double* r) const
    {
      const int t = grp.rank(), nq = grp.size() >= (int)D ? grp.size() / (int)D : 1;
      if (nq == 1) {
        grp.sync();
        for (int i = t; i < (int)D; i += grp.size()) {
          double a = 0.0;
          for (int j = 0; j < (int)D; ++j)
            a = fma(M[j * D + i], x[j], a);
          r[i] = a;
        }
        grp.sync();
        return;
      }
      const int i = t % (int)D, q = t / (int)D;
      double a = 0.0;
      if (q < nq) {
        // C comes from L2 (it does not fit beside H in shared memory):
        // unrolled with two sums so that many loads are in flight at once
        double a1 = 0.0;
        int j = q;
#pragma unroll 8
        for (; j + nq < (int)D; j += 2 * nq) {
          a = fma(M[j * D + i], x[j], a);
          a1 = fma(M[(j + nq) * D + i], x[j + nq], a1);
        }
        if (j < (int)D)
          a = fma(M[j * D + i], x[j], a);
        a += a1;
      }
      grp.sync();
      if (q < nq)
        grp.scratch[q * D + i] = a;
      grp.sync();
      if (t < (int)D) {
        double b = 0.0;
        for (int k = 0; k < nq; ++k)
          b += grp.scratch[k * D + t];
        r[t] = b;
      }
      grp.sync();
    }

    // rx = C^T x and rp = C^T p in one pass over C: each element of C is
    // loaded once and feeds two FMAs.  Member t owns column i = t % D and
    // segment t / D as in ctx_coop (even D: a column pair and segment
    // t / (D/2)); the segments' partial sums meet in the shared arrays sx
    // and sp (size() doubles each, 16-byte aligned; the pair form only
    // where C is 16-byte aligned).  Ends with a sync.
    template <class G>
    __device__ void
    ctx2_coop(const G& grp, const double* x, const double* p, double* rx,
              double* rp, double* sx, double* sp) const
    {
      constexpr int NP = (int)D / 2;
      if constexpr (D % 2 == 0) {
        if (grp.size() >= NP && (reinterpret_cast<uintptr_t>(C) & 15u) == 0) {
          // even D: member t owns the column pair (2c, 2c+1), c = t % NP,
          // and segment t / NP, reading C a 16-byte pair at a time
          const int t = grp.rank(), nq = grp.size() / NP;
          const int c = t % NP, q = t / NP;
          double ax0 = 0.0, ax1 = 0.0, ap0 = 0.0, ap1 = 0.0;
          if (q < nq) {
            double bx0 = 0.0, bx1 = 0.0, bp0 = 0.0, bp1 = 0.0;
            const double2* C2 = reinterpret_cast<const double2*>(C) + c;
            int j = q;
#pragma unroll 8
            for (; j + nq < (int)D; j += 2 * nq) {
              const double2 c0 = C2[j * NP], c1 = C2[(j + nq) * NP];
              const double x0 = x[j], p0 = p[j], x1 = x[j + nq], p1 = p[j + nq];
              ax0 = fma(c0.x, x0, ax0);
              ax1 = fma(c0.y, x0, ax1);
              ap0 = fma(c0.x, p0, ap0);
              ap1 = fma(c0.y, p0, ap1);
              bx0 = fma(c1.x, x1, bx0);
              bx1 = fma(c1.y, x1, bx1);
              bp0 = fma(c1.x, p1, bp0);
              bp1 = fma(c1.y, p1, bp1);
            }
            if (j < (int)D) {
              const double2 c0 = C2[j * NP];
              ax0 = fma(c0.x, x[j], ax0);
              ax1 = fma(c0.y, x[j], ax1);
              ap0 = fma(c0.x, p[j], ap0);
              ap1 = fma(c0.y, p[j], ap1);
            }
            ax0 += bx0;
            ax1 += bx1;
            ap0 += bp0;
            ap1 += bp1;
            *reinterpret_cast<double2*>(sx + q * D + 2 * c) = make_double2(ax0, ax1);
            *reinterpret_cast<double2*>(sp + q * D + 2 * c) = make_double2(ap0, ap1);
          }
          grp.sync();
          if (t < (int)D) {
            double bx = 0.0, bp = 0.0;
            for (int k = 0; k < nq; ++k) {
              bx += sx[k * D + t];
              bp += sp[k * D + t];
            }
            rx[t] = bx;
            rp[t] = bp;
          }
          grp.sync();
          return;
        }
      }
      const int t = grp.rank(), nq = grp.size() >= (int)D ? grp.size() / (int)D : 1;
      const int i = t % (int)D, q = t / (int)D;
      double ax = 0.0, ap = 0.0;
      if (q < nq) {
        double ax1 = 0.0, ap1 = 0.0;
        int j = q;
#pragma unroll 8
        for (; j + nq < (int)D; j += 2 * nq) {
          const double c0 = C[j * D + i], c1 = C[(j + nq) * D + i];
          ax = fma(c0, x[j], ax);
          ap = fma(c0, p[j], ap);
          ax1 = fma(c1, x[j + nq], ax1);
          ap1 = fma(c1, p[j + nq], ap1);
        }
        if (j < (int)D) {
          const double c0 = C[j * D + i];
          ax = fma(c0, x[j], ax);
          ap = fma(c0, p[j], ap);
        }
        ax += ax1;
        ap += ap1;
      }
      if (nq == 1) {
        // one segment: every member past D idles; members below D loop
        for (int k = t + grp.size(); k < (int)D; k += grp.size()) {
          double bx = 0.0, bp = 0.0;
          for (int jj = 0; jj < (int)D; ++jj) {
            bx = fma(C[jj * D + k], x[jj], bx);
            bp = fma(C[jj * D + k], p[jj], bp);
          }
          rx[k] = bx;
          rp[k] = bp;
        }
        if (t < (int)D) {
          rx[t] = ax;
          rp[t] = ap;
        }
        grp.sync();
        return;
      }
      if (q < nq) {
        sx[q * D + i] = ax;
        sp[q * D + i] = ap;
      }
      grp.sync();
      if (t < (int)D) {
        double bx = 0.0, bp = 0.0;
        for (int k = 0; k < nq; ++k) {
          bx += sx[k * D + t];
          bp += sp[k * D + t];
        }
        rx[t] = bx;
        rp[t] = bp;
      }
      grp.sync();
    }

    // f alone, 0.5 x.(C^T x): member t forms (C^T x)_i for its columns i
    // (reads of C coalesced across members); used where a whole f is
    // evaluated by a small group (a PSO particle's warp, line-search trial
    // groups of the dual-gradient form).
    template <class G>
    __device__ double
    value_coop(const G& grp, const double* x) const
    {
      double part = 0.0;
      detail::coop_for<(int)D>(grp, [&](int i) {
        double a0 = 0.0, a1 = 0.0;
        int j = 0;
        for (; j + 1 < (int)D; j += 2) {
          a0 = fma(C[j * D + i], x[j], a0);
          a1 = fma(C[(j + 1) * D + i], x[j + 1], a1);
        }
        if (j < (int)D)
          a0 = fma(C[j * D + i], x[j], a0);
        part = fma(x[i], a0 + a1, part);
      });
      return 0.5 * grp.sum(part);
    }

    // f = 0.5 x.r with r = C^T x formed by ctx_coop into the shared vector
    // r (the whole group streams C once, coalesced).
    template <class G>
    __device__ double
    value_ctx(const G& grp, const double* x, double* r) const
    {
      ctx_coop(grp, x, C, r);
      double part = 0.0;
      for (int i = grp.rank(); i < (int)D; i += grp.size())
        part = fma(x[i], r[i], part);
      return 0.5 * grp.sum(part);
    }

    // f = 0.5 x.(C^T x); g = C^T x (symmetric C) else (C x + C^T x) / 2.
    // `g` must be shared by the group (it is written by one member per i
    // and read back by all after the final sync).
    template <class G>
    __device__ double
    adjoint_coop(const G& grp, const double* x, double* g) const
    {
      const double f = value_ctx(grp, x, g);
      if (!symmetric) {
        // C x = (C^T)^T x: same kernel on the transpose via row reads
        for (int i = grp.rank(); i < (int)D; i += grp.size()) {
          double a = 0.0;
          for (int j = 0; j < (int)D; ++j)
            a = fma(C[i * D + j], x[j], a);
          g[i] = 0.5 * (g[i] + a);
        }
        grp.sync();
      }
      return f;
    }
    // The value costs the same matrix-vector product as the gradient; the
    // kernels evaluate line-search trials with adjoint_coop and keep g.
    static constexpr bool kTrialsWithGradient = true;
    // f is a quadratic form: f(x + a p) = f(x) + a grad f(x).p + a^2 f(p)
    // for every x, p, a, so a line search needs f(p) once, not f per trial.
    static constexpr bool kQuadraticForm = true;
  };

  // Binned Poisson negative log-likelihood of the dijet shape
  // lambda_i = a (1-x_i)^b / x_i^(c + d ln x_i) (LogLikelihood.h:29-58).
  // `bins` holds per-bin constants for the fast paths, 4 doubles per bin:
  // {ln x_i, ln(1 - x_i), k_i, lgamma(k_i + 1)}; centres/counts feed the
  // reference-order operator().
  struct PoissonNLL {
    static constexpr std::size_t arity = 4;
    static constexpr int kind = 4;
    const double* centres = nullptr;
    const int* counts = nullptr;
    const double* bins = nullptr;
    int nbins = 0;

    template <class T>
    __host__ __device__ T
    operator()(const std::array<T, 4>& th) const
    {
      using ::lgamma;
      using ::log;
      using ::pow;
      const T a = th[0], b = th[1], c = th[2], d = th[3];
      T nll = T(0);
      for (int i = 0; i < nbins; ++i) {
        const T x = T(centres[i]);
        const int ki = counts[i];
        const T mean = a * pow(T(1.0) - x, b) / pow(x, c + d * log(x));
        const T log_p = T(ki) * log(mean) - mean - lgamma(T(ki) + T(1));
        nll -= log_p;
      }
      return nll;
    }

    // ln lambda = ln a + b ln(1-x) - (c + d ln x) ln x
    __host__ __device__ double
    value(const double* th) const
    {
      const double la = ::log(th[0]);
      double nll = 0.0;
      for (int i = 0; i < nbins; ++i) {
        const double lx = bins[4 * i], l1 = bins[4 * i + 1];
        const double k = bins[4 * i + 2], lgk = bins[4 * i + 3];
        const double ll = la + fma(th[1], l1, -fma(th[3], lx, th[2]) * lx);
        nll += ::exp(ll) - fma(k, ll, -lgk);
      }
      return nll;
    }

    // dNLL/dtheta = sum (lambda - k) dln(lambda)/dtheta with
    // dln(lambda) = (1/a, ln(1-x), -ln x, -(ln x)^2)
    __host__ __device__ double
    adjoint(const double* th, double* g) const
    {
      const double la = ::log(th[0]);
      double nll = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0, g3 = 0.0;
      for (int i = 0; i < nbins; ++i) {
        const double lx = bins[4 * i], l1 = bins[4 * i + 1];
        const double k = bins[4 * i + 2], lgk = bins[4 * i + 3];
        const double ll = la + fma(th[1], l1, -fma(th[3], lx, th[2]) * lx);
        const double lam = ::exp(ll);
        nll += lam - fma(k, ll, -lgk);
        const double w = lam - k;
        g0 += w;
        g1 = fma(w, l1, g1);
        g2 = fma(-w, lx, g2);
        g3 = fma(-w * lx, lx, g3);
      }
      g[0] = g0 / th[0];
      g[1] = g1;
      g[2] = g2;
      g[3] = g3;
      return nll;
    }

    // Cooperative forms split the bins over the group.
    template <class G>
    __device__ double
    value_coop(const G& grp, const double* th) const
    {
      const double la = ::log(th[0]);
      double part = 0.0;
      for (int i = grp.rank(); i < nbins; i += grp.size()) {
        const double lx = bins[4 * i], l1 = bins[4 * i + 1];
        const double k = bins[4 * i + 2], lgk = bins[4 * i + 3];
        const double ll = la + fma(th[1], l1, -fma(th[3], lx, th[2]) * lx);
        part += ::exp(ll) - fma(k, ll, -lgk);
      }
      return grp.sum(part);
    }
    template <class G>
    __device__ double
    adjoint_coop(const G& grp, const double* th, double* g) const
    {
      const double la = ::log(th[0]);
      double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
      for (int i = grp.rank(); i < nbins; i += grp.size()) {
        const double lx = bins[4 * i], l1 = bins[4 * i + 1];
        const double k = bins[4 * i + 2], lgk = bins[4 * i + 3];
        const double ll = la + fma(th[1], l1, -fma(th[3], lx, th[2]) * lx);
        const double lam = ::exp(ll);
        v[0] += lam - fma(k, ll, -lgk);
        const double w = lam - k;
        v[1] += w;
        v[2] = fma(w, l1, v[2]);
        v[3] = fma(-w, lx, v[3]);
        v[4] = fma(-w * lx, lx, v[4]);
      }
      grp.template sum<5>(v);
      if (grp.rank() == 0) {
        g[0] = v[1] / th[0];
        g[1] = v[2];
        g[2] = v[3];
        g[3] = v[4];
      }
      return v[0];
    }
  };

} // namespace zeus
