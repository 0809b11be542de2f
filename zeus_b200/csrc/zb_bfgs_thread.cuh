// Fast BFGS, one run per thread, for small D (the layout for D <= 8).
//
// Everything a run owns lives in registers: x, g, p and the inverse Hessian
// H, stored as its upper triangle (D(D+1)/2 doubles).  The symmetric rank-2
// form of the reference's update (utils.cuh:245-287),
//   H+ = H + s w^T + w s^T,  u = H y,  w = -rho u + rho (1 + rho y.u)/2 s,
// costs O(D^2) instead of the reference's O(D^4) and keeps H exactly
// symmetric (each (i, j) pair is formed once).  The line search, the
// |s.y| < 1e-14 skip, accept-if-better and the termination protocol are the
// reference's (utils.cuh:376-412, bfgs_sequential.cuh:99-219); f at the
// accepted trial point is reused as f(x_new) and f(x) at termination is
// the tracked best value, both identical to what the reference recomputes.
#pragma once

#include "zb_common.cuh"

namespace zb {

  template <int D>
  __host__ __device__ constexpr int
  tri(int i, int j) // packed upper-triangle index, i <= j
  {
    return i * D - (i * (i - 1)) / 2 + (j - i);
  }
  template <int D>
  __host__ __device__ constexpr int
  sym(int i, int j)
  {
    return i <= j ? tri<D>(i, j) : tri<D>(j, i);
  }

  // f(x) through the objective's fast path when it has one.
  template <class F, int D>
  __device__ __forceinline__ double
  fast_value(const F& f, const double* x)
  {
    if constexpr (HasValue<F>) {
      return f.value(x);
    } else {
      std::array<double, D> a;
#pragma unroll
      for (int i = 0; i < D; ++i)
        a[i] = x[i];
      return f(a);
    }
  }

  // Gradient by D forward dual passes (the plain form), or by the
  // objective's adjoint.
  template <class F, int D, bool Adjoint>
  __device__ __forceinline__ void
  fast_gradient(const F& f, const double* x, double* g)
  {
    if constexpr (Adjoint && HasAdjoint<F>) {
      (void)f.adjoint(x, g);
    } else {
      std::array<dual::DualNumber, D> xd;
#pragma unroll
      for (int j = 0; j < D; ++j)
        xd[j] = dual::DualNumber(x[j], 0.0);
#pragma unroll
      for (int i = 0; i < D; ++i) {
        xd[i].dual = 1.0;
        g[i] = f(xd).dual;
        xd[i].dual = 0.0;
      }
    }
  }

  // One run, start x0[D], results to slot idx of `out`.
  template <class F, int D, bool Adjoint, bool kTimed = false>
  __device__ __forceinline__ void
  thread_run(const F& f, const BfgsParams& prm, const double* __restrict__ x0,
             int64_t idx, const RunOut& out, Control* ctl)
  {
    constexpr int NT = D * (D + 1) / 2;
    double x[D], g[D], p[D], H[NT];
#pragma unroll
    for (int i = 0; i < D; ++i)
      x[i] = x0[i];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = i; j < D; ++j)
        H[tri<D>(i, j)] = (i == j) ? 1.0 : 0.0;

    const CycleTimer<kTimed> tm(out, idx, true);
    double best = fast_value<F, D>(f, x);
    tm.start_grad();
    fast_gradient<F, D, Adjoint>(f, x, g);
    tm.stop_grad();
    long long n_eval = 1, n_grad = 1;
#pragma unroll
    for (int i = 0; i < D; ++i)
      p[i] = -g[i];

    int status = kUnset, iter, executed = -1;
    double fout = best, gout = 0.0;
    for (iter = 0; iter < prm.max_iter; ++iter) {
      if (load_stop(ctl)) {
        status = kStopped;
        break;
      }
      double ddir = 0.0;
#pragma unroll
      for (int i = 0; i < D; ++i)
        ddir = fma(g[i], p[i], ddir);
      double xn[D], alpha = 1.0, fnew = 0.0;
      bool ok = false;
      for (int k = 0; k < kLineSearchTrials; ++k) {
#pragma unroll
        for (int i = 0; i < D; ++i)
          xn[i] = fma(alpha, p[i], x[i]);
        const double f1 = fast_value<F, D>(f, xn);
        ++n_eval;
        if (f1 <= best + kArmijoC1 * alpha * ddir && f1 < best) {
          ok = true;
          fnew = f1;
          break;
        }
        alpha *= 0.5;
      }
      if (!ok) {
#pragma unroll
        for (int i = 0; i < D; ++i)
          xn[i] = fma(alpha, p[i], x[i]);
        fnew = fast_value<F, D>(f, xn);
        ++n_eval;
      }
      double gn[D], s[D], y[D];
      tm.start_grad();
      fast_gradient<F, D, Adjoint>(f, xn, gn);
      tm.stop_grad();
      ++n_grad;
      tm.start_update();
      double sy = 0.0;
#pragma unroll
      for (int i = 0; i < D; ++i) {
        s[i] = xn[i] - x[i];
        y[i] = gn[i] - g[i];
        sy = fma(s[i], y[i], sy);
      }
      const bool skipped = fabs(sy) < kMinCurvature;
      if (!skipped) {
        const double rho = 1.0 / sy;
        double u[D], yu = 0.0;
#pragma unroll
        for (int i = 0; i < D; ++i) {
          double a = 0.0;
#pragma unroll
          for (int j = 0; j < D; ++j)
            a = fma(H[sym<D>(i, j)], y[j], a);
          u[i] = a;
          yu = fma(y[i], a, yu);
        }
        const double half_beta = 0.5 * rho * fma(rho, yu, 1.0);
        double w[D];
#pragma unroll
        for (int i = 0; i < D; ++i)
          w[i] = fma(half_beta, s[i], -rho * u[i]);
#pragma unroll
        for (int i = 0; i < D; ++i)
#pragma unroll
          for (int j = i; j < D; ++j)
            H[tri<D>(i, j)] += s[i] * w[j] + w[i] * s[j];
      }
      tm.stop_update();
      const bool take = fnew < best;
      if (take) {
        best = fnew;
#pragma unroll
        for (int i = 0; i < D; ++i) {
          x[i] = xn[i];
          g[i] = gn[i];
        }
      }
      double gg = 0.0;
#pragma unroll
      for (int i = 0; i < D; ++i)
        gg = fma(g[i], g[i], gg);
      const double gnrm = sqrt(gg);
      if (!isfinite(gnrm) || !isfinite(fnew)) {
        status = kNonFinite;
        fout = fnew;
        gout = gnrm;
        break;
      }
      if (gnrm < prm.tol) {
        note_converged(ctl, prm.required);
        status = kConverged;
        fout = best;
        gout = gnrm;
        break;
      }
      if (!take && skipped && !(prm.flags & kFlagNoFixedPoint)) {
        executed = iter + 1; // fixed point: the rest would repeat this
        iter = prm.max_iter;
        break;
      }
#pragma unroll
      for (int i = 0; i < D; ++i) {
        double a = 0.0;
#pragma unroll
        for (int j = 0; j < D; ++j)
          a = fma(H[sym<D>(i, j)], g[j], a);
        p[i] = -a;
      }
    }
    if (status == kUnset || status == kStopped) {
      if (status == kUnset)
        status = kSurrender;
      fout = best;
      double gg = 0.0;
#pragma unroll
      for (int i = 0; i < D; ++i)
        gg = fma(g[i], g[i], gg);
      gout = sqrt(gg);
    }
    if (out.fval)
      out.fval[idx] = fout;
    if (out.status)
      out.status[idx] = status;
    if (out.iter)
      out.iter[idx] = iter;
    if (out.gnorm)
      out.gnorm[idx] = gout;
    if (out.x)
#pragma unroll
      for (int i = 0; i < D; ++i)
        out.x[idx * D + i] = x[i];
    if (out.counters) {
      out.counters[3 * idx + 0] = executed >= 0 ? executed : iter;
      out.counters[3 * idx + 1] = n_eval;
      out.counters[3 * idx + 2] = n_grad;
    }
    tm.finish();
  }

  template <class F, int D, bool Adjoint, bool kTimed = false>
  __global__ void __launch_bounds__(128)
    bfgs_thread_kernel(F f, BfgsParams prm, const double* __restrict__ starts,
                       RunOut out, Control* ctl)
  {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < prm.n)
      thread_run<F, D, Adjoint, kTimed>(f, prm, starts + idx * D, idx, out, ctl);
  }

} // namespace zb
