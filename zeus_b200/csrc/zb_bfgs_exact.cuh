// Exact-mode BFGS: the reference's arithmetic, one run per CTA.
//
// Reproduces bfgs::sequential::optimize (bfgs_sequential.cuh:46-234) value
// for value: same line search (utils.cuh:376-412), same inverse update
// (utils.cuh:245-287), same dual-number gradient (duals.cuh:241-266), same
// accept / termination order (bfgs_common.cuh:110-238).  The translation
// unit that instantiates this header is compiled with -fmad=false, so with
// the reference's own operation order every +,-,*,/ and sqrt rounds exactly
// as in the reference built for the host; only CUDA's transcendental
// functions may differ from the host libm by an ulp.
//
// The CTA spreads the work that the reference does serially but whose
// per-element arithmetic is independent, without changing any summation
// order:
//   * the D dual passes of the gradient, one per thread;
//   * the 20 line-search trials alpha = 2^-k, one per thread, taking the
//     first k that passes (the sequential loop returns exactly that alpha);
//   * p_i = -sum_j H_ij g_j, one row per thread (j ascending);
//   * the update's inner sums T_kj = sum_m H_km B_mj, computed once per
//     (k, j) instead of once per (i, k, j) -- the reference recomputes the
//     same value D times -- then H_ij = sum_k A_ik T_kj + rho s_i s_j.
// Dot products and the gradient norm stay on thread 0 in index order.
// H and T (2 D^2 doubles) live in a global workspace slice per CTA.
#pragma once

#include "zb_common.cuh"

namespace zb {

  struct ExactShared {
    double best, f1, fnew, ddir, sy, gnorm;
    int accepted, done, status, stop, executed;
  };

  template <class F, int D>
  __device__ __forceinline__ double
  eval_array(const F& f, const double* x)
  {
    std::array<double, D> a;
#pragma unroll 1
    for (int i = 0; i < D; ++i)
      a[i] = x[i];
    return f(a);
  }

  // g_i = d f / d x_i by a forward pass seeded with e_i, i = tid, tid+bs, ...
  template <class F, int D>
  __device__ __forceinline__ void
  exact_dual_gradient(const F& f, const double* x, double* g)
  {
    for (int i = threadIdx.x; i < D; i += blockDim.x) {
      std::array<dual::DualNumber, D> xd;
#pragma unroll 1
      for (int j = 0; j < D; ++j)
        xd[j] = dual::DualNumber(x[j], 0.0);
      xd[i].dual = 1.0;
      g[i] = f(xd).dual;
    }
  }

  template <class F, int D, bool Traj>
  __global__ void __launch_bounds__(128)
    bfgs_exact_kernel(F f, BfgsParams prm, const double* __restrict__ starts,
                      RunOut out, Control* ctl, double* __restrict__ scratch)
  {
    extern __shared__ __align__(16) double sm[];
    double* x = sm;
    double* xn = x + D;
    double* g = xn + D;
    double* gn = g + D;
    double* p = gn + D;
    double* s = p + D;
    double* y = s + D;
    __shared__ ExactShared sh;
    __shared__ int trial_ok[kLineSearchTrials];
    __shared__ double trial_f[kLineSearchTrials];

    double* H = scratch + (size_t)blockIdx.x * 2 * D * D;
    double* T = H + (size_t)D * D;
    const int tid = threadIdx.x, bs = blockDim.x;
    const int N = (int)prm.n;

    for (int64_t run = blockIdx.x; run < prm.n; run += gridDim.x) {
      const int idx = (int)run;
      for (int d = tid; d < D; d += bs) {
        x[d] = starts[(size_t)idx * D + d];
        g[d] = 0.0;
      }
      for (int e = tid; e < D * D; e += bs)
        H[e] = (e / D == e % D) ? 1.0 : 0.0;
      long long n_eval = 0, n_grad = 0;
      __syncthreads();
      const CycleTimer<true> tm(out, idx, tid == 0);
      if (tid == 0) {
        sh.best = eval_array<F, D>(f, x);
        sh.done = 0;
        sh.status = kUnset;
      }
      tm.start_grad();
      exact_dual_gradient<F, D>(f, x, g);
      ++n_eval;
      ++n_grad;
      __syncthreads();
      tm.stop_grad();

      int iter;
      for (iter = 0; iter < prm.max_iter; ++iter) {
        if constexpr (Traj) {
          for (int d = tid; d < D; d += bs)
            out.traj_x[(size_t)iter * D * N + (size_t)d * N + idx] = x[d];
          if (tid == 0) {
            double gg = 0.0;
            for (int i = 0; i < D; ++i)
              gg += g[i] * g[i];
            out.traj_f[(size_t)iter * N + idx] = sh.best;
            out.traj_g[(size_t)iter * N + idx] = ::sqrt(gg);
            out.traj_status[(size_t)iter * N + idx] = -1;
          }
        }
        if (tid == 0)
          sh.stop = load_stop(ctl);
        __syncthreads();
        if (sh.stop) {
          if (tid == 0) {
            sh.status = kStopped;
            double gg = 0.0;
            for (int i = 0; i < D; ++i)
              gg += g[i] * g[i];
            sh.gnorm = ::sqrt(gg);
            sh.fnew = sh.best; // f(x_arr) == bestVal by construction
            if constexpr (Traj)
              out.traj_status[(size_t)iter * N + idx] = kStopped;
          }
          __syncthreads();
          break;
        }
        // p = -H g (utils.cuh:148-161)
        for (int i = tid; i < D; i += bs) {
          double sum = 0.0;
          for (int j = 0; j < D; ++j)
            sum += H[(size_t)i * D + j] * g[j];
          p[i] = -sum;
        }
        __syncthreads();
        if (tid == 0) {
          double dd = 0.0;
          for (int i = 0; i < D; ++i)
            dd += g[i] * p[i];
          sh.ddir = dd;
        }
        __syncthreads();
        // line search trials alpha_k = 2^-k, k = 0..19
        for (int k = tid; k < kLineSearchTrials; k += bs) {
          double alpha = 1.0;
          for (int h = 0; h < k; ++h)
            alpha *= 0.5;
          std::array<double, D> xt;
#pragma unroll 1
          for (int j = 0; j < D; ++j)
            xt[j] = x[j] + alpha * p[j];
          const double f1 = f(xt);
          const double f0 = sh.best;
          trial_ok[k] = (f1 <= f0 + kArmijoC1 * alpha * sh.ddir && f1 < f0);
          trial_f[k] = f1;
        }
        __syncthreads();
        if (tid == 0) {
          int k = 0;
          while (k < kLineSearchTrials && !trial_ok[k])
            ++k;
          sh.accepted = k;
          sh.f1 = k < kLineSearchTrials ? trial_f[k] : 0.0;
          n_eval += (k < kLineSearchTrials ? k + 1 : kLineSearchTrials);
        }
        __syncthreads();
        {
          const int k = sh.accepted;
          double alpha = 1.0;
          for (int h = 0; h < k; ++h)
            alpha *= 0.5; // k == 20 gives the reference's 2^-20
          for (int i = tid; i < D; i += bs) {
            xn[i] = x[i] + alpha * p[i];
            s[i] = xn[i] - x[i];
          }
        }
        __syncthreads();
        if (tid == 0) {
          if (sh.accepted < kLineSearchTrials) {
            sh.fnew = sh.f1; // same point, same arithmetic as f(x_new)
          } else {
            sh.fnew = eval_array<F, D>(f, xn);
            ++n_eval;
          }
        }
        tm.start_grad();
        exact_dual_gradient<F, D>(f, xn, gn);
        ++n_grad;
        __syncthreads();
        tm.stop_grad();
        for (int i = tid; i < D; i += bs)
          y[i] = gn[i] - g[i];
        __syncthreads();
        if (tid == 0) {
          double sy = 0.0;
          for (int i = 0; i < D; ++i)
            sy += s[i] * y[i];
          sh.sy = sy;
        }
        __syncthreads();
        tm.start_update();
        if (!(::fabs(sh.sy) < kMinCurvature)) {
          const double rho = 1.0 / sh.sy;
          for (int e = tid; e < D * D; e += bs) {
            const int k = e / D, j = e % D;
            double inner = 0.0;
            for (int m = 0; m < D; ++m) {
              const double B_mj = ((m == j) ? 1.0 : 0.0) - rho * y[m] * s[j];
              inner += H[(size_t)k * D + m] * B_mj;
            }
            T[e] = inner;
          }
          __syncthreads();
          for (int e = tid; e < D * D; e += bs) {
            const int i = e / D, j = e % D;
            double sum = 0.0;
            for (int k = 0; k < D; ++k) {
              const double A_ik = ((i == k) ? 1.0 : 0.0) - rho * s[i] * y[k];
              sum += A_ik * T[(size_t)k * D + j];
            }
            H[e] = sum + rho * s[i] * s[j];
          }
        }
        const bool skipped = ::fabs(sh.sy) < kMinCurvature;
        __syncthreads();
        tm.stop_update();
        const bool take = sh.fnew < sh.best;
        if (take)
          for (int i = tid; i < D; i += bs) {
            x[i] = xn[i];
            g[i] = gn[i];
          }
        __syncthreads();
        if (tid == 0) {
          if (take)
            sh.best = sh.fnew;
          double gg = 0.0;
          for (int i = 0; i < D; ++i)
            gg += g[i] * g[i];
          const double gnrm = ::sqrt(gg);
          sh.gnorm = gnrm;
          if (!::isfinite(gnrm) || !::isfinite(sh.fnew)) {
            sh.status = kNonFinite; // fval = fnew (bfgs_common.cuh:156-157)
            sh.done = 1;
          } else if (gnrm < prm.tol) {
            note_converged(ctl, prm.required);
            sh.status = kConverged;
            sh.fnew = sh.best;
            sh.done = 1;
          } else if (!Traj && !take && skipped &&
                     !(prm.flags & kFlagNoFixedPoint)) {
            sh.done = 2; // fixed point: the rest would repeat this iteration
          }
          if constexpr (Traj)
            if (sh.done)
              out.traj_status[(size_t)iter * N + idx] = (int8_t)sh.status;
        }
        __syncthreads();
        if (sh.done == 2) {
          sh.executed = iter + 1;
          iter = prm.max_iter;
          break;
        }
        if (sh.done)
          break;
      }
      if (sh.done != 2)
        sh.executed = iter;
      if (tid == 0) {
        if (sh.status == kUnset) { // bfgs_common.cuh:213-238
          sh.status = kSurrender;
          sh.fnew = sh.best;
          double gg = 0.0;
          for (int i = 0; i < D; ++i)
            gg += g[i] * g[i];
          sh.gnorm = ::sqrt(gg);
          if constexpr (Traj)
            if (prm.max_iter > 0)
              out.traj_status[(size_t)(prm.max_iter - 1) * N + idx] = 0;
        }
        if (out.fval)
          out.fval[idx] = sh.fnew;
        if (out.status)
          out.status[idx] = sh.status;
        if (out.iter)
          out.iter[idx] = iter;
        if (out.gnorm)
          out.gnorm[idx] = sh.gnorm;
        if (out.counters) {
          out.counters[3 * (size_t)idx + 0] = sh.executed;
          out.counters[3 * (size_t)idx + 1] = n_eval;
          out.counters[3 * (size_t)idx + 2] = n_grad;
        }
        tm.finish();
      }
      if (out.x)
        for (int d = tid; d < D; d += bs)
          out.x[(size_t)idx * D + d] = x[d];
      __syncthreads();
    }
  }

  template <int D>
  inline size_t
  exact_smem_bytes()
  {
    return sizeof(double) * 7 * D;
  }

} // namespace zb
