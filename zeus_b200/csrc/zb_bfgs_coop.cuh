// Fast BFGS with one optimisation per cooperating group:
//
//   bfgs_tile_kernel  (mid D, up to 32): a tile of TS lanes per run.  Lane l
//     owns coordinates l, l+TS, ... (R = ceil(D/TS) of them) and the same rows
//     of the inverse Hessian H, in registers.  Vectors other lanes need (y, s,
//     w, g for H products; the trial point for f) go through a small
//     per-tile shared buffer; scalars through butterfly shuffles.
//
//   bfgs_cta_kernel   (large D, up to ~160): a thread block per run, H in
//     shared memory (D x D doubles, kept exactly symmetric).  One sweep
//     reads H once and forms both u = H y and h = H g_next (thread t walks
//     column t % D over a 1/Q share of the rows; Q = blockDim / D partial
//     sums meet in shared memory) -- column walks by consecutive threads are
//     bank-conflict free; a second sweep applies the rank-2 update in place.
//     The next search direction follows without a third sweep:
//     H+ g = h + s (w.g) + w (s.g).
//
// Both keep the reference's iteration semantics (line search, skip rule,
// accept-if-better, status protocol) and the fixed-point exit.  The update
// H+ = H + s w^T + w s^T forms each product with __dmul_rn so that entry
// (i, j) and (j, i) round identically and H stays exactly symmetric (the
// CTA kernel reads columns as rows).
#pragma once

#include "zb_bfgs_thread.cuh"
#include "zb_common.cuh"
#include "zb_group.cuh"

namespace zb {

  template <class F, class G>
  concept HasValueCoop = requires(const F& f, const G& g, const double* x) {
    { f.value_coop(g, x) } -> std::convertible_to<double>;
  };
  template <class F, class G>
  concept HasAdjointCoop =
    requires(const F& f, const G& g, const double* x, double* gr) {
      { f.adjoint_coop(g, x, gr) } -> std::convertible_to<double>;
    };
  template <class F>
  concept TrialsWithGradient = requires { F::kTrialsWithGradient; };

  // f(x) for a shared x, the same value in every member.
  template <class F, int D, class G>
  __device__ __forceinline__ double
  coop_value(const F& f, const G& grp, const double* x)
  {
    if constexpr (HasValueCoop<F, G>) {
      return f.value_coop(grp, x);
    } else {
      double v = 0.0;
      if (grp.rank() == 0)
        v = fast_value<F, D>(f, x);
      return grp.bcast(v, 0);
    }
  }

  // g = grad f(x) into shared g (one member per entry); the caller syncs
  // before reading it.  Returns f(x) when the adjoint computed it, else NaN.
  template <class F, int D, bool Adjoint, class G>
  __device__ __forceinline__ double
  coop_gradient(const F& f, const G& grp, const double* x, double* g)
  {
    if constexpr (Adjoint && HasAdjointCoop<F, G>) {
      return f.adjoint_coop(grp, x, g);
    } else if constexpr (Adjoint && HasAdjoint<F>) {
      double v = 0.0;
      if (grp.rank() == 0)
        v = f.adjoint(x, g);
      return grp.bcast(v, 0);
    } else {
      // the plain form: D forward dual passes spread over the members
      for (int i = grp.rank(); i < D; i += grp.size()) {
        std::array<dual::DualNumber, D> xd;
#pragma unroll 1
        for (int j = 0; j < D; ++j)
          xd[j] = dual::DualNumber(x[j], 0.0);
        xd[i].dual = 1.0;
        g[i] = f(xd).dual;
      }
      return __longlong_as_double(0x7ff8000000000000ll);
    }
  }

  // ---------------------------------------------------------------- tile
  inline constexpr int kTileBlock = 128;

  template <int D, int TS>
  constexpr int
  tile_smem_doubles()
  {
    return 4 * D + TS; // xs, gs, b1, b2, scratch
  }

  // One run on a tile: `buf` is the tile's tile_smem_doubles<D, TS>()
  // doubles of shared memory; start x0[D]; results to slot `run` of `out`.
  template <class F, int D, int TS, bool Adjoint>
  __device__ __forceinline__ void
  tile_run(const F& f, cg::thread_block_tile<TS> tile, double* buf,
           const BfgsParams& prm, const double* __restrict__ x0, int64_t run,
           const RunOut& out, Control* ctl)
  {
    constexpr int R = (D + TS - 1) / TS;
    const int lane = (int)tile.thread_rank();
    double* xs = buf;
    double* gs = xs + D;
    double* b1 = gs + D;
    double* b2 = b1 + D;
    TileGroup<TS> grp(tile, b2 + D);

    double x[R], g[R], p[R], H[R][D];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = lane + r * TS;
      x[r] = i < D ? x0[i] : 0.0;
      if (i < D)
        xs[i] = x[r];
#pragma unroll
      for (int j = 0; j < D; ++j)
        H[r][j] = (i == j) ? 1.0 : 0.0;
    }
    grp.sync();
    double best = coop_value<F, D>(f, grp, xs);
    coop_gradient<F, D, Adjoint>(f, grp, xs, gs);
    grp.sync();
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = lane + r * TS;
      g[r] = i < D ? gs[i] : 0.0;
      p[r] = -g[r];
    }
    long long n_eval = 1, n_grad = 1;
    int status = kUnset, iter, executed = -1;
    double fout = best, gout = 0.0;

    for (iter = 0; iter < prm.max_iter; ++iter) {
      const int stop = grp.bcast(lane == 0 ? load_stop(ctl) : 0, 0);
      if (stop) {
        status = kStopped;
        break;
      }
      double dd = 0.0;
#pragma unroll
      for (int r = 0; r < R; ++r)
        dd = fma(g[r], p[r], dd);
      const double ddir = grp.sum(dd);
      double xn[R], alpha = 1.0, fnew = 0.0;
      bool ok = false;
      for (int k = 0; k <= kLineSearchTrials; ++k) {
        grp.sync(); // earlier readers of xs are done
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = lane + r * TS;
          xn[r] = fma(alpha, p[r], x[r]);
          if (i < D)
            xs[i] = xn[r];
        }
        grp.sync();
        const double f1 = coop_value<F, D>(f, grp, xs);
        ++n_eval;
        if (k == kLineSearchTrials) { // all 20 failed: alpha = 2^-20
          fnew = f1;
          break;
        }
        if (f1 <= best + kArmijoC1 * alpha * ddir && f1 < best) {
          ok = true;
          fnew = f1;
          break;
        }
        alpha *= 0.5;
      }
      (void)ok;
      grp.sync();
      coop_gradient<F, D, Adjoint>(f, grp, xs, gs);
      ++n_grad;
      grp.sync();
      double gn[R], s[R], y[R];
      double sy_part = 0.0;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = lane + r * TS;
        gn[r] = i < D ? gs[i] : 0.0;
        s[r] = xn[r] - x[r];
        y[r] = gn[r] - g[r];
        sy_part = fma(s[r], y[r], sy_part);
      }
      const double sy = grp.sum(sy_part);
      const bool skipped = fabs(sy) < kMinCurvature;
      if (!skipped) {
        const double rho = 1.0 / sy;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = lane + r * TS;
          if (i < D)
            b1[i] = y[r];
        }
        grp.sync();
        double u[R], yu_part = 0.0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          double a = 0.0;
#pragma unroll
          for (int j = 0; j < D; ++j)
            a = fma(H[r][j], b1[j], a);
          u[r] = a;
          yu_part = fma(y[r], a, yu_part);
        }
        const double yu = grp.sum(yu_part);
        const double hb = 0.5 * rho * fma(rho, yu, 1.0);
        double w[R];
#pragma unroll
        for (int r = 0; r < R; ++r)
          w[r] = fma(hb, s[r], -rho * u[r]);
        grp.sync(); // b1 (= y) fully read
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = lane + r * TS;
          if (i < D) {
            b1[i] = s[r];
            b2[i] = w[r];
          }
        }
        grp.sync();
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
          for (int j = 0; j < D; ++j)
            H[r][j] += __dadd_rn(__dmul_rn(s[r], b2[j]), __dmul_rn(w[r], b1[j]));
      }
      const bool take = fnew < best;
      if (take) {
        best = fnew;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          x[r] = xn[r];
          g[r] = gn[r];
        }
      }
      double gg = 0.0;
#pragma unroll
      for (int r = 0; r < R; ++r)
        gg = fma(g[r], g[r], gg);
      const double gnrm = sqrt(grp.sum(gg));
      if (!isfinite(gnrm) || !isfinite(fnew)) {
        status = kNonFinite;
        fout = fnew;
        gout = gnrm;
        break;
      }
      if (gnrm < prm.tol) {
        if (lane == 0)
          note_converged(ctl, prm.required);
        status = kConverged;
        fout = best;
        gout = gnrm;
        break;
      }
      if (!take && skipped && !(prm.flags & kFlagNoFixedPoint)) {
        executed = iter + 1;
        iter = prm.max_iter;
        break;
      }
      grp.sync(); // b1 / b2 fully read
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = lane + r * TS;
        if (i < D)
          b1[i] = g[r];
      }
      grp.sync();
#pragma unroll
      for (int r = 0; r < R; ++r) {
        double a = 0.0;
#pragma unroll
        for (int j = 0; j < D; ++j)
          a = fma(H[r][j], b1[j], a);
        p[r] = -a;
      }
    }
    if (status == kUnset || status == kStopped) {
      if (status == kUnset)
        status = kSurrender;
      fout = best;
      double gg = 0.0;
#pragma unroll
      for (int r = 0; r < R; ++r)
        gg = fma(g[r], g[r], gg);
      gout = sqrt(grp.sum(gg));
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = lane + r * TS;
      if (out.x && i < D)
        out.x[run * D + i] = x[r];
    }
    if (lane == 0) {
      if (out.fval)
        out.fval[run] = fout;
      if (out.status)
        out.status[run] = status;
      if (out.iter)
        out.iter[run] = iter;
      if (out.gnorm)
        out.gnorm[run] = gout;
      if (out.counters) {
        out.counters[3 * run + 0] = executed >= 0 ? executed : iter;
        out.counters[3 * run + 1] = n_eval;
        out.counters[3 * run + 2] = n_grad;
      }
    }
  }

  template <class F, int D, int TS, bool Adjoint>
  __global__ void __launch_bounds__(kTileBlock)
    bfgs_tile_kernel(F f, BfgsParams prm, const double* __restrict__ starts,
                     RunOut out, Control* ctl)
  {
    constexpr int TPB = kTileBlock / TS;
    extern __shared__ double sm[];
    auto tile = cg::tiled_partition<TS>(cg::this_thread_block());
    const int tslot = threadIdx.x / TS;
    const int64_t run = (int64_t)blockIdx.x * TPB + tslot;
    if (run >= prm.n)
      return; // the whole tile leaves together
    tile_run<F, D, TS, Adjoint>(f, tile, sm + tslot * tile_smem_doubles<D, TS>(),
                                prm, starts + run * D, run, out, ctl);
  }

  // ---------------------------------------------------------------- CTA
  // Shared-memory layout (doubles): H[D*D] | 11 vectors of D | partial sums
  // 2*Q*D | reduction buffers kCtaRedDoubles | scratch blockDim | trial
  // values 2*32 | flags 4 | (warp trials) one trial point per warp,
  // (blockDim/32)*D.
  __host__ __device__ constexpr size_t
  cta_smem_doubles_rt(int d, int block, bool warp_trials)
  {
    const int q = block >= d ? block / d : 1;
    return (size_t)d * d + 11 * d + 2 * q * d + kCtaRedDoubles + block + 64 + 4 +
           (warp_trials ? (size_t)(block / 32) * d : 0);
  }

  // Line-search trials are evaluated one per warp, all warps at once, unless
  // a trial carries a gradient (the Gaussian's C x needs the whole block).
  template <class F, bool Adjoint>
  __host__ __device__ constexpr bool
  cta_warp_trials()
  {
    return !(Adjoint && TrialsWithGradient<F>);
  }

  template <class F, int D, bool Adjoint>
  __host__ __device__ constexpr size_t
  cta_smem_doubles(int block)
  {
    return cta_smem_doubles_rt(D, block, cta_warp_trials<F, Adjoint>());
  }

  // One run on the whole block (blockDim.x == kBlock): `sm` holds
  // cta_smem_doubles<D>(kBlock) doubles; start x0[D]; results to slot `run`.
  template <class F, int D, bool Adjoint, int kBlock>
  __device__ __forceinline__ void
  cta_run(const F& f, double* sm, const BfgsParams& prm,
          const double* __restrict__ x0, int64_t run, const RunOut& out,
          Control* ctl)
  {
    constexpr int Q = kBlock >= D ? kBlock / D : 1;
    constexpr bool kTrialGrad = Adjoint && TrialsWithGradient<F>;
    constexpr bool kWarpTrials = cta_warp_trials<F, Adjoint>();
    constexpr int NW = kBlock / 32;
    double* H = sm;
    double* x = H + D * D;
    double* g = x + D;
    double* p = g + D;
    double* xn = p + D;
    double* gn = xn + D;
    double* s = gn + D;
    double* y = s + D;
    double* w = y + D;
    double* u = w + D;
    double* h = u + D;
    double* gt = h + D; // gradient computed at line-search trials
    double* partU = gt + D;
    double* partH = partU + Q * D;
    double* red = partH + Q * D;
    double* scratch = red + kCtaRedDoubles;
    double* trial_f = scratch + kBlock; // 2 x 32: alternate rounds
    double* trial_x = trial_f + 64 + 4; // NW x D when kWarpTrials
    CtaGroup grp{red, scratch};
    const int t = threadIdx.x;

    for (int i = t; i < D; i += kBlock)
      x[i] = x0[i];
    for (int e = t; e < D * D; e += kBlock)
      H[e] = (e / D == e % D) ? 1.0 : 0.0;
    __syncthreads();
    double best;
    if constexpr (kTrialGrad)
      best = coop_gradient<F, D, Adjoint>(f, grp, x, g);
    else {
      best = coop_value<F, D>(f, grp, x);
      coop_gradient<F, D, Adjoint>(f, grp, x, g);
    }
    __syncthreads();
    double ddir;
    bool stop;
    {
      double v[2] = {0.0, t == 0 ? (double)load_stop(ctl) : 0.0};
      for (int i = t; i < D; i += kBlock) {
        p[i] = -g[i];
        v[0] = fma(g[i], p[i], v[0]);
      }
      grp.template sum<2>(v);
      ddir = v[0];
      stop = v[1] != 0.0;
    }
    long long n_eval = 1, n_grad = 1;
    int status = kUnset, iter, executed = -1;
    double fout = best, gout = 0.0;

    for (iter = 0; iter < prm.max_iter; ++iter) {
      if (stop) {
        status = kStopped;
        break;
      }
      // ---- line search: alpha_k = 2^-k, first k in 0..19 that passes,
      // else alpha = 2^-20 (utils.cuh:376-412)
      double fnew = 0.0;
      bool have_grad = false;
      if constexpr (kWarpTrials) {
        // warp w evaluates trial k = r0 + w of each round on its own copy of
        // the trial point (shuffle reductions, no block barrier); one
        // barrier per round publishes the values, which every thread scans
        // in trial order
        const int warp = t >> 5, lane = t & 31;
        double* wx = trial_x + warp * D;
        const TileGroup<32> wg(cg::tiled_partition<32>(cg::this_thread_block()),
                               scratch + warp * 32);
        int found = -1, round = 0;
        double alpha = 0.0;
        for (int r0 = 0; found < 0; r0 += NW, ++round) {
          const int k = r0 + warp;
          double f1 = 0.0;
          if (k <= kLineSearchTrials) {
            const double ak = ldexp(1.0, -k);
            for (int i = lane; i < D; i += 32)
              wx[i] = fma(ak, p[i], x[i]);
            __syncwarp();
            f1 = coop_value<F, D>(f, wg, wx);
            __syncwarp();
          }
          double* tf = trial_f + (round & 1) * 32;
          if (lane == 0)
            tf[warp] = f1;
          __syncthreads();
          for (int w = 0; w < NW; ++w) {
            const int kk = r0 + w;
            if (kk > kLineSearchTrials)
              break;
            const double fk = tf[w], ak = ldexp(1.0, -kk);
            if (kk == kLineSearchTrials ||
                (fk <= best + kArmijoC1 * ak * ddir && fk < best)) {
              found = kk;
              fnew = fk;
              alpha = ak;
              break;
            }
          }
        }
        n_eval += found + 1;
        for (int i = t; i < D; i += kBlock)
          xn[i] = fma(alpha, p[i], x[i]);
      } else {
        double alpha = 1.0;
        for (int k = 0; k <= kLineSearchTrials; ++k) {
          for (int i = t; i < D; i += kBlock)
            xn[i] = fma(alpha, p[i], x[i]);
          __syncthreads();
          double f1;
          if constexpr (kTrialGrad)
            f1 = coop_gradient<F, D, Adjoint>(f, grp, xn, gt);
          else
            f1 = coop_value<F, D>(f, grp, xn);
          ++n_eval;
          if (k == kLineSearchTrials ||
              (f1 <= best + kArmijoC1 * alpha * ddir && f1 < best)) {
            fnew = f1;
            have_grad = kTrialGrad;
            break;
          }
          alpha *= 0.5;
          __syncthreads(); // xn fully read before the next trial writes it
        }
      }
      __syncthreads();
      if (have_grad) {
        for (int i = t; i < D; i += kBlock)
          gn[i] = gt[i];
      } else {
        coop_gradient<F, D, Adjoint>(f, grp, xn, gn);
      }
      ++n_grad;
      __syncthreads();
      const bool take = fnew < best;
      double sy_part = 0.0;
      for (int i = t; i < D; i += kBlock) {
        s[i] = xn[i] - x[i];
        y[i] = gn[i] - g[i];
        sy_part = fma(s[i], y[i], sy_part);
      }
      const double sy = grp.sum(sy_part); // (its barriers publish s, y)
      const bool skipped = fabs(sy) < kMinCurvature;
      const double* gnext = take ? gn : g;
      // sweep 1: u = H y (if updating) and h = H g_next, by columns
      {
        const int i = t % D, q = t / D;
        if (q < Q && t < Q * D) {
          double au = 0.0, ah = 0.0;
          for (int m = q; m < D; m += Q) {
            const double hv = H[m * D + i];
            ah = fma(hv, gnext[m], ah);
            if (!skipped)
              au = fma(hv, y[m], au);
          }
          partU[q * D + i] = au;
          partH[q * D + i] = ah;
        }
      }
      __syncthreads();
      double yu_part = 0.0;
      for (int i = t; i < D; i += kBlock) {
        double au = 0.0, ah = 0.0;
        for (int q = 0; q < Q; ++q) {
          au += partU[q * D + i];
          ah += partH[q * D + i];
        }
        u[i] = au;
        h[i] = ah;
        yu_part = fma(y[i], au, yu_part);
      }
      if (!skipped) {
        const double yu = grp.sum(yu_part);
        const double rho = 1.0 / sy;
        const double hb = 0.5 * rho * fma(rho, yu, 1.0);
        double wg = 0.0, sg2 = 0.0;
        for (int i = t; i < D; i += kBlock) {
          const double wi = fma(hb, s[i], -rho * u[i]);
          w[i] = wi;
          wg = fma(wi, gnext[i], wg);
          sg2 = fma(s[i], gnext[i], sg2);
        }
        double v[2] = {wg, sg2};
        grp.template sum<2>(v); // barriers publish w
        // sweep 2: H += s w^T + w s^T
        for (int e = t; e < D * D; e += kBlock) {
          const int i = e / D, j = e - (e / D) * D;
          H[e] += __dadd_rn(__dmul_rn(s[i], w[j]), __dmul_rn(w[i], s[j]));
        }
        for (int i = t; i < D; i += kBlock)
          p[i] = -(h[i] + s[i] * v[0] + w[i] * v[1]);
      } else {
        for (int i = t; i < D; i += kBlock)
          p[i] = -h[i];
      }
      if (take) {
        best = fnew;
        for (int i = t; i < D; i += kBlock) {
          x[i] = xn[i];
          g[i] = gn[i];
        }
      }
      // one reduction: ||g||, the next g.p and the stop flag for the next
      // iteration's check
      double v3[3] = {0.0, 0.0, t == 0 ? (double)load_stop(ctl) : 0.0};
      for (int i = t; i < D; i += kBlock) {
        v3[0] = fma(g[i], g[i], v3[0]);
        v3[1] = fma(g[i], p[i], v3[1]);
      }
      grp.template sum<3>(v3);
      const double gnrm = sqrt(v3[0]);
      ddir = v3[1];
      stop = v3[2] != 0.0;
      if (!isfinite(gnrm) || !isfinite(fnew)) {
        status = kNonFinite;
        fout = fnew;
        gout = gnrm;
        break;
      }
      if (gnrm < prm.tol) {
        if (t == 0)
          note_converged(ctl, prm.required);
        status = kConverged;
        fout = best;
        gout = gnrm;
        break;
      }
      if (!take && skipped && !(prm.flags & kFlagNoFixedPoint)) {
        executed = iter + 1;
        iter = prm.max_iter;
        break;
      }
    }
    if (status == kUnset || status == kStopped) {
      if (status == kUnset)
        status = kSurrender;
      fout = best;
      double gg = 0.0;
      for (int i = t; i < D; i += kBlock)
        gg = fma(g[i], g[i], gg);
      gout = sqrt(grp.sum(gg));
    }
    if (out.x)
      for (int i = t; i < D; i += kBlock)
        out.x[run * D + i] = x[i];
    if (t == 0) {
      if (out.fval)
        out.fval[run] = fout;
      if (out.status)
        out.status[run] = status;
      if (out.iter)
        out.iter[run] = iter;
      if (out.gnorm)
        out.gnorm[run] = gout;
      if (out.counters) {
        out.counters[3 * run + 0] = executed >= 0 ? executed : iter;
        out.counters[3 * run + 1] = n_eval;
        out.counters[3 * run + 2] = n_grad;
      }
    }
    __syncthreads();
  }

  template <class F, int D, bool Adjoint, int kBlock>
  __global__ void __launch_bounds__(kBlock)
    bfgs_cta_kernel(F f, BfgsParams prm, const double* __restrict__ starts,
                    RunOut out, Control* ctl)
  {
    extern __shared__ double sm[];
    for (int64_t run = blockIdx.x; run < prm.n; run += gridDim.x)
      cta_run<F, D, Adjoint, kBlock>(f, sm, prm, starts + run * D, run, out,
                                     ctl);
  }

} // namespace zb
