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
// H+ = H + s w^T + w s^T: the CTA kernel forms each product with __dmul_rn
// so that entry (i, j) and (j, i) round identically and H stays exactly
// symmetric (it reads columns as rows); the tile kernel reads its rows as
// rows and applies the update as two FMAs.
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
  // f(x + a p) = f(x) + a grad f(x).p + a^2 f(p), with value_ctx(grp, x, r)
  // giving f(x) over a shared scratch vector r (the Gaussian's 0.5 x^T C x)
  template <class F>
  concept QuadraticForm = requires { F::kQuadraticForm; };

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

  template <class F, class G>
  concept HasGradientCoop =
    requires(const F& f, const G& g, const double* x, double* gr) {
      f.gradient_coop(g, x, gr);
    };

  // g = grad f(x) without f(x): objectives with a reduction-free gradient
  // skip the value's reduction.
  template <class F, int D, bool Adjoint, class G>
  __device__ __forceinline__ void
  coop_gradient_only(const F& f, const G& grp, const double* x, double* g)
  {
    if constexpr (Adjoint && HasGradientCoop<F, G>)
      f.gradient_coop(grp, x, g);
    else
      (void)coop_gradient<F, D, Adjoint>(f, grp, x, g);
  }

  // ---------------------------------------------------------------- tile
  inline constexpr int kTileBlock = 128;

  // Per-tile shared memory (doubles): trial point xs[D] | gradient gs[D] |
  // {s, w, y, g_next}[D] | {x, p}[D] | scratch TS.
  __host__ __device__ constexpr int
  tile_buf_doubles(int d, int ts)
  {
    return 8 * d + ts;
  }
  template <int D, int TS>
  constexpr int
  tile_smem_doubles()
  {
    return tile_buf_doubles(D, TS);
  }

  // f(x + a p) evaluated by one thread from interleaved {x_i, p_i}.
  template <class F>
  concept HasValueLine = requires(const F& f, const double2* xp, double a) {
    { f.value_line(xp, a) } -> std::convertible_to<double>;
  };

  // One run on a tile: `buf` is the tile's tile_smem_doubles<D, TS>()
  // doubles of shared memory (16-byte aligned); start x0[D]; results to
  // slot `run` of `out`.
  //
  // Line search: trial 0 on the whole tile (cooperative value), then, for
  // objectives with value_line, the remaining trials lane-per-trial, TS at
  // a time, the first passing one found by a ballot (for D <= 8 every trial
  // goes lane-per-trial).  Then one pass over the H rows in registers
  // applies the previous iteration's deferred update H += s w^T + w s^T and
  // forms u = H y and h = H g_next together, and one butterfly reduction of
  // {s.y, y.u, u.g, s.g, g.h, g.g, stop} gives every scalar:
  //   p+ = -(h + s (w.g) + w (s.g)),  g.p+ = -(g.h + 2 (s.g)(w.g)).
  template <class F, int D, int TS, bool Adjoint, bool kTimed = false>
  __device__ __forceinline__ void
  tile_run(const F& f, cg::thread_block_tile<TS> tile, double* buf,
           const BfgsParams& prm, const double* __restrict__ x0, int64_t run,
           const RunOut& out, Control* ctl)
  {
    constexpr int R = (D + TS - 1) / TS;
    constexpr bool kLine = HasValueLine<F>;
    constexpr bool kCoopFirst = !kLine || D > 8;
    const int lane = (int)tile.thread_rank();
    double* xs = buf;
    double* gs = xs + D;
    double* quad = gs + D; // [D][4]: s, w, y, g_next
    double* xp = quad + 4 * D; // [D][2]: x, p
    TileGroup<TS> grp(tile, xp + 2 * D);

    double x[R], g[R], p[R], sp[R], wp[R], H[R][D];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = lane + r * TS;
      x[r] = i < D ? x0[i] : 0.0;
      if (i < D)
        xs[i] = x[r];
      sp[r] = 0.0;
      wp[r] = 0.0;
#pragma unroll
      for (int j = 0; j < D; ++j)
        H[r][j] = (i == j) ? 1.0 : 0.0;
    }
    grp.sync();
    const CycleTimer<kTimed> tm(out, run, lane == 0);
    double best = coop_value<F, D>(f, grp, xs);
    tm.start_grad();
    coop_gradient_only<F, D, Adjoint>(f, grp, xs, gs);
    grp.sync();
    tm.stop_grad();
    double ddir;
    bool stop;
    {
      double v[2] = {0.0, lane == 0 ? (double)load_stop(ctl) : 0.0};
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = lane + r * TS;
        g[r] = i < D ? gs[i] : 0.0;
        p[r] = -g[r];
        v[0] = fma(g[r], p[r], v[0]);
      }
      grp.template sum<2>(v);
      ddir = v[0];
      stop = v[1] != 0.0;
    }
    bool pend = false;
    long long n_eval = 1, n_grad = 1;
    int status = kUnset, iter, executed = -1;
    double fout = best, gout = 0.0;

    for (iter = 0; iter < prm.max_iter; ++iter) {
      if (stop) {
        status = kStopped;
        break;
      }
      // This iteration's read of the stop flag (consumed at the reduction)
      // is issued after a sync and before a stretch of arithmetic: every
      // sync waits for the thread's outstanding loads, so issued before one
      // it would stall the tile for a global-memory round trip.
      int stop_now = 0;
      // ---- line search: alpha_k = 2^-k, first k in 0..19 that passes,
      // else alpha = 2^-20 (utils.cuh:376-412)
      int found = -1;
      double fnew = 0.0;
      if constexpr (kCoopFirst) {
        grp.sync(); // earlier readers of xs are done
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = lane + r * TS;
          if (i < D)
            xs[i] = fma(1.0, p[r], x[r]);
        }
        grp.sync();
        if (lane == 0)
          stop_now = load_stop(ctl);
        const double f0 = coop_value<F, D>(f, grp, xs);
        if (f0 <= best + kArmijoC1 * ddir && f0 < best) {
          found = 0;
          fnew = f0;
        }
      }
      if (found < 0) {
        constexpr int k0 = kCoopFirst ? 1 : 0;
        if constexpr (kLine) {
          grp.sync(); // earlier readers of xp are done
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int i = lane + r * TS;
            if (i < D)
              *reinterpret_cast<double2*>(xp + 2 * i) = make_double2(x[r], p[r]);
          }
          grp.sync();
          if (!kCoopFirst && lane == 0)
            stop_now = load_stop(ctl);
          for (int base = k0; found < 0; base += TS) {
            const int k = base + lane;
            double fk = 0.0;
            bool pass = false;
            if (k <= kLineSearchTrials) {
              const double ak = pow2neg(k);
              fk = f.value_line(reinterpret_cast<const double2*>(xp), ak);
              pass = k == kLineSearchTrials ||
                     (fk <= best + kArmijoC1 * ak * ddir && fk < best);
            }
            const unsigned m = tile.ballot(pass);
            if (m) {
              const int wl = __ffs(m) - 1;
              found = base + wl;
              fnew = tile.shfl(fk, wl);
            }
          }
        } else {
          double a = pow2neg(k0);
          for (int k = k0; k <= kLineSearchTrials; ++k, a *= 0.5) {
            grp.sync();
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int i = lane + r * TS;
              if (i < D)
                xs[i] = fma(a, p[r], x[r]);
            }
            grp.sync();
            const double f1 = coop_value<F, D>(f, grp, xs);
            if (k == kLineSearchTrials ||
                (f1 <= best + kArmijoC1 * a * ddir && f1 < best)) {
              found = k;
              fnew = f1;
              break;
            }
          }
        }
      }
      n_eval += found + 1;
      const double alpha = pow2neg(found);
      double xn[R];
      grp.sync(); // readers of xs are done
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = lane + r * TS;
        xn[r] = fma(alpha, p[r], x[r]);
        if (i < D)
          xs[i] = xn[r];
      }
      grp.sync();
      tm.start_grad();
      coop_gradient_only<F, D, Adjoint>(f, grp, xs, gs);
      ++n_grad;
      grp.sync();
      tm.stop_grad();
      const bool take = fnew < best;
      double gn[R], s[R], y[R], gx[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = lane + r * TS;
        gn[r] = i < D ? gs[i] : 0.0;
        s[r] = xn[r] - x[r];
        y[r] = gn[r] - g[r];
        gx[r] = take ? gn[r] : g[r];
        if (i < D)
          *reinterpret_cast<double2*>(quad + 4 * i + 2) = make_double2(y[r], gx[r]);
      }
      grp.sync();
      // ---- one pass: deferred update, u = H y, h = H g_next (even and odd
      // columns in separate sums: half the chain of dependent FMAs)
      tm.start_update();
      double u[R], hh[R];
      {
        double ua[R][2], ha[R][2];
#pragma unroll
        for (int r = 0; r < R; ++r)
          ua[r][0] = ua[r][1] = ha[r][0] = ha[r][1] = 0.0;
        if (pend) {
#pragma unroll
          for (int j = 0; j < D; ++j) {
            const double2 sw = *reinterpret_cast<const double2*>(quad + 4 * j);
            const double2 yg = *reinterpret_cast<const double2*>(quad + 4 * j + 2);
#pragma unroll
            for (int r = 0; r < R; ++r) {
              // rows are read as rows here: two FMAs, no symmetric rounding
              H[r][j] = fma(sp[r], sw.y, fma(wp[r], sw.x, H[r][j]));
              ua[r][j & 1] = fma(H[r][j], yg.x, ua[r][j & 1]);
              ha[r][j & 1] = fma(H[r][j], yg.y, ha[r][j & 1]);
            }
          }
        } else {
#pragma unroll
          for (int j = 0; j < D; ++j) {
            const double2 yg = *reinterpret_cast<const double2*>(quad + 4 * j + 2);
#pragma unroll
            for (int r = 0; r < R; ++r) {
              ua[r][j & 1] = fma(H[r][j], yg.x, ua[r][j & 1]);
              ha[r][j & 1] = fma(H[r][j], yg.y, ha[r][j & 1]);
            }
          }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
          u[r] = ua[r][0] + ua[r][1];
          hh[r] = ha[r][0] + ha[r][1];
        }
      }
      double v[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, (double)stop_now};
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = lane + r * TS;
        if (i < D) {
          v[0] = fma(s[r], y[r], v[0]);
          v[1] = fma(y[r], u[r], v[1]);
          v[2] = fma(u[r], gx[r], v[2]);
          v[3] = fma(s[r], gx[r], v[3]);
          v[4] = fma(gx[r], hh[r], v[4]);
          v[5] = fma(gx[r], gx[r], v[5]);
        }
      }
      grp.template sum<7>(v);
      const bool skipped = fabs(v[0]) < kMinCurvature;
      const double sg = v[3], gh = v[4];
      double rho = 0.0, hb = 0.0, wg = 0.0;
      if (!skipped) {
        rho = 1.0 / v[0];
        hb = 0.5 * rho * fma(rho, v[1], 1.0);
        wg = hb * sg - rho * v[2];
      }
      grp.sync(); // every lane's pass has read quad
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = lane + r * TS;
        if (!skipped) {
          const double w = fma(hb, s[r], -rho * u[r]);
          p[r] = -(hh[r] + s[r] * wg + w * sg);
          sp[r] = s[r];
          wp[r] = w;
          if (i < D)
            *reinterpret_cast<double2*>(quad + 4 * i) = make_double2(s[r], w);
        } else {
          p[r] = -hh[r];
        }
      }
      tm.stop_update();
      pend = !skipped;
      ddir = skipped ? -gh : -(gh + 2.0 * sg * wg);
      stop = v[6] != 0.0;
      if (take) {
        best = fnew;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          x[r] = xn[r];
          g[r] = gn[r];
        }
      }
      const double gnrm = sqrt(v[5]);
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
      tm.finish();
    }
    grp.sync();
  }

  template <class F, int D, int TS, bool Adjoint, bool kTimed = false>
  __global__ void __launch_bounds__(kTileBlock)
    bfgs_tile_kernel(F f, BfgsParams prm, const double* __restrict__ starts,
                     RunOut out, Control* ctl)
  {
    constexpr int TPB = kTileBlock / TS;
    extern __shared__ __align__(16) double sm[];
    auto tile = cg::tiled_partition<TS>(cg::this_thread_block());
    const int tslot = threadIdx.x / TS;
    const int64_t run = (int64_t)blockIdx.x * TPB + tslot;
    if (run >= prm.n)
      return; // the whole tile leaves together
    tile_run<F, D, TS, Adjoint, kTimed>(f, tile, sm + tslot * tile_smem_doubles<D, TS>(),
                                        prm, starts + run * D, run, out, ctl);
  }

  // ---------------------------------------------------------------- CTA
  // One run on the whole thread block, H in shared memory (D x D doubles,
  // exactly symmetric).  An iteration meets at four block barriers:
  //
  //   1. line search: warp w evaluates trial k = r0 + w of a round on its own
  //      copy of the trial point (shuffle reductions only); one barrier
  //      publishes the round's values and every warp finds the first passing
  //      trial with one ballot.  (Objectives whose trials carry the gradient
  //      -- the Gaussian's C x -- evaluate trials one at a time on the whole
  //      block.)
  //   2. gradient at the accepted point.
  //   3. one sweep over H: it applies the previous iteration's deferred
  //      rank-2 update H += s w^T + w s^T in place and forms the column
  //      partial sums of u = H y and h = H g_next (C = 2 columns per thread
  //      with 16-byte accesses, Q = blockDim / (D / C) groups of rows).
  //   4. one block reduction of {s.y, y.u, u.g, s.g, g.h, g.g, stop}; every
  //      scalar of the update follows from it:
  //        w = hb s - rho u,  w.g = hb (s.g) - rho (u.g),
  //        p+ = -H+ g = -(h + s (w.g) + w (s.g)),  g.p+ = -(g.h + 2 (s.g)(w.g)).
  //
  // x, p and the accepted point stay in registers, replicated in every warp
  // (lane l holds coordinates l, l+32, ...): each warp forms the same p+
  // from u and h in shared memory, so no barrier publishes p.
  template <int D>
  struct CtaShape {
    static constexpr int C = (D % 2 == 0) ? 2 : 1; // sweep columns per thread
    static constexpr int NCOL = D / C;
    static constexpr int RV = (D + 31) / 32; // coordinates per lane
  };

  __host__ __device__ constexpr int
  cta_sweep_q(int d, int block)
  {
    const int ncol = (d % 2 == 0) ? d / 2 : d;
    return block >= ncol ? block / ncol : 1;
  }

  // Rows of H per thread in the sweep; with at most 8 (16 doubles) H lives
  // in the sweep threads' registers instead of shared memory (D = 64 at
  // 256-512 threads): the sweep then moves no H bytes at all.
  __host__ __device__ constexpr int
  cta_rows_per_thread(int d, int block)
  {
    const int q = cta_sweep_q(d, block);
    return (d + q - 1) / q;
  }
  // D <= 64, D % 8 == 0: column-warps. Warp w < D/8 owns columns
  // 8w .. 8w+7; its four lane quarters take rows q, q+4, ... (D/4 doubles
  // of H per lane), and a column's four partial sums meet by two shuffles:
  // no partial sums in shared memory and no barrier after the sweep.
  __host__ __device__ constexpr bool
  cta_col_warps(int d, int block)
  {
    return d % 8 == 0 && d <= 64 && d / 8 <= block / 32;
  }
  __host__ __device__ constexpr bool
  cta_h_in_registers(int d, int block)
  {
    return cta_col_warps(d, block) ||
           (d % 2 == 0 && cta_rows_per_thread(d, block) <= 8);
  }

  // Everything in shared memory but H and the trial points.
  __host__ __device__ constexpr size_t
  cta_vec_doubles(int d, int block)
  {
    const int q = cta_sweep_q(d, block);
    return 7 * (size_t)d + 2 * (size_t)q * d + (size_t)d + 64 + kCtaRedDoubles + block;
  }

  // Past about D = 160 H no longer fits in shared memory beside the vectors
  // (even with the fewest trial points): it lives in a global-memory slice
  // per block (D*D doubles, L2-resident for the blocks in flight -- 148
  // slices of a 256-D H are 78 MB of the 126 MB L2) and the sweep streams
  // it with the same coalesced 16-byte row accesses.
  __host__ __device__ constexpr bool
  cta_h_global(int d, int block)
  {
    return !cta_h_in_registers(d, block) &&
           ((((size_t)d * d + 1) & ~(size_t)1) + cta_vec_doubles(d, block) +
            (size_t)(block / 32) * d) * sizeof(double) > 227 * 1024;
  }

  // Shared-memory layout (doubles): H[D*D, rounded up to even; none when H
  // is in registers or in global memory] | {s,w}[D] | g[2][D] | u[D] | h[D]
  // | x[D] | partial sums 2*Q*D | trial point D | (group trials) one trial
  // point per trial group | trial values 2*32 | reductions | scratch
  // blockDim.
  __host__ __device__ constexpr size_t
  cta_smem_base_doubles(int d, int block)
  {
    return (cta_h_in_registers(d, block) || cta_h_global(d, block)
              ? 0
              : (((size_t)d * d + 1) & ~(size_t)1)) +
           cta_vec_doubles(d, block);
  }

  // Lanes per line-search trial group: the widest of 32, 16, 8 that gives
  // the block at least 21 groups (every trial of a line search in one
  // round), narrower only while the trial points fit in shared memory.
  __host__ __device__ constexpr int
  cta_trial_width(int d, int block)
  {
    const int nw = block / 32;
    const size_t cap = 227 * 1024 / sizeof(double);
    int st = nw >= 21 ? 32 : 2 * nw >= 21 ? 16 : 8;
    while (st < 32 &&
           cta_smem_base_doubles(d, block) + (size_t)nw * (32 / st) * d > cap)
      st *= 2;
    return st;
  }

  __host__ __device__ constexpr size_t
  cta_smem_doubles_rt(int d, int block, bool warp_trials)
  {
    return cta_smem_base_doubles(d, block) +
           (warp_trials ? (size_t)(block / 32) * (32 / cta_trial_width(d, block)) * d
                        : 0);
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

  // The first line-search trial k (alpha = 2^-k) that passes the
  // reference's test on the quadratic model f(alpha) = f0 + alpha gp +
  // alpha^2 fp, else kLineSearchTrials: lane k judges trial k, one ballot
  // picks the lowest.  Every warp of a block gets the same answer.
  __device__ __forceinline__ int
  model_trial(double f0, double gp, double fp, int lane)
  {
    bool pass = false;
    if (lane <= kLineSearchTrials) {
      const double ak = pow2neg(lane);
      const double fk = f0 + ak * fma(ak, fp, gp);
      pass = lane == kLineSearchTrials ||
             (fk <= f0 + kArmijoC1 * ak * gp && fk < f0);
    }
    return __ffs(__ballot_sync(0xffffffffu, pass)) - 1;
  }

  __device__ __forceinline__ double
  warp_allsum(double v)
  {
#pragma unroll
    for (int m = 16; m > 0; m >>= 1)
      v += __shfl_xor_sync(0xffffffffu, v, m);
    return v;
  }

  // One run on the whole block (blockDim.x == kBlock): `sm` holds
  // cta_smem_doubles<F, D, Adjoint>(kBlock) doubles, 16-byte aligned; start
  // x0[D]; results to slot `run`.
  template <class F, int D, bool Adjoint, int kBlock, bool kTimed = false>
  __device__ __forceinline__ void
  cta_run(const F& f, double* sm, const BfgsParams& prm,
          const double* __restrict__ x0, int64_t run, const RunOut& out,
          Control* ctl, double* __restrict__ hglob = nullptr)
  {
    using S = CtaShape<D>;
    constexpr int C = S::C, NCOL = S::NCOL, RV = S::RV;
    constexpr int Q = cta_sweep_q(D, kBlock);
    constexpr bool kTrialGrad = Adjoint && TrialsWithGradient<F>;
    constexpr bool kWarpTrials = cta_warp_trials<F, Adjoint>();
    constexpr int NW = kBlock / 32;
    constexpr int ST = cta_trial_width(D, kBlock); // lanes per trial group
    constexpr int TPW = 32 / ST;                   // trial groups per warp
    constexpr int NG = NW * TPW;
    static_assert(kBlock % 32 == 0 && NCOL <= kBlock, "block too small for D");
    static_assert(NG <= 32, "one ballot judges a round");
    static_assert(RV <= NW, "one warp per 32 coordinates at least");
    constexpr bool kColWarp = cta_col_warps(D, kBlock);
    constexpr bool kHReg = cta_h_in_registers(D, kBlock) && !kColWarp;
    constexpr int RQ = cta_rows_per_thread(D, kBlock);
    constexpr bool kHGlob = cta_h_global(D, kBlock);
    // H: shared memory, or this block's global slice `hglob` (16 B aligned)
    double* H = kHGlob ? hglob : sm;
    // {s_i, w_i} of the deferred update (16 B aligned)
    double* SW = sm + (kHReg || kColWarp || kHGlob ? 0 : ((D * D + 1) & ~1));
    double* gb = SW + 2 * D;    // two gradient slots of D
    double* u = gb + 2 * D;
    double* h = u + D;
    double* xcur = h + D; // x, for the column-warp sweep
    double* partU = xcur + D;
    double* partH = partU + Q * D;
    double* xt = partH + Q * D; // block trial point / start
    double* trial_x = xt + D;   // NG x D when kWarpTrials
    double* tf = trial_x + (kWarpTrials ? NG * D : 0); // 2 x 32
    double* red = tf + 64;
    double* scratch = red + kCtaRedDoubles;
    CtaGroup grp{red, scratch};
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;

    double xr[RV], pr[RV], xnr[RV];
#pragma unroll
    for (int r = 0; r < RV; ++r) {
      const int i = lane + 32 * r;
      xr[r] = i < D ? x0[i] : 0.0;
      pr[r] = 0.0;
      xnr[r] = 0.0;
    }
    for (int i = t; i < D; i += kBlock)
      xt[i] = x0[i];
    // H = I; with kHReg thread (c, q) keeps rows q, q+Q, ... of columns
    // C*c .. C*c+C-1 in Hr
    double Hr[kHReg ? RQ : 1][C];
    {
      const int c = t % NCOL, q = t / NCOL;
#pragma unroll
      for (int r = 0; r < (kHReg ? RQ : 1); ++r)
#pragma unroll
        for (int j = 0; j < C; ++j)
          Hr[r][j] = (q + Q * r == C * c + j) ? 1.0 : 0.0;
    }
    // with kColWarp lane (w, l) keeps rows q, q+4, ... (q = l / 8) of
    // column 8w + l % 8 in Hc
    double Hc[kColWarp ? D / 4 : 1];
#pragma unroll
    for (int k = 0; k < (kColWarp ? D / 4 : 1); ++k)
      Hc[k] = (4 * k + (lane >> 3) == warp * 8 + (lane & 7)) ? 1.0 : 0.0;
    if constexpr (!kHReg && !kColWarp)
      for (int e = t; e < D * D; e += kBlock)
        H[e] = (e / D == e % D) ? 1.0 : 0.0;
    for (int i = t; i < D; i += kBlock)
      xcur[i] = x0[i];
    __syncthreads();
    int cur = 0; // current gradient in slot cur, the new one goes to cur ^ 1
    const CycleTimer<kTimed> tm(out, run, t == 0);
    double best;
    tm.start_grad();
    if constexpr (kTrialGrad)
      best = coop_gradient<F, D, Adjoint>(f, grp, xt, gb);
    else {
      best = coop_value<F, D>(f, grp, xt);
      coop_gradient_only<F, D, Adjoint>(f, grp, xt, gb);
    }
    __syncthreads();
    tm.stop_grad();
    double ddir;
    bool stop;
    {
      double v[2] = {0.0, t == 0 ? (double)load_stop(ctl) : 0.0};
      if (t < D)
        v[0] = fma(gb[t], -gb[t], 0.0);
      grp.template sum<2>(v);
      ddir = v[0];
      stop = v[1] != 0.0;
#pragma unroll
      for (int r = 0; r < RV; ++r) {
        const int i = lane + 32 * r;
        if (i < D)
          pr[r] = -gb[i];
      }
    }
    long long n_eval = 1, n_grad = 1;
    // the symmetric quadratic form carries f and g one step from C x (see
    // the line search); where a run ends, they are formed exactly at x:
    // f into fd, ||g|| into gd, g into the current slot
    const auto exact_at_x = [&](int slot, double& fd, double& gd) {
      double* gc = gb + slot * D;
      __syncthreads(); // gc and xcur no longer read
      if (warp == 0) {
#pragma unroll
        for (int r = 0; r < RV; ++r) {
          const int i = lane + 32 * r;
          if (i < D)
            xcur[i] = xr[r];
        }
      }
      __syncthreads();
      if constexpr (QuadraticForm<F>)
        fd = f.value_ctx(grp, xcur, gc);
      double v1[1] = {t < D ? gc[t] * gc[t] : 0.0};
      grp.template sum<1>(v1);
      gd = sqrt(v1[0]);
      ++n_eval;
    };
    bool carried = false; // f and g of this run are carried (symmetric quadratic)
    if constexpr (QuadraticForm<F>)
      carried = f.symmetric;
    int status = kUnset, iter, executed = -1;
    double fout = best, gout = 0.0;
    bool pend = false; // SW holds an update not yet applied to H

    for (iter = 0; iter < prm.max_iter; ++iter) {
      if (stop) {
        status = kStopped;
        break;
      }
      // this iteration's read of the stop flag, consumed at the reduction:
      // issued after the line search's first sync, before a stretch of
      // arithmetic (every barrier waits for the thread's outstanding loads)
      int stop_now = 0;
      // ---- line search: alpha_k = 2^-k, first k in 0..19 that passes,
      // else alpha = 2^-20 (utils.cuh:376-412)
      double fnew = 0.0, alpha = 1.0;
      const double* xn_s = xt; // accepted point in shared memory
      if constexpr (kWarpTrials) {
        // trial group g = warp * TPW + sub (ST lanes) evaluates trial
        // k = r0 + g of each round on its own copy of the trial point; the
        // warp writes its TPW trial points from its registers
        double* wx = trial_x + warp * TPW * D;
        const int sub = lane / ST;
        const TileGroup<ST> sg(cg::tiled_partition<ST>(cg::this_thread_block()),
                               scratch + warp * 32 + sub * ST);
        int found = -1;
        for (int r0 = 0, round = 0; found < 0; r0 += NG, ++round) {
#pragma unroll
          for (int q = 0; q < TPW; ++q) {
            const int k = r0 + warp * TPW + q;
            if (k <= kLineSearchTrials) {
              const double ak = pow2neg(k);
#pragma unroll
              for (int r = 0; r < RV; ++r) {
                const int i = lane + 32 * r;
                if (i < D)
                  wx[q * D + i] = fma(ak, pr[r], xr[r]);
              }
            }
          }
          __syncwarp();
          if (round == 0 && t == 0)
            stop_now = load_stop(ctl);
          const int k = r0 + warp * TPW + sub;
          double f1 = 0.0;
          if (k <= kLineSearchTrials) // uniform within the group
            f1 = coop_value<F, D>(f, sg, wx + sub * D);
          double* tfr = tf + (round & 1) * 32;
          if (sg.rank() == 0)
            tfr[warp * TPW + sub] = f1;
          __syncthreads();
          // lane l judges trial r0 + l; the lowest passing trial wins
          const int kk = r0 + lane;
          bool pass = false;
          double fk = 0.0;
          if (lane < NG && kk <= kLineSearchTrials) {
            fk = tfr[lane];
            const double ak = pow2neg(kk);
            pass = kk == kLineSearchTrials ||
                   (fk <= best + kArmijoC1 * ak * ddir && fk < best);
          }
          const unsigned m = __ballot_sync(0xffffffffu, pass);
          if (m) {
            const int wl = __ffs(m) - 1;
            found = r0 + wl;
            fnew = __shfl_sync(0xffffffffu, fk, wl);
            alpha = pow2neg(found);
            xn_s = trial_x + wl * D;
          }
        }
        n_eval += found + 1;
      } else {
        double* gt = gb + (cur ^ 1) * D;
        int k0 = 0;
        bool searched = false;
        if constexpr (QuadraticForm<F>) {
          if (f.symmetric) {
            // C x and C p in one pass over C: f(x), f(p) and g.p, exact at
            // this iteration's x, decide every trial; the accepted point's
            // gradient is g + alpha C p and its value f(x) + alpha g.p +
            // alpha^2 f(p).  g is formed afresh from C x every iteration,
            // so these carry one step's rounding, never an accumulation.
            double* gc = gb + cur * D;
            if (warp == 0) {
#pragma unroll
              for (int r = 0; r < RV; ++r) {
                const int i = lane + 32 * r;
                if (i < D) {
                  xt[i] = pr[r];
                  xcur[i] = xr[r];
                }
              }
            }
            __syncthreads();
            if (t == 0)
              stop_now = load_stop(ctl);
            f.ctx2_coop(grp, xcur, xt, gc, gt, partU, partH);
            double v3[3] = {0.0, 0.0, 0.0};
            if (t < D) {
              v3[0] = xcur[t] * gc[t];
              v3[1] = xt[t] * gt[t];
              v3[2] = gc[t] * xt[t];
            }
            grp.template sum<3>(v3);
            best = 0.5 * v3[0];
            const double fp = 0.5 * v3[1];
            ddir = v3[2];
            n_eval += 2;
            k0 = model_trial(best, ddir, fp, lane);
            alpha = pow2neg(k0);
            fnew = best + alpha * fma(alpha, fp, ddir);
            if (t < D) // this thread read gt[t] and gc[t] above, no one else
              gt[t] = fma(alpha, gt[t], gc[t]);
            if constexpr (kColWarp) {
              __syncthreads(); // xt fully read
              if (warp == 0) {
#pragma unroll
                for (int r = 0; r < RV; ++r) {
                  const int i = lane + 32 * r;
                  if (i < D)
                    xt[i] = fma(alpha, pr[r], xr[r]);
                }
              }
            }
            searched = true;
          }
        }
        if constexpr (QuadraticForm<F>) {
          if (!searched) {
            // (non-symmetric C: g needs C x and C^T x) f along the line is
            // best + a ddir + a^2 f(p): one pass over the objective's data
            // for f(p), then the first passing trial is found without
            // evaluating f; only that trial is evaluated (it carries the
            // new gradient), and should its true value fail the test the
            // search goes on trial by trial from there
            if (warp == 0) {
#pragma unroll
              for (int r = 0; r < RV; ++r) {
                const int i = lane + 32 * r;
                if (i < D)
                  xt[i] = pr[r];
              }
            }
            __syncthreads();
            if (t == 0)
              stop_now = load_stop(ctl);
            const double fp = f.value_ctx(grp, xt, gt);
            ++n_eval;
            k0 = model_trial(best, ddir, fp, lane);
            alpha = pow2neg(k0);
            __syncthreads(); // xt and gt fully read before the trial writes them
          }
        }
        for (int k = k0; !searched && k <= kLineSearchTrials; ++k) {
          if (warp == 0) {
#pragma unroll
            for (int r = 0; r < RV; ++r) {
              const int i = lane + 32 * r;
              if (i < D)
                xt[i] = fma(alpha, pr[r], xr[r]);
            }
          }
          __syncthreads();
          if (k == 0 && t == 0 && !QuadraticForm<F>)
            stop_now = load_stop(ctl);
          double f1;
          if constexpr (kTrialGrad)
            f1 = coop_gradient<F, D, Adjoint>(f, grp, xt, gt);
          else
            f1 = coop_value<F, D>(f, grp, xt);
          ++n_eval;
          if (k == kLineSearchTrials ||
              (f1 <= best + kArmijoC1 * alpha * ddir && f1 < best)) {
            fnew = f1;
            break;
          }
          alpha *= 0.5;
          __syncthreads(); // xt fully read before the next trial writes it
        }
      }
#pragma unroll
      for (int r = 0; r < RV; ++r) // the accepted point, bit for bit
        xnr[r] = fma(alpha, pr[r], xr[r]);
      double* gn = gb + (cur ^ 1) * D;
      const double* g = gb + cur * D;
      tm.start_grad();
      if constexpr (!kTrialGrad)
        coop_gradient_only<F, D, Adjoint>(f, grp, xn_s, gn);
      ++n_grad;
      __syncthreads();
      tm.stop_grad();
      const bool take = fnew < best;
      const double* gx = take ? gn : g; // the gradient p+ is formed for

      // ---- sweep: deferred update + column sums of H y and H g_next, and
      // the seven values of the iteration's one reduction
      tm.start_update();
      double v[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      if constexpr (kColWarp) {
        if (warp < D / 8) {
          const int i = warp * 8 + (lane & 7), q = lane >> 3;
          const double si = pend ? SW[2 * i] : 0.0, wi = pend ? SW[2 * i + 1] : 0.0;
          double au2[2] = {0.0, 0.0}, ah2[2] = {0.0, 0.0};
#pragma unroll
          for (int k = 0; k < D / 4; ++k) {
            const int m = 4 * k + q;
            const double go = g[m], gnm = gn[m];
            const double gm = take ? gnm : go, ym = gnm - go;
            if (pend) {
              const double2 sw = *reinterpret_cast<const double2*>(SW + 2 * m);
              Hc[k] += __dadd_rn(__dmul_rn(sw.x, wi), __dmul_rn(sw.y, si));
            }
            ah2[k & 1] = fma(Hc[k], gm, ah2[k & 1]);
            au2[k & 1] = fma(Hc[k], ym, au2[k & 1]);
          }
          double uu = au2[0] + au2[1], hh = ah2[0] + ah2[1];
          uu += __shfl_xor_sync(0xffffffffu, uu, 8);
          hh += __shfl_xor_sync(0xffffffffu, hh, 8);
          uu += __shfl_xor_sync(0xffffffffu, uu, 16);
          hh += __shfl_xor_sync(0xffffffffu, hh, 16);
          if (q == 0) {
            u[i] = uu;
            h[i] = hh;
            const double st = xn_s[i] - xcur[i]; // the registers' s_i, bit for bit
            const double yt = gn[i] - g[i], gt = gx[i];
            v[0] = st * yt;
            v[1] = yt * uu;
            v[2] = uu * gt;
            v[3] = st * gt;
            v[4] = gt * hh;
            v[5] = gt * gt;
          }
        }
      } else {
        const int c = t % NCOL, q = t / NCOL;
        if (q < Q) {
          const int i0 = C * c;
          double si[C], wi[C], au[C], ah[C];
#pragma unroll
          for (int j = 0; j < C; ++j) {
            si[j] = pend ? SW[2 * (i0 + j)] : 0.0;
            wi[j] = pend ? SW[2 * (i0 + j) + 1] : 0.0;
            au[j] = 0.0;
            ah[j] = 0.0;
          }
          if constexpr (kHReg) {
#pragma unroll
            for (int r = 0; r < RQ; ++r) {
              const int m = q + Q * r;
              if (m < D) {
                const double go = g[m], gnm = gn[m];
                const double gm = take ? gnm : go, ym = gnm - go;
                if (pend) {
                  const double2 sw = *reinterpret_cast<const double2*>(SW + 2 * m);
#pragma unroll
                  for (int j = 0; j < C; ++j)
                    Hr[r][j] +=
                      __dadd_rn(__dmul_rn(sw.x, wi[j]), __dmul_rn(sw.y, si[j]));
                }
#pragma unroll
                for (int j = 0; j < C; ++j) {
                  ah[j] = fma(Hr[r][j], gm, ah[j]);
                  au[j] = fma(Hr[r][j], ym, au[j]);
                }
              }
            }
          } else if (pend) {
#pragma unroll 4
            for (int m = q; m < D; m += Q) {
              const double2 sw = *reinterpret_cast<const double2*>(SW + 2 * m);
              const double go = g[m], gnm = gn[m];
              const double gm = take ? gnm : go, ym = gnm - go;
              double* row = H + m * D + i0;
              double hv[C];
              if constexpr (C == 2) {
                const double2 v2 = *reinterpret_cast<const double2*>(row);
                hv[0] = v2.x;
                hv[1] = v2.y;
              } else {
                hv[0] = row[0];
              }
#pragma unroll
              for (int j = 0; j < C; ++j)
                hv[j] += __dadd_rn(__dmul_rn(sw.x, wi[j]), __dmul_rn(sw.y, si[j]));
              if constexpr (C == 2)
                *reinterpret_cast<double2*>(row) = make_double2(hv[0], hv[1]);
              else
                row[0] = hv[0];
#pragma unroll
              for (int j = 0; j < C; ++j) {
                ah[j] = fma(hv[j], gm, ah[j]);
                au[j] = fma(hv[j], ym, au[j]);
              }
            }
          } else {
#pragma unroll 4
            for (int m = q; m < D; m += Q) {
              const double go = g[m], gnm = gn[m];
              const double gm = take ? gnm : go, ym = gnm - go;
              const double* row = H + m * D + i0;
              double hv[C];
              if constexpr (C == 2) {
                const double2 v2 = *reinterpret_cast<const double2*>(row);
                hv[0] = v2.x;
                hv[1] = v2.y;
              } else {
                hv[0] = row[0];
              }
#pragma unroll
              for (int j = 0; j < C; ++j) {
                ah[j] = fma(hv[j], gm, ah[j]);
                au[j] = fma(hv[j], ym, au[j]);
              }
            }
          }
#pragma unroll
          for (int j = 0; j < C; ++j) {
            partU[q * D + i0 + j] = au[j];
            partH[q * D + i0 + j] = ah[j];
          }
        }
      __syncthreads();

      // ---- the seven values from the column partial sums
      if (t < D) { // coordinate t is slot r = warp of this lane
        double uu = 0.0, hh = 0.0;
#pragma unroll 4
        for (int q = 0; q < Q; ++q) {
          uu += partU[q * D + t];
          hh += partH[q * D + t];
        }
        u[t] = uu;
        h[t] = hh;
        double st = 0.0;
#pragma unroll
        for (int r = 0; r < RV; ++r)
          if (r == warp)
            st = xnr[r] - xr[r];
        const double yt = gn[t] - g[t], gt = gx[t];
        v[0] = st * yt;
        v[1] = yt * uu;
        v[2] = uu * gt;
        v[3] = st * gt;
        v[4] = gt * hh;
        v[5] = gt * gt;
      }
      } // column-warp / shared-memory sweep
      v[6] = (double)stop_now;
      grp.template sum<7>(v); // its barrier publishes u and h
      const bool skipped = fabs(v[0]) < kMinCurvature;
      const double sg = v[3], gh = v[4];
      double rho = 0.0, hb = 0.0, wg = 0.0;
      if (!skipped) {
        rho = 1.0 / v[0];
        hb = 0.5 * rho * fma(rho, v[1], 1.0);
        wg = hb * sg - rho * v[2];
      }
#pragma unroll
      for (int r = 0; r < RV; ++r) {
        const int i = lane + 32 * r;
        if (i < D) {
          const double si = xnr[r] - xr[r];
          if (!skipped) {
            const double wi = fma(hb, si, -rho * u[i]);
            pr[r] = -(h[i] + si * wg + wi * sg);
            if (warp == 0)
              *reinterpret_cast<double2*>(SW + 2 * i) = make_double2(si, wi);
          } else {
            pr[r] = -h[i];
          }
        }
        if (take) {
          xr[r] = xnr[r];
          if (kColWarp && warp == 0 && i < D)
            xcur[i] = xnr[r];
        }
      }
      tm.stop_update();
      pend = !skipped;
      ddir = skipped ? -gh : -(gh + 2.0 * sg * wg);
      stop = v[6] != 0.0;
      if (take) {
        best = fnew;
        cur ^= 1;
      }
      const double gnrm = sqrt(v[5]);
      if (!isfinite(gnrm) || !isfinite(fnew)) {
        status = kNonFinite;
        fout = fnew;
        gout = gnrm;
        break;
      }
      if (gnrm < prm.tol) {
        double fd = best, gd = gnrm;
        if (carried) {
          // converged on the carried gradient: confirm on the exact one
          exact_at_x(cur, fd, gd);
          best = fd;
          if (!(gd < prm.tol))
            continue;
        }
        if (t == 0)
          note_converged(ctl, prm.required);
        status = kConverged;
        fout = fd;
        gout = gd;
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
      if (carried) {
        exact_at_x(cur, fout, gout);
      } else {
        double gg = 0.0;
        const double* g = gb + cur * D;
        for (int i = lane; i < D; i += 32)
          gg = fma(g[i], g[i], gg);
        gout = sqrt(warp_allsum(gg));
      }
    }
    if (warp == 0 && out.x) {
#pragma unroll
      for (int r = 0; r < RV; ++r) {
        const int i = lane + 32 * r;
        if (i < D)
          out.x[run * D + i] = xr[r];
      }
    }
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
      tm.finish();
    }
    __syncthreads();
  }

  // `hws`: gridDim.x slices of D*D doubles when cta_h_global(D, kBlock),
  // else unused.  `queue` (zeroed before the launch): block b runs run b,
  // then takes runs gridDim.x, gridDim.x + 1, ... from the counter as it
  // finishes them, so a long run does not hold back runs statically queued
  // behind it; without a queue, block b runs b, b + gridDim.x, ...
  template <class F, int D, bool Adjoint, int kBlock, bool kTimed = false>
  __global__ void __launch_bounds__(kBlock)
    bfgs_cta_kernel(F f, BfgsParams prm, const double* __restrict__ starts,
                    RunOut out, Control* ctl, double* __restrict__ hws = nullptr,
                    unsigned long long* queue = nullptr)
  {
    extern __shared__ __align__(16) double sm[];
    double* hg = hws ? hws + (size_t)blockIdx.x * D * D : nullptr;
    int64_t run = blockIdx.x;
    while (run < prm.n) {
      cta_run<F, D, Adjoint, kBlock, kTimed>(f, sm, prm, starts + run * D, run, out,
                                             ctl, hg);
      if (!queue) {
        run += gridDim.x;
        continue;
      }
      // the run's shared memory is dead after its final barrier: the next
      // index goes through sm[0], fenced by one barrier on each side
      if (threadIdx.x == 0)
        reinterpret_cast<long long*>(sm)[0] =
          (long long)gridDim.x + (long long)atomicAdd(queue, 1ull);
      __syncthreads();
      run = reinterpret_cast<const long long*>(sm)[0];
      __syncthreads();
    }
  }

} // namespace zb
