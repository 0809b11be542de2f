// Fast BFGS with the inverse Hessian in registers, one optimisation per group
// of NT = S * D threads (the "row" layout, for mid-to-large D where H fits
// the register file: D = 64 at S = 2, D = 128 at S = 3 or 4).
//
// Thread t of the group owns row r = t % D of H and segment c = t / D of
// its columns, [c * CW, c * CW + CW), CW = ceil(D / S): CW doubles of H in
// registers, no shared-memory traffic for H at all.  Several groups share a
// block (named barriers 1..15), so that a block runs several independent
// optimisations at once and the latency of one run's barriers and
// reductions overlaps the others' arithmetic.
//
// An iteration (the reference's semantics, bfgs_sequential.cuh:99-219):
//   1. line search: the group's warps split into trial groups of ST lanes,
//      enough for all 21 trials (alpha = 2^-k, k = 0..20) in one round; each
//      evaluates f at its materialised trial point; one barrier publishes
//      the values and a ballot in every warp picks the first passing trial
//      (c1 = 0.1, strict decrease; trial 20 is taken when none passes);
//   2. the gradient at the accepted point (its trial point, already in
//      shared memory, is the same bits as fma(alpha, p, x));
//   3. one pass over the registers: the previous iteration's deferred
//      rank-2 update H_rj += s_r w_j + w_r s_j (two FMAs; each thread reads
//      its row as a row, so exact symmetry is not needed) and the partial
//      row sums of u = H y and h = H g_x; the S partials of a row meet in
//      shared memory;
//   4. one group reduction of {s.y, y.u, u.g, s.g, g.h, g.g, stop}, from
//      which p+ = -(h + s (w.g) + w (s.g)) and g.p+ follow without a
//      second pass over H (w = hb s - rho u, rho = 1/s.y, hb = rho (1 +
//      rho y.u) / 2); the update is skipped when |s.y| < 1e-14.
// Accept-if-better, the fixed-point exit and the termination protocol are
// those of the thread, tile and CTA layouts.
#pragma once

#include "zb_bfgs_coop.cuh"
#include "zb_common.cuh"
#include "zb_group.cuh"

namespace zb {

  // lanes per line-search trial group for a group of nw warps: the widest
  // that still gives the 21 trials a group each (one round)
  __host__ __device__ constexpr int
  row_trial_width(int nw)
  {
    return nw >= 21 ? 32 : 2 * nw >= 21 ? 16 : 4 * nw >= 21 ? 8 : 8 * nw >= 21 ? 4 : 2;
  }

  // Shared memory of one group (doubles): x | p | g[2] | {s, w, y, g_x}[D]
  // | row partial sums 2 x S x D (S > 1) | trial points NG x D | trial
  // values 32 | reductions | scratch NT | run slot 2.  Every part is an
  // even number of doubles, so the parts stay 16-byte aligned.
  __host__ __device__ constexpr int
  row_smem_doubles_rt(int d, int s)
  {
    const int nt = s * d, nw = nt / 32, de = (d + 1) & ~1;
    const int ng = nw * (32 / row_trial_width(nw));
    return 4 * de + 4 * d + (s > 1 ? 2 * s * de : 0) + ng * de + 32 +
           row_red_doubles(nw) + nt + 2;
  }

  template <int D, int S>
  struct RowShape {
    static constexpr int NT = S * D;
    static constexpr int NW = NT / 32;
    static constexpr int CW = (D + S - 1) / S; // columns per segment
    static constexpr int ST = row_trial_width(NW);
    static constexpr int TPW = 32 / ST; // trial groups per warp
    static constexpr int NG = NW * TPW;
    static constexpr int DE = (D + 1) & ~1; // vector stride (16-byte aligned)
    static_assert(NT % 32 == 0, "the group is a whole number of warps");
    static_assert(NG >= kLineSearchTrials + 1 && NG <= 32,
                  "one round of trial groups, judged by one ballot");
  };

  template <int D, int S>
  __host__ __device__ constexpr int
  row_smem_doubles()
  {
    return row_smem_doubles_rt(D, S);
  }

  template <class F>
  concept RowLayoutObjective = !TrialsWithGradient<F>;

  // One run on the group: `sm` holds row_smem_doubles<D, S>() doubles
  // (16-byte aligned); the group is threads [base, base + S*D) of the
  // block, synchronised by named barrier `bar`.
  template <class F, int D, int S, bool Adjoint>
  __device__ __forceinline__ void
  row_run(const F& f, double* sm, int bar, int base, const BfgsParams& prm,
          const double* __restrict__ x0, int64_t run, const RunOut& out,
          Control* ctl)
  {
    using RS = RowShape<D, S>;
    constexpr int NT = RS::NT, CW = RS::CW, ST = RS::ST, TPW = RS::TPW;
    constexpr int DE = RS::DE;
    double* X = sm;
    double* P = X + DE;
    double* G = P + DE; // two slots of DE
    double* SWYG = G + 2 * DE;
    double* PART = SWYG + 4 * D;
    double* TX = PART + (S > 1 ? 2 * S * DE : 0);
    double* TF = TX + RS::NG * DE;
    double* red = TF + 32;
    double* scratch = red + row_red_doubles(RS::NW);
    const RowGroup<NT> grp{base, bar, red, scratch};
    const int t = grp.rank(), lw = t >> 5, lane = t & 31;
    const int r = t % D, c = t / D, j0 = c * CW;
    const bool owner = c == 0;

    double H[CW];
#pragma unroll
    for (int k = 0; k < CW; ++k)
      H[k] = (j0 + k == r) ? 1.0 : 0.0;
    for (int i = t; i < D; i += NT)
      X[i] = x0[i];
    grp.sync();
    double best = coop_value<F, D>(f, grp, X);
    coop_gradient_only<F, D, Adjoint>(f, grp, X, G);
    grp.sync();
    double ddir;
    bool stop;
    {
      double v[2] = {0.0, t == 0 ? (double)load_stop(ctl) : 0.0};
      if (owner) {
        const double gi = G[r];
        v[0] = fma(gi, -gi, 0.0);
        P[r] = -gi;
      }
      grp.template sum<2>(v); // its barriers publish p
      ddir = v[0];
      stop = v[1] != 0.0;
    }
    long long n_eval = 1, n_grad = 1;
    int status = kUnset, iter, executed = -1, cur = 0;
    double fout = best, gout = 0.0;
    bool pend = false; // SWYG's {s, w} hold an update not yet applied to H

    for (iter = 0; iter < prm.max_iter; ++iter) {
      if (stop) {
        status = kStopped;
        break;
      }
      // ---- line search, one round of trial groups
      int stop_now = 0;
      int found;
      double fnew;
      {
        const int sub = lane / ST;
#pragma unroll
        for (int q = 0; q < TPW; ++q) {
          const int k = lw * TPW + q;
          if (k <= kLineSearchTrials) {
            const double ak = pow2neg(k);
            double* tx = TX + k * DE;
            for (int i = lane; i < D; i += 32)
              tx[i] = fma(ak, P[i], X[i]);
          }
        }
        __syncwarp();
        if (t == 0)
          stop_now = load_stop(ctl);
        const int k = lw * TPW + sub;
        const TileGroup<ST> sg(cg::tiled_partition<ST>(cg::this_thread_block()),
                               scratch + lw * 32 + sub * ST);
        double f1 = 0.0;
        if (k <= kLineSearchTrials) // uniform within the trial group
          f1 = coop_value<F, D>(f, sg, TX + k * DE);
        if (sg.rank() == 0)
          TF[k] = f1;
        grp.sync();
        bool pass = false;
        double fk = 0.0;
        if (lane <= kLineSearchTrials) {
          fk = TF[lane];
          const double ak = pow2neg(lane);
          pass = lane == kLineSearchTrials ||
                 (fk <= best + kArmijoC1 * ak * ddir && fk < best);
        }
        found = __ffs(__ballot_sync(0xffffffffu, pass)) - 1;
        fnew = __shfl_sync(0xffffffffu, fk, found);
        n_eval += found + 1;
      }
      const double* xa = TX + found * DE; // the accepted point
      double* gn = G + (cur ^ 1) * DE;
      const double* g = G + cur * DE;
      coop_gradient_only<F, D, Adjoint>(f, grp, xa, gn);
      ++n_grad;
      grp.sync();
      const bool take = fnew < best;
      double s_r = 0.0, y_r = 0.0, gx_r = 0.0;
      if (owner) {
        const double go = g[r], gnr = gn[r];
        s_r = xa[r] - X[r];
        y_r = gnr - go;
        gx_r = take ? gnr : go;
        *reinterpret_cast<double2*>(SWYG + 4 * r + 2) = make_double2(y_r, gx_r);
      }
      grp.sync();

      // ---- the pass over H: deferred update, partial sums of H y and H g_x
      double au[2] = {0.0, 0.0}, ah[2] = {0.0, 0.0};
      {
        const double2 swr = *reinterpret_cast<const double2*>(SWYG + 4 * r);
        const double sr = swr.x, wr = swr.y;
        if (pend) {
#pragma unroll
          for (int k = 0; k < CW; ++k) {
            const int j = j0 + k;
            if (D % S == 0 || j < D) {
              const double2 sw = *reinterpret_cast<const double2*>(SWYG + 4 * j);
              const double2 yg = *reinterpret_cast<const double2*>(SWYG + 4 * j + 2);
              H[k] = fma(sr, sw.y, fma(wr, sw.x, H[k]));
              au[k & 1] = fma(H[k], yg.x, au[k & 1]);
              ah[k & 1] = fma(H[k], yg.y, ah[k & 1]);
            }
          }
        } else {
#pragma unroll
          for (int k = 0; k < CW; ++k) {
            const int j = j0 + k;
            if (D % S == 0 || j < D) {
              const double2 yg = *reinterpret_cast<const double2*>(SWYG + 4 * j + 2);
              au[k & 1] = fma(H[k], yg.x, au[k & 1]);
              ah[k & 1] = fma(H[k], yg.y, ah[k & 1]);
            }
          }
        }
      }
      double uu = au[0] + au[1], hh = ah[0] + ah[1];
      if constexpr (S > 1) {
        PART[c * DE + r] = uu;
        PART[(S + c) * DE + r] = hh;
        grp.sync();
        if (owner) {
          uu = PART[r];
          hh = PART[S * DE + r];
#pragma unroll
          for (int cc = 1; cc < S; ++cc) {
            uu += PART[cc * DE + r];
            hh += PART[(S + cc) * DE + r];
          }
        }
      }
      double v[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      if (owner) {
        v[0] = s_r * y_r;
        v[1] = y_r * uu;
        v[2] = uu * gx_r;
        v[3] = s_r * gx_r;
        v[4] = gx_r * hh;
        v[5] = gx_r * gx_r;
      }
      v[6] = (double)stop_now;
      grp.template sum<7>(v); // every thread has finished reading SWYG's s, w
      const bool skipped = fabs(v[0]) < kMinCurvature;
      const double sg = v[3], gh = v[4];
      double rho = 0.0, hb = 0.0, wg = 0.0;
      if (!skipped) {
        rho = 1.0 / v[0];
        hb = 0.5 * rho * fma(rho, v[1], 1.0);
        wg = hb * sg - rho * v[2];
      }
      if (owner) {
        if (!skipped) {
          const double wi = fma(hb, s_r, -rho * uu);
          P[r] = -(hh + s_r * wg + wi * sg);
          *reinterpret_cast<double2*>(SWYG + 4 * r) = make_double2(s_r, wi);
        } else {
          P[r] = -hh;
        }
        if (take)
          X[r] = xa[r];
      }
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
      grp.sync(); // x, p and the accepted point read before new trial points
    }
    if (status == kUnset || status == kStopped) {
      if (status == kUnset)
        status = kSurrender;
      fout = best;
      double gg[1] = {0.0};
      if (owner) {
        const double gi = G[cur * DE + r];
        gg[0] = gi * gi;
      }
      grp.template sum<1>(gg);
      gout = sqrt(gg[0]);
    }
    if (owner && out.x)
      out.x[run * D + r] = X[r];
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
    grp.sync(); // the group's shared memory is free for its next run
  }

  // Segments per row for D in a block of `block` threads: the fewest that
  // keep H's share per thread at most kRowMaxRegDoubles (so a thread's
  // registers hold it beside the working set) and give whole warps
  // dividing the block; 0 where none does.
  inline constexpr int kRowMaxRegDoubles = 48;

  __host__ __device__ constexpr int
  row_segments(int d, int block)
  {
    for (int s = 1; s <= 8; ++s) {
      const int nt = s * d, cw = (d + s - 1) / s;
      if (nt % 32 == 0 && nt <= block && block % nt == 0 && cw <= kRowMaxRegDoubles &&
          nt / 32 * (32 / 2) >= 21)
        return s;
    }
    return 0;
  }

  // Standalone launches: one group per block, blocks take runs from the
  // workspace queue as they finish (block b starts with run b).
  template <class F, int D, int S, bool Adjoint>
  __global__ void __launch_bounds__(S * D)
    bfgs_rows_kernel(F f, BfgsParams prm, const double* __restrict__ starts,
                     RunOut out, Control* ctl, unsigned long long* queue)
  {
    extern __shared__ __align__(16) double sm[];
    constexpr int NT = S * D;
    double* slot = sm + row_smem_doubles<D, S>() - 2;
    int64_t run = blockIdx.x;
    while (run < prm.n) {
      row_run<F, D, S, Adjoint>(f, sm, 1, 0, prm, starts + run * D, run, out, ctl);
      if (threadIdx.x == 0)
        reinterpret_cast<long long*>(slot)[0] =
          (long long)gridDim.x + (long long)atomicAdd(queue, 1ull);
      asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
      run = reinterpret_cast<const long long*>(slot)[0];
      asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
    }
  }

} // namespace zb
