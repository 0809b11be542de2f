// Fast BFGS with the inverse Hessian in registers, one optimisation per group
// of NW warps (the "row" layout, for D a multiple of 32 where H fits the
// register file: D = 32 on 2 warps, 64 on 4, 128 on 12 or 16).
//
// Warp w of the group owns column segment w of H, [w * CW, w * CW + CW)
// with CW = ceil(D / NW), and lane l the R = D / 32 rows l*R .. l*R + R - 1:
// R x CW doubles of H per thread, in registers, so H costs no
// shared-memory traffic at all.  All lanes of a warp walk the same column,
// so each column's four vector entries (s, w, y, g_x) are one broadcast
// load serving R rows.  Several groups share a block (named barriers
// 1..15), so that a block runs several independent optimisations at once
// and one run's barriers and reductions overlap the others' arithmetic.
//
// An iteration (the reference's semantics, bfgs_sequential.cuh:99-219):
//   1. line search: the group's warps split into trial groups of ST lanes,
//      enough for all 21 trials (alpha = 2^-k, k = 0..20) in one round; each
//      evaluates f at its trial point, written from registers at a padded
//      stride (the groups of a warp read different banks); one barrier
//      publishes the values and a ballot in every warp picks the first
//      passing trial (c1 = 0.1, strict decrease; trial 20 is taken when none
//      passes);
//   2. the gradient at the accepted point (its trial point, already in
//      shared memory, is the same bits as fma(alpha, p, x));
//   3. one pass over the registers: the previous iteration's deferred
//      rank-2 update H_rj += s_r w_j + w_r s_j (two FMAs; each thread reads
//      its rows as rows, so exact symmetry is not needed) and the partial
//      row sums of u = H y and h = H g_x; the NW segment partials of a row
//      meet in shared memory;
//   4. one group reduction of {s.y, y.u, u.g, s.g, g.h, g.g, stop}, from
//      which p+ = -(h + s (w.g) + w (s.g)) and g.p+ follow without a
//      second pass over H (w = hb s - rho u, rho = 1/s.y, hb = rho (1 +
//      rho y.u) / 2); the update is skipped when |s.y| < 1e-14.
// Thread t < D (the first R warps) keeps the scalars of one coordinate
// (x, p, s, w, y, g_x); only those warps take part in the group sums.
// Accept-if-better, the fixed-point exit and the termination protocol are
// those of the thread, tile and CTA layouts.
//
// That is row_run_points.  For objectives with line forms (value terms and
// gradient entries read from {x_i, p_i}, e.g. Rosenbrock) and D <= 64,
// row_run_line stores no trial points: trial groups evaluate f(x + a p)
// from {x, p}, every warp computes the gradient entries it needs itself,
// and the row partials and dot products share one reduction -- three group
// barriers an iteration instead of five.
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

  // Trial points are stored at a stride whose offset modulo 16 doubles (one
  // pass over the 32 banks) equals the trial group's width: the ST-lane
  // groups of a warp then read disjoint banks.
  __host__ __device__ constexpr int
  row_trial_stride(int d, int st)
  {
    const int want = st % 16, have = d % 16;
    return d + ((want - have + 16) % 16);
  }

  // Shared memory of one group (doubles): x | p | g[2] | {s, w, y, g_x}[D]
  // | row partial sums 2 x NW x D | trial points 21 at the padded stride |
  // trial values 32 | reductions | scratch NT | the last KS columns of every
  // thread's H segment, KS x R x NT | run slot 2.  Every part is an even
  // number of doubles, so the parts stay 16-byte aligned.
  __host__ __device__ constexpr int
  row_smem_doubles_rt(int d, int nw, int ks = 0)
  {
    const int nt = 32 * nw, de = (d + 1) & ~1, st = row_trial_width(nw);
    const int ntx = kLineSearchTrials + 1; // trial points stored: the 21 trials
    return 4 * de + 4 * d + 2 * nw * de + ntx * ((row_trial_stride(d, st) + 1) & ~1) + 32 +
           row_red_doubles(nw) + nt + ks * (d / 32) * nt + 2;
  }

  template <int D, int NWG>
  struct RowShape {
    static constexpr int NW = NWG;
    static constexpr int NT = 32 * NW;
    static constexpr int R = D / 32;              // rows per lane
    static constexpr int CW = (D + NW - 1) / NW;  // columns per warp
    static constexpr int ST = row_trial_width(NW);
    static constexpr int TPW = 32 / ST; // trial groups per warp
    static constexpr int NG = NW * TPW;
    static constexpr int DE = (D + 1) & ~1; // vector stride (16-byte aligned)
    static constexpr int TSTR = (row_trial_stride(D, ST) + 1) & ~1;
    static_assert(D % 32 == 0, "the rows split evenly over the lanes");
    static_assert(NG >= kLineSearchTrials + 1 && NG <= 32,
                  "one round of trial groups, judged by one ballot");
  };

  template <int D, int NW, int KS = 0>
  __host__ __device__ constexpr int
  row_smem_doubles()
  {
    return row_smem_doubles_rt(D, NW, KS);
  }

  template <class F>
  concept RowLayoutObjective = !TrialsWithGradient<F>;

  // A RowGroup whose members are renumbered so that the member computing
  // coordinate r of a cooperative gradient (rank r) is the thread that owns
  // r: that thread then reads its entry back without a barrier.
  template <int NT, int R>
  struct OwnerGroup {
    const RowGroup<NT>& g;
    __device__ __forceinline__ int
    rank() const
    {
      const int t = g.rank();
      return t < 32 * R ? (t % 32) * R + t / 32 : t;
    }
    static constexpr int
    size()
    {
      return NT;
    }
    __device__ __forceinline__ void
    sync() const
    {
      g.sync();
    }
    template <int K>
    __device__ __forceinline__ void
    sum(double (&v)[K]) const
    {
      g.template sum<K>(v);
    }
    __device__ __forceinline__ double
    sum(double v) const
    {
      return g.sum(v);
    }
    __device__ __forceinline__ double
    bcast(double v, int src) const
    {
      return g.bcast(v, src);
    }
  };

  // Objectives whose cooperative gradient has member r write entry r
  // (coop_for over the group, or the dual passes): the owner's entry needs
  // no barrier.
  template <class F, class G, bool Adjoint>
  concept OwnerWritesGradient =
    !Adjoint || HasGradientCoop<F, G> || HasAdjointCoop<F, G>;

  // One run on the group, trial points stored: `sm` holds
  // row_smem_doubles<D, NW, KS>() doubles (16-byte aligned); the group is
  // threads [base, base + 32 NW) of the block, synchronised by named
  // barrier `bar`.  With KS > 0 the last KS columns of each thread's H
  // segment live in shared memory (thread-major: a warp's accesses are
  // consecutive), the rest in registers, so that a group of half the warps
  // holds the same H and two groups share a block.
  template <class F, int D, int NW, bool Adjoint, bool kTimed = false, int KS = 0>
  __device__ __forceinline__ void
  row_run_points(const F& f, double* sm, int bar, int base, const BfgsParams& prm,
                 const double* __restrict__ x0, int64_t run, const RunOut& out,
                 Control* ctl)
  {
    using RS = RowShape<D, NW>;
    constexpr int NT = RS::NT, R = RS::R, CW = RS::CW, ST = RS::ST, TPW = RS::TPW;
    constexpr int DE = RS::DE, TSTR = RS::TSTR;
    constexpr int KR = CW - KS; // columns in registers
    static_assert(KS >= 0 && KR >= 1 && (KS == 0 || R % 2 == 0),
                  "shared columns hold row pairs");
    double* X = sm;
    double* P = X + DE;
    double* G = P + DE; // two slots of DE
    // per-coordinate vectors of the H pass, {s, w} and {y, g_x} pairs, and
    // the row partial sums [u | h][warp][.], all in owner order: coordinate
    // r sits at oi(r) = (r % R) * 32 + r / R, so the owner of r (thread
    // oi(r)) and each lane reading its R rows touch consecutive slots
    double* SW = G + 2 * DE;
    double* YG = SW + 2 * D;
    double* PART = SW + 4 * D;
    double* TX = PART + 2 * NW * DE;
    double* TF = TX + (kLineSearchTrials + 1) * TSTR;
    double* red = TF + 32;
    double* scratch = red + row_red_doubles(NW);
    const RowGroup<NT> grp{base, bar, red, scratch};
    const int t = grp.rank(), lw = t >> 5, lane = t & 31;
    const int j0 = lw * CW, r0 = lane * R; // my columns and rows
    const bool owner = t < D;              // thread oi(r) keeps coordinate r
    const int r = owner ? (t % 32) * R + t / 32 : 0;
    // rows q, q + 1 of shared column KR + c: HS[(c * R / 2 + q / 2) * NT + t]
    double2* HS = reinterpret_cast<double2*>(scratch + NT);

    double H[R][KR];
#pragma unroll
    for (int q = 0; q < R; ++q)
#pragma unroll
      for (int k = 0; k < KR; ++k)
        H[q][k] = (j0 + k == r0 + q) ? 1.0 : 0.0;
#pragma unroll
    for (int c = 0; c < KS; ++c)
#pragma unroll
      for (int q = 0; q < R; q += 2)
        HS[(c * R / 2 + q / 2) * NT + t] =
          make_double2(j0 + KR + c == r0 + q ? 1.0 : 0.0,
                       j0 + KR + c == r0 + q + 1 ? 1.0 : 0.0);
    for (int i = t; i < D; i += NT)
      X[i] = x0[i];
    grp.sync();
    const CycleTimer<kTimed> tm(out, run, t == 0);
    double best = coop_value<F, D>(f, grp, X);
    tm.start_grad();
    coop_gradient_only<F, D, Adjoint>(f, grp, X, G);
    grp.sync();
    tm.stop_grad();
    double ddir;
    bool stop;
    {
      double v[2] = {0.0, t == 0 ? (double)load_stop(ctl) : 0.0};
      if (owner) {
        const double gi = G[r];
        v[0] = fma(gi, -gi, 0.0);
        P[r] = -gi;
      }
      grp.template sum<2, R>(v); // its barrier publishes p
      ddir = v[0];
      stop = v[1] != 0.0;
    }
    long long n_eval = 1, n_grad = 1;
    int status = kUnset, iter, executed = -1, cur = 0;
    const double tol_sq4 = 4.0 * prm.tol * prm.tol;
    double fout = best, gout = 0.0;
    bool pend = false; // SW holds an update not yet applied to H
    // the stop flag read in the previous iteration (a run sees the flag one
    // iteration after it reads it, so the read's latency is off the path)
    int stop_seen = 0;

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
        // this lane's coordinates of x and p, read once: the trial points
        // are written from registers
        constexpr int RV = (D + 31) / 32;
        double xr[RV], pr[RV];
#pragma unroll
        for (int q = 0; q < RV; ++q) {
          const int i = lane + 32 * q;
          xr[q] = i < D ? X[i] : 0.0;
          pr[q] = i < D ? P[i] : 0.0;
        }
        if (t == 0)
          stop_now = load_stop(ctl);
        const int sub = lane / ST;
#pragma unroll
        for (int q = 0; q < TPW; ++q) {
          const int k = lw * TPW + q;
          if (k <= kLineSearchTrials) {
            const double ak = pow2neg(k);
            double* tx = TX + k * TSTR;
#pragma unroll
            for (int v = 0; v < RV; ++v) {
              const int i = lane + 32 * v;
              if (i < D)
                tx[i] = fma(ak, pr[v], xr[v]);
            }
          }
        }
        __syncwarp();
        const int k = lw * TPW + sub;
        const TileGroup<ST> sg(cg::tiled_partition<ST>(cg::this_thread_block()),
                               scratch + lw * 32 + sub * ST);
        double f1 = 0.0;
        if (k <= kLineSearchTrials) // uniform within the trial group
          f1 = coop_value<F, D>(f, sg, TX + k * TSTR);
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
      const double* xa = TX + found * TSTR; // the accepted point
      double* gn = G + (cur ^ 1) * DE;
      const double* g = G + cur * DE;
      tm.start_grad();
      {
        const OwnerGroup<NT, R> og{grp};
        coop_gradient_only<F, D, Adjoint>(f, og, xa, gn);
        if constexpr (!OwnerWritesGradient<F, OwnerGroup<NT, R>, Adjoint>)
          grp.sync();
      }
      tm.stop_grad();
      ++n_grad;
      const bool take = fnew < best;
      double s_r = 0.0, y_r = 0.0, gx_r = 0.0;
      if (owner) {
        const double go = g[r], gnr = gn[r];
        s_r = xa[r] - X[r];
        y_r = gnr - go;
        gx_r = take ? gnr : go;
        *reinterpret_cast<double2*>(YG + 2 * t) = make_double2(y_r, gx_r);
      }
      grp.sync();

      // ---- the pass over H: deferred update, partial sums of H y and H g_x
      // over this warp's columns for this lane's rows
      tm.start_update();
      double au[R], ah[R];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        au[q] = 0.0;
        ah[q] = 0.0;
      }
      if (pend) {
        double sr[R], wr[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const double2 sw = *reinterpret_cast<const double2*>(SW + 2 * (q * 32 + lane));
          sr[q] = sw.x;
          wr[q] = sw.y;
        }
#pragma unroll
        for (int k = 0; k < CW; ++k) {
          const int j = j0 + k;
          if (D % NW == 0 || j < D) {
            const int oj = (j % R) * 32 + j / R;
            const double2 sw = *reinterpret_cast<const double2*>(SW + 2 * oj);
            const double2 yg = *reinterpret_cast<const double2*>(YG + 2 * oj);
            if (k < KR) {
#pragma unroll
              for (int q = 0; q < R; ++q) {
                H[q][k < KR ? k : 0] =
                  fma(sr[q], sw.y, fma(wr[q], sw.x, H[q][k < KR ? k : 0]));
                au[q] = fma(H[q][k < KR ? k : 0], yg.x, au[q]);
                ah[q] = fma(H[q][k < KR ? k : 0], yg.y, ah[q]);
              }
            } else {
#pragma unroll
              for (int q = 0; q < R; q += 2) {
                double2* hp = HS + ((k - KR) * R / 2 + q / 2) * NT + t;
                double2 h = *hp;
                h.x = fma(sr[q], sw.y, fma(wr[q], sw.x, h.x));
                h.y = fma(sr[q + 1], sw.y, fma(wr[q + 1], sw.x, h.y));
                *hp = h;
                au[q] = fma(h.x, yg.x, au[q]);
                ah[q] = fma(h.x, yg.y, ah[q]);
                au[q + 1] = fma(h.y, yg.x, au[q + 1]);
                ah[q + 1] = fma(h.y, yg.y, ah[q + 1]);
              }
            }
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < CW; ++k) {
          const int j = j0 + k;
          if (D % NW == 0 || j < D) {
            const int oj = (j % R) * 32 + j / R;
            const double2 yg = *reinterpret_cast<const double2*>(YG + 2 * oj);
            if (k < KR) {
#pragma unroll
              for (int q = 0; q < R; ++q) {
                au[q] = fma(H[q][k < KR ? k : 0], yg.x, au[q]);
                ah[q] = fma(H[q][k < KR ? k : 0], yg.y, ah[q]);
              }
            } else {
#pragma unroll
              for (int q = 0; q < R; q += 2) {
                const double2 h = HS[((k - KR) * R / 2 + q / 2) * NT + t];
                au[q] = fma(h.x, yg.x, au[q]);
                ah[q] = fma(h.x, yg.y, ah[q]);
                au[q + 1] = fma(h.y, yg.x, au[q + 1]);
                ah[q + 1] = fma(h.y, yg.y, ah[q + 1]);
              }
            }
          }
        }
      }
#pragma unroll
      for (int q = 0; q < R; ++q) {
        PART[lw * D + q * 32 + lane] = au[q];
        PART[(NW + lw) * D + q * 32 + lane] = ah[q];
      }
      grp.sync();
      double uu = 0.0, hh = 0.0;
      if (owner) {
        double u2[2] = {PART[t], NW > 1 ? PART[D + t] : 0.0};
        double h2[2] = {PART[NW * D + t], NW > 1 ? PART[(NW + 1) * D + t] : 0.0};
#pragma unroll
        for (int w = 2; w < NW; ++w) {
          u2[w & 1] += PART[w * D + t];
          h2[w & 1] += PART[(NW + w) * D + t];
        }
        uu = u2[0] + u2[1];
        hh = h2[0] + h2[1];
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
      v[6] = (double)stop_seen;
      stop_seen = stop_now;
      grp.template sum<7, R>(v); // every thread has finished reading SW
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
          *reinterpret_cast<double2*>(SW + 2 * t) = make_double2(s_r, wi);
        } else {
          P[r] = -hh;
        }
        if (take)
          X[r] = xa[r];
      }
      tm.stop_update();
      pend = !skipped;
      ddir = skipped ? -gh : -(gh + 2.0 * sg * wg);
      stop = v[6] != 0.0;
      if (take) {
        best = fnew;
        cur ^= 1;
      }
      // ||g|| = sqrt(g.g): taken only where it decides something (far
      // above tol^2, g.g cannot pass the test)
      if (!isfinite(v[5]) || !isfinite(fnew)) {
        status = kNonFinite;
        fout = fnew;
        gout = sqrt(v[5]);
        break;
      }
      if (v[5] <= tol_sq4 && sqrt(v[5]) < prm.tol) {
        if (t == 0)
          note_converged(ctl, prm.required);
        status = kConverged;
        fout = best;
        gout = sqrt(v[5]);
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
      grp.template sum<1, R>(gg);
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
      tm.finish();
    }
    grp.sync(); // the group's shared memory is free for its next run
  }

  // Objectives whose value along the search line and whose gradient entries
  // are read from {x_i, p_i} pairs in owner order (slot (i % R) * 32 + i /
  // R; coordinate i of x + a p is fma(a, p_i, x_i), the bits of a stored
  // trial point): member m of an S-lane trial group returns its partial sum
  // of the value's terms, and gradient entry i needs only a few
  // coordinates, so any thread computes the entries it uses itself.
  template <class F>
  concept RowLineObjective = requires(const F& f, const double2* xp, double a, int i) {
    { f.template value_line_part<8, 1>(xp, a, i) } -> std::convertible_to<double>;
    { f.template gradient_line_entry<1>(xp, a, i) } -> std::convertible_to<double>;
  };

  // Shared memory of row_run_line (doubles): {x, p}[D] | {s, w}[D] | per
  // warp {y, g_x}[D] | row partial sums 2 x NW x D | trial values 32 |
  // reductions | scratch NT; all vectors in owner order; within
  // row_smem_doubles.
  __host__ __device__ constexpr int
  row_line_smem_doubles(int d, int nw)
  {
    const int de = (d + 1) & ~1;
    return 2 * de + 2 * d + 2 * nw * d + 2 * nw * de + 32 + row_red_doubles(nw) + 32 * nw;
  }

  // One run on the group for a RowLineObjective with analytic gradients.
  // Three barriers an iteration instead of five, and no trial points or
  // gradients in shared memory:
  //   1. line search: trial group k evaluates f(x + 2^-k p) from {x, p};
  //      one barrier publishes the 21 values, a ballot picks the trial;
  //   2. every lane computes the gradient entries at the accepted point of
  //      its R rows, so each warp fills its own {y, g_x} table of all D
  //      coordinates (no group barrier); gradients at x stay in registers
  //      from one iteration to the next;
  //   3. the pass over H (the previous iteration's deferred update, then
  //      each warp's row partials of H y and H g_x, as in row_run_points);
  //      the partials go to shared memory and the warp's share of y.Hy, g.Hy and
  //      g.Hg (its rows' y and g_x times its column-segment partials) joins
  //      s.y, s.g and g.g (warp 0) in ONE group reduction, whose barrier
  //      also publishes the partials;
  //   4. the owner of coordinate r adds up its row's NW partials, forms
  //      p+_r and w_r and writes {x, p}[r] and {s, w}[r]; the end-of-
  //      iteration barrier publishes them.
  // The arithmetic of a run is that of row_run_points up to the order of
  // the reductions' additions.
  template <class F, int D, int NW, bool kTimed = false>
  __device__ __forceinline__ void
  row_run_line(const F& f, double* sm, int bar, int base, const BfgsParams& prm,
               const double* __restrict__ x0, int64_t run, const RunOut& out,
               Control* ctl)
  {
    using RS = RowShape<D, NW>;
    constexpr int NT = RS::NT, R = RS::R, CW = RS::CW, ST = RS::ST, TPW = RS::TPW;
    constexpr int DE = RS::DE;
    static_assert(row_line_smem_doubles(D, NW) <= row_smem_doubles<D, NW>() - 2,
                  "fits the row layout's shared memory, run slot excluded");
    double2* XP = reinterpret_cast<double2*>(sm); // {x, p}, owner order
    double* SW = sm + 2 * DE;                      // {s, w}, owner order
    double* YGW = SW + 2 * D; // warp w's {y, g_x} at YGW + 2 D w, owner order
    double* PART = YGW + 2 * D * NW;
    double* TF = PART + 2 * NW * DE;
    double* red = TF + 32;
    double* scratch = red + row_red_doubles(NW);
    const RowGroup<NT> grp{base, bar, red, scratch};
    const int t = grp.rank(), lw = t >> 5, lane = t & 31;
    const int j0 = lw * CW, r0 = lane * R;
    // warps 0..R-1: thread t keeps coordinate r, whose slot is t
    const bool owner = t < D;
    const int r = owner ? lane * R + lw : 0;

    double H[R][CW];
#pragma unroll
    for (int q = 0; q < R; ++q)
#pragma unroll
      for (int k = 0; k < CW; ++k)
        H[q][k] = (j0 + k == r0 + q) ? 1.0 : 0.0;
    // f and the gradient at the start, from a plain copy of x0
    double* X0 = PART;
    double* G0 = PART + DE;
    for (int i = t; i < D; i += NT)
      X0[i] = x0[i];
    grp.sync();
    const CycleTimer<kTimed> tm(out, run, t == 0);
    double best = coop_value<F, D>(f, grp, X0);
    tm.start_grad();
    coop_gradient_only<F, D, true>(f, grp, X0, G0);
    grp.sync();
    tm.stop_grad();
    double gq[R]; // the gradient at x, this lane's rows
#pragma unroll
    for (int q = 0; q < R; ++q)
      gq[q] = G0[r0 + q];
    double ddir;
    bool stop;
    {
      double v[2] = {0.0, t == 0 ? (double)load_stop(ctl) : 0.0};
      if (owner) {
        const double gi = G0[r];
        v[0] = fma(gi, -gi, 0.0);
        XP[t] = make_double2(X0[r], -gi);
      }
      grp.template sum<2, R>(v); // its barrier publishes {x, p}
      ddir = v[0];
      stop = v[1] != 0.0;
    }
    long long n_eval = 1, n_grad = 1;
    int status = kUnset, iter, executed = -1;
    const double tol_sq4 = 4.0 * prm.tol * prm.tol;
    double fout = best, gout = 0.0;
    bool pend = false; // SW holds an update not yet applied to H
    // the stop flag read in the previous iteration (a run sees the flag one
    // iteration after it reads it, so the read's latency is off the path)
    int stop_seen = 0;

    for (iter = 0; iter < prm.max_iter; ++iter) {
      if (stop) {
        status = kStopped;
        break;
      }
      int stop_now = 0;
      if (t == 0)
        stop_now = load_stop(ctl);
      // ---- line search: trial k = TPW lw + (lane / ST) on ST lanes; the
      // groups past trial 20 evaluate trial 20 again (no divergence) and
      // their values are dropped
      int found;
      double fnew;
      {
        const int sub = lane / ST, k = lw * TPW + sub;
        const int kk = k < kLineSearchTrials ? k : kLineSearchTrials;
        double part = f.template value_line_part<ST, R>(XP, pow2neg(kk), lane % ST);
#pragma unroll
        for (int o = ST / 2; o >= 1; o >>= 1)
          part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane % ST == 0 && k <= kLineSearchTrials)
          TF[k] = part;
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
      const double alpha = pow2neg(found);
      const bool take = fnew < best;
      ++n_grad;
      // ---- gradient entries at the accepted point for this lane's rows,
      // into the warp's {y, g_x} table
      tm.start_grad();
      double sq[R], yq[R], gxq[R];
      double2 xpo = make_double2(0.0, 0.0); // the owner's {x, p}
      double* yg_w = YGW + 2 * D * lw;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const double2 c = XP[q * 32 + lane];
        const double gn = f.template gradient_line_entry<R>(XP, alpha, r0 + q);
        sq[q] = fma(alpha, c.y, c.x) - c.x;
        yq[q] = gn - gq[q];
        gxq[q] = take ? gn : gq[q];
        *reinterpret_cast<double2*>(yg_w + 2 * (q * 32 + lane)) = make_double2(yq[q], gxq[q]);
        if (q == lw)
          xpo = c;
      }
      __syncwarp();
      tm.stop_grad();
      tm.start_update();

      // ---- the pass over H: deferred update, partial sums of H y and H g_x
      double au[R], ah[R];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        au[q] = 0.0;
        ah[q] = 0.0;
      }
      if (pend) {
        double sr[R], wr[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const double2 sw = *reinterpret_cast<const double2*>(SW + 2 * (q * 32 + lane));
          sr[q] = sw.x;
          wr[q] = sw.y;
        }
#pragma unroll
        for (int k = 0; k < CW; ++k) {
          const int j = j0 + k;
          if (D % NW == 0 || j < D) {
            const int oj = (j % R) * 32 + j / R;
            const double2 sw = *reinterpret_cast<const double2*>(SW + 2 * oj);
            const double2 yg = *reinterpret_cast<const double2*>(yg_w + 2 * oj);
#pragma unroll
            for (int q = 0; q < R; ++q) {
              H[q][k] = fma(sr[q], sw.y, fma(wr[q], sw.x, H[q][k]));
              au[q] = fma(H[q][k], yg.x, au[q]);
              ah[q] = fma(H[q][k], yg.y, ah[q]);
            }
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < CW; ++k) {
          const int j = j0 + k;
          if (D % NW == 0 || j < D) {
            const int oj = (j % R) * 32 + j / R;
            const double2 yg = *reinterpret_cast<const double2*>(yg_w + 2 * oj);
#pragma unroll
            for (int q = 0; q < R; ++q) {
              au[q] = fma(H[q][k], yg.x, au[q]);
              ah[q] = fma(H[q][k], yg.y, ah[q]);
            }
          }
        }
      }
      double v[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int q = 0; q < R; ++q) {
        PART[lw * DE + q * 32 + lane] = au[q];
        PART[(NW + lw) * DE + q * 32 + lane] = ah[q];
        v[1] = fma(yq[q], au[q], v[1]);
        v[2] = fma(gxq[q], au[q], v[2]);
        v[4] = fma(gxq[q], ah[q], v[4]);
        if (lw == 0) {
          v[0] = fma(sq[q], yq[q], v[0]);
          v[3] = fma(sq[q], gxq[q], v[3]);
          v[5] = fma(gxq[q], gxq[q], v[5]);
        }
      }
      v[6] = (double)stop_seen;
      stop_seen = stop_now;
      grp.template sum<7>(v); // its barrier also publishes the partials
      const bool skipped = fabs(v[0]) < kMinCurvature;
      const double sg = v[3], gh = v[4];
      double rho = 0.0, hb = 0.0, wg = 0.0;
      if (!skipped) {
        rho = 1.0 / v[0];
        hb = 0.5 * rho * fma(rho, v[1], 1.0);
        wg = hb * sg - rho * v[2];
      }
      if (owner) {
        double u2[2] = {PART[t], NW > 1 ? PART[DE + t] : 0.0};
        double h2[2] = {PART[NW * DE + t], NW > 1 ? PART[(NW + 1) * DE + t] : 0.0};
#pragma unroll
        for (int w = 2; w < NW; ++w) {
          u2[w & 1] += PART[w * DE + t];
          h2[w & 1] += PART[(NW + w) * DE + t];
        }
        const double uu = u2[0] + u2[1], hh = h2[0] + h2[1];
        double s_r = sq[0];
#pragma unroll
        for (int q = 1; q < R; ++q)
          if (q == lw)
            s_r = sq[q];
        double pn;
        if (!skipped) {
          const double wi = fma(hb, s_r, -rho * uu);
          pn = -(hh + s_r * wg + wi * sg);
          *reinterpret_cast<double2*>(SW + 2 * t) = make_double2(s_r, wi);
        } else {
          pn = -hh;
        }
        XP[t] = make_double2(take ? fma(alpha, xpo.y, xpo.x) : xpo.x, pn);
      }
      tm.stop_update();
#pragma unroll
      for (int q = 0; q < R; ++q)
        gq[q] = gxq[q];
      pend = !skipped;
      ddir = skipped ? -gh : -(gh + 2.0 * sg * wg);
      stop = v[6] != 0.0;
      if (take)
        best = fnew;
      // ||g|| = sqrt(g.g): taken only where it decides something (far
      // above tol^2, g.g cannot pass the test)
      if (!isfinite(v[5]) || !isfinite(fnew)) {
        status = kNonFinite;
        fout = fnew;
        gout = sqrt(v[5]);
        break;
      }
      if (v[5] <= tol_sq4 && sqrt(v[5]) < prm.tol) {
        if (t == 0)
          note_converged(ctl, prm.required);
        status = kConverged;
        fout = best;
        gout = sqrt(v[5]);
        break;
      }
      if (!take && skipped && !(prm.flags & kFlagNoFixedPoint)) {
        executed = iter + 1;
        iter = prm.max_iter;
        break;
      }
      grp.sync(); // {x, p} and {s, w} written before the next line search
    }
    if (status == kUnset || status == kStopped) {
      if (status == kUnset)
        status = kSurrender;
      fout = best;
      double gg[1] = {0.0};
      if (lw == 0) {
#pragma unroll
        for (int q = 0; q < R; ++q)
          gg[0] = fma(gq[q], gq[q], gg[0]);
      }
      grp.template sum<1, 1>(gg);
      gout = sqrt(gg[0]);
    }
    if (owner && out.x)
      out.x[run * D + r] = XP[t].x;
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
    grp.sync(); // the group's shared memory is free for its next run
  }

  // One run on the group: the line form where the objective has one,
  // gradients are analytic and a lane holds at most two rows, else trial
  // points in shared memory.  (At D = 128, four rows a lane on twelve
  // warps, the line form measured slower on a B200: twelve warps each
  // computing all 128 gradient entries and a twelve-warp reduction cost
  // more than the two barriers saved.)
  inline constexpr int kRowLineMaxDim = 64;

  template <class F, int D, int NW, bool Adjoint, bool kTimed = false, int KS = 0>
  __device__ __forceinline__ void
  row_run(const F& f, double* sm, int bar, int base, const BfgsParams& prm,
          const double* __restrict__ x0, int64_t run, const RunOut& out,
          Control* ctl)
  {
    if constexpr (KS == 0 && Adjoint && RowLineObjective<F> && D <= kRowLineMaxDim)
      row_run_line<F, D, NW, kTimed>(f, sm, bar, base, prm, x0, run, out, ctl);
    else
      row_run_points<F, D, NW, Adjoint, kTimed, KS>(f, sm, bar, base, prm, x0, run,
                                                    out, ctl);
  }

  // Warps of a group for D in a block of `block` threads: among the counts
  // that divide the block, keep H's share per thread at most
  // kRowMaxRegDoubles (so a thread's registers hold it beside the working
  // set) and give the line search one round of trial groups, the fewest
  // whose column segments split D evenly (no guarded tail), else the
  // fewest; 0 where none fits (D not a multiple of 32, or too large).
  inline constexpr int kRowMaxRegDoubles = 48;

  __host__ __device__ constexpr bool
  row_warps_fit(int d, int block, int nw)
  {
    const int nt = 32 * nw, cw = (d + nw - 1) / nw;
    return nt <= block && block % nt == 0 && (d / 32) * cw <= kRowMaxRegDoubles &&
           nw * (32 / row_trial_width(nw)) >= kLineSearchTrials + 1;
  }

  __host__ __device__ constexpr int
  row_warps(int d, int block)
  {
    if (d % 32 != 0)
      return 0;
    for (int nw = 1; nw <= 32; ++nw)
      if (d % nw == 0 && row_warps_fit(d, block, nw))
        return nw;
    for (int nw = 1; nw <= 32; ++nw)
      if (row_warps_fit(d, block, nw))
        return nw;
    return 0;
  }

  // H doubles a thread of a split group keeps in registers: those of a
  // thread of the unsplit group (44 at D = 128), which the batch kernel's
  // register budget holds without spilling in the sweep.
  inline constexpr int kRowSplitRegDoubles = 44;

  // Split groups (the standalone row kernel): where one group of
  // row_warps(d, block) warps fills the whole block (D = 128 at 384
  // threads: twelve warps), two blocks of half the warps share the SM
  // instead, each thread keeping as many columns of its segment in registers
  // as before and the last `row_split_cols` in shared memory.  Two runs then
  // go through an SM at once, one's barriers and reductions overlapping the
  // other's sweep: the 128-D class of 1365 runs 14.1 -> 11.1 ms on a B200,
  // though one run alone is slower (3.18 against 2.80 us an iteration).
  __host__ __device__ constexpr int
  row_split_warps(int d, int block)
  {
    const int nw = row_warps(d, block);
    return (nw > 0 && 32 * nw == block && block <= 384 && d >= 128 && nw % 2 == 0)
             ? nw / 2
             : 0;
  }
  __host__ __device__ constexpr int
  row_split_cols(int d, int block)
  {
    const int nw2 = row_split_warps(d, block);
    if (!nw2)
      return 0;
    const int r = d / 32, cw = (d + nw2 - 1) / nw2, kr = kRowSplitRegDoubles / r;
    return cw > kr ? cw - kr : 0;
  }
  // Warps of one group and shared columns per thread in a block of `block`
  __host__ __device__ constexpr int
  row_group_warps(int d, int block)
  {
    return row_split_warps(d, block) ? row_split_warps(d, block) : row_warps(d, block);
  }

  // Standalone launches: one group per block (two blocks per SM for split
  // groups, the registers of the two summing to one full block's), blocks
  // take runs from the workspace queue as they finish (block b starts with
  // run b).
  template <class F, int D, int NW, bool Adjoint, bool kTimed = false, int KS = 0>
  __global__ void __launch_bounds__(32 * NW, KS > 0 ? 2 : 1)
    bfgs_rows_kernel(F f, BfgsParams prm, const double* __restrict__ starts,
                     RunOut out, Control* ctl, unsigned long long* queue)
  {
    extern __shared__ __align__(16) double sm[];
    constexpr int NT = 32 * NW;
    double* slot = sm + row_smem_doubles<D, NW, KS>() - 2;
    int64_t run = blockIdx.x;
    while (run < prm.n) {
      row_run<F, D, NW, Adjoint, kTimed, KS>(f, sm, 1, 0, prm, starts + run * D, run, out,
                                             ctl);
      if (threadIdx.x == 0)
        reinterpret_cast<long long*>(slot)[0] =
          (long long)gridDim.x + (long long)atomicAdd(queue, 1ull);
      asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
      run = reinterpret_cast<const long long*>(slot)[0];
      asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
    }
  }

} // namespace zb
