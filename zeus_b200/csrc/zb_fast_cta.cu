// CTA-per-run fast BFGS launcher (D > 32; H in shared memory, or past
// about D = 160 in a global-memory slice per block taken from the caller's
// workspace).
#include "zb_bfgs_coop.cuh"
#include "zb_bfgs_rows.cuh"
#include "zb_objective_visit.cuh"

namespace zb {

  namespace {
    constexpr int kMinCtaDim = 33;
    constexpr size_t kSmemLimit = 227 * 1024;
    constexpr size_t kQueueBytes = 256; // the run queue, ahead of any H slices

    template <int D>
    constexpr int
    cta_block()
    {
      return D <= 64 ? 256 : 512;
    }

    // blocks of a global-H launch (and slices of its workspace)
    int64_t
    global_h_slices(int64_t n)
    {
      const int64_t cap = 2 * (int64_t)sm_count();
      return n < cap ? n : cap;
    }

    template <class F, int D, bool Adj, bool kTimed>
    int
    launch_one(const F& f, const BfgsParams& prm, const double* starts,
               const RunOut& out, Control* ctl, void* ws, size_t ws_bytes,
               cudaStream_t st)
    {
      constexpr int B = cta_block<D>();
      const size_t smem = sizeof(double) * cta_smem_doubles<F, D, Adj>(B);
      auto kern = bfgs_cta_kernel<F, D, Adj, B, kTimed>;
      int rc = cuda_fail(cudaFuncSetAttribute(
                           kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem),
                         "CTA-layout shared memory attribute");
      if (rc)
        return rc;
      int per_sm = 0;
      rc = cuda_fail(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                       &per_sm, kern, B, smem),
                     "CTA-layout occupancy");
      if (rc)
        return rc;
      if (per_sm < 1) {
        set_error("CTA layout: dim %d does not fit on an SM", D);
        return ZEUS_E_UNSUPPORTED;
      }
      int64_t cap = (int64_t)sm_count() * per_sm;
      const size_t need = cta_workspace_bytes(D, prm.n);
      if (!ws || ws_bytes < need) {
        set_error("CTA layout at dim %d: %zu workspace bytes needed, got %zu", D,
                  need, ws_bytes);
        return ZEUS_E_WORKSPACE;
      }
      auto* queue = static_cast<unsigned long long*>(ws);
      double* hws = nullptr;
      if constexpr (cta_h_global(D, B)) {
        hws = reinterpret_cast<double*>(static_cast<char*>(ws) + kQueueBytes);
        const int64_t slices = global_h_slices(prm.n);
        cap = cap < slices ? cap : slices;
      }
      if ((rc = cuda_fail(cudaMemsetAsync(queue, 0, sizeof *queue, st),
                          "CTA-layout run queue reset")))
        return rc;
      const unsigned grid = (unsigned)(prm.n < cap ? prm.n : cap);
      kern<<<grid, B, smem, st>>>(f, prm, starts, out, ctl, hws, queue);
      return cuda_fail(cudaGetLastError(), "CTA-layout BFGS launch");
    }
    // the row layout standalone: one group per block
    constexpr int kRowBlockCap = 384;

    template <class F, int D, bool Adj, bool kTimed>
    int
    launch_rows_one(const F& f, const BfgsParams& prm, const double* starts,
                    const RunOut& out, Control* ctl, void* ws, size_t ws_bytes,
                    cudaStream_t st)
    {
      // the batch's groups: split groups for D = 128, two blocks per SM
      constexpr int NW = row_group_warps(D, kRowBlockCap), NT = 32 * NW;
      constexpr int KS = row_split_cols(D, kRowBlockCap);
      const size_t smem = sizeof(double) * row_smem_doubles<D, NW, KS>();
      auto kern = bfgs_rows_kernel<F, D, NW, Adj, kTimed, KS>;
      int rc = cuda_fail(cudaFuncSetAttribute(
                           kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem),
                         "row-layout shared memory attribute");
      if (rc)
        return rc;
      int per_sm = 0;
      if ((rc = cuda_fail(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern,
                                                                         NT, smem),
                          "row-layout occupancy")))
        return rc;
      if (per_sm < 1) {
        set_error("row layout: dim %d does not fit on an SM", D);
        return ZEUS_E_UNSUPPORTED;
      }
      if (!ws || ws_bytes < kQueueBytes) {
        set_error("row layout at dim %d: %zu workspace bytes needed, got %zu", D,
                  kQueueBytes, ws_bytes);
        return ZEUS_E_WORKSPACE;
      }
      auto* queue = static_cast<unsigned long long*>(ws);
      if ((rc = cuda_fail(cudaMemsetAsync(queue, 0, sizeof *queue, st),
                          "row-layout run queue reset")))
        return rc;
      const int64_t cap = (int64_t)sm_count() * per_sm;
      const unsigned grid = (unsigned)(prm.n < cap ? prm.n : cap);
      kern<<<grid, NT, smem, st>>>(f, prm, starts, out, ctl, queue);
      return cuda_fail(cudaGetLastError(), "row-layout BFGS launch");
    }

    template <class F>
    constexpr bool
    rows_built()
    {
      constexpr int D = (int)F::arity;
      return D >= 32 && RowLayoutObjective<F> && row_warps(D, kRowBlockCap) > 0;
    }
  } // namespace

  bool
  rows_layout_supported(int kind, int dim)
  {
    if (!builtin_supported(kind, dim))
      return false;
    Objective o{kind, dim, nullptr, nullptr, 0, 0, nullptr};
    return visit_objective(o, [](auto f) -> int {
             return rows_built<decltype(f)>() ? 1 : 0;
           }) == 1;
  }

  int
  launch_rows(const Objective& o, const zeus_bfgs_config& c, const BfgsParams& prm,
              const double* starts, const RunOut& out, Control* ctl, void* ws,
              size_t ws_bytes, cudaStream_t st)
  {
    const bool adjoint = c.gradient == ZEUS_GRAD_ADJOINT;
    return visit_objective(o, [&](auto f) -> int {
      using F = decltype(f);
      constexpr int D = (int)F::arity;
      if constexpr (rows_built<F>()) {
        // the cycle timers are compiled in only where they are asked for
        const bool timed = out.cycles != nullptr;
        if (adjoint && timed)
          return launch_rows_one<F, D, true, true>(f, prm, starts, out, ctl, ws, ws_bytes,
                                                   st);
        if (adjoint)
          return launch_rows_one<F, D, true, false>(f, prm, starts, out, ctl, ws, ws_bytes,
                                                    st);
        if (timed)
          return launch_rows_one<F, D, false, true>(f, prm, starts, out, ctl, ws,
                                                    ws_bytes, st);
        return launch_rows_one<F, D, false, false>(f, prm, starts, out, ctl, ws, ws_bytes,
                                                   st);
      } else {
        set_error("row layout: kind %d dim %d not built", F::kind, D);
        return ZEUS_E_UNSUPPORTED;
      }
    });
  }

  bool
  cta_layout_supported(int kind, int dim)
  {
    if (!builtin_supported(kind, dim) || dim < kMinCtaDim)
      return false;
    const int b = dim <= 64 ? 256 : 512;
    // the larger of the two variants (warp trials need an extra D per warp)
    return cta_smem_doubles_rt(dim, b, true) * sizeof(double) <= kSmemLimit;
  }

  size_t
  cta_workspace_bytes(int dim, int64_t n)
  {
    if (dim < 32 || n <= 0)
      return 0;
    if (dim < kMinCtaDim) // the row layout's run queue
      return kQueueBytes;
    const int b = dim <= 64 ? 256 : 512;
    return kQueueBytes +
           (cta_h_global(dim, b)
              ? sizeof(double) * (size_t)dim * dim * (size_t)global_h_slices(n)
              : 0);
  }

  int
  launch_cta(const Objective& o, const zeus_bfgs_config& c,
             const BfgsParams& prm, const double* starts, const RunOut& out,
             Control* ctl, void* ws, size_t ws_bytes, cudaStream_t st)
  {
    const bool adjoint = c.gradient == ZEUS_GRAD_ADJOINT;
    return visit_objective(o, [&](auto f) -> int {
      using F = decltype(f);
      constexpr int D = (int)F::arity;
      if constexpr (D >= kMinCtaDim &&
                    sizeof(double) * cta_smem_doubles_rt(D, cta_block<D>(), true) <=
                      kSmemLimit) {
        // the cycle timers are compiled in only where they are asked for
        const bool timed = out.cycles != nullptr;
        if (adjoint && timed)
          return launch_one<F, D, true, true>(f, prm, starts, out, ctl, ws, ws_bytes, st);
        if (adjoint)
          return launch_one<F, D, true, false>(f, prm, starts, out, ctl, ws, ws_bytes, st);
        if (timed)
          return launch_one<F, D, false, true>(f, prm, starts, out, ctl, ws, ws_bytes, st);
        return launch_one<F, D, false, false>(f, prm, starts, out, ctl, ws, ws_bytes, st);
      } else {
        set_error("CTA layout: dim %d not built", D);
        return ZEUS_E_UNSUPPORTED;
      }
    });
  }

} // namespace zb
