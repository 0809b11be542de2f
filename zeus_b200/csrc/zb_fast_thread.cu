// Thread-per-run fast BFGS launcher (D <= 10).
#include "zb_bfgs_thread.cuh"
#include "zb_objective_visit.cuh"

namespace zb {

  namespace {
    constexpr int kThreadBlock = 128;
    constexpr int kMaxThreadDim = 10;
  } // namespace

  bool
  thread_layout_supported(int kind, int dim)
  {
    return builtin_supported(kind, dim) && dim <= kMaxThreadDim;
  }

  int
  launch_thread(const Objective& o, const zeus_bfgs_config& c,
                const BfgsParams& prm, const double* starts, const RunOut& out,
                Control* ctl, cudaStream_t st)
  {
    const bool adjoint = c.gradient == ZEUS_GRAD_ADJOINT;
    return visit_objective(o, [&](auto f) -> int {
      using F = decltype(f);
      constexpr int D = (int)F::arity;
      if constexpr (D <= kMaxThreadDim) {
        const int block = c.block > 0 ? c.block : kThreadBlock;
        const unsigned grid = (unsigned)((prm.n + block - 1) / block);
        // the cycle timers are compiled in only where they are asked for
        const bool timed = out.cycles != nullptr;
        if (adjoint && timed)
          bfgs_thread_kernel<F, D, true, true>
            <<<grid, block, 0, st>>>(f, prm, starts, out, ctl);
        else if (adjoint)
          bfgs_thread_kernel<F, D, true>
            <<<grid, block, 0, st>>>(f, prm, starts, out, ctl);
        else if (timed)
          bfgs_thread_kernel<F, D, false, true>
            <<<grid, block, 0, st>>>(f, prm, starts, out, ctl);
        else
          bfgs_thread_kernel<F, D, false>
            <<<grid, block, 0, st>>>(f, prm, starts, out, ctl);
        return cuda_fail(cudaGetLastError(), "thread-layout BFGS launch");
      } else {
        set_error("thread layout: dim %d not built", D);
        return ZEUS_E_UNSUPPORTED;
      }
    });
  }

} // namespace zb
