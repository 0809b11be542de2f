// Fast-mode BFGS launchers: layout chosen by dimension.
#include "zb_bfgs_thread.cuh"
#include "zb_objective_visit.cuh"

namespace zb {

  namespace {
    constexpr int kThreadBlock = 128;
    constexpr int kMaxThreadDim = 10; // H (55 doubles) + vectors in registers
  } // namespace

  bool
  fast_supported(int kind, int dim, int gradient)
  {
    (void)gradient;
    return builtin_supported(kind, dim) && dim <= kMaxThreadDim;
  }

  size_t
  fast_workspace_bytes(const Objective& o, const zeus_bfgs_config& c,
                       int64_t n)
  {
    (void)o;
    (void)c;
    (void)n;
    return 0;
  }

  int
  launch_fast(const Objective& o, const zeus_bfgs_config& c,
              const BfgsParams& prm, const double* starts, const RunOut& out,
              Control* ctl, void* ws, size_t ws_bytes, cudaStream_t st)
  {
    (void)ws;
    (void)ws_bytes;
    if (prm.n <= 0)
      return ZEUS_OK;
    const bool adjoint = c.gradient == ZEUS_GRAD_ADJOINT;
    return visit_objective(o, [&](auto f) -> int {
      using F = decltype(f);
      constexpr int D = (int)F::arity;
      if constexpr (D <= kMaxThreadDim) {
        const int block = c.block > 0 ? c.block : kThreadBlock;
        const unsigned grid = (unsigned)((prm.n + block - 1) / block);
        if (adjoint)
          bfgs_thread_kernel<F, D, true>
            <<<grid, block, 0, st>>>(f, prm, starts, out, ctl);
        else
          bfgs_thread_kernel<F, D, false>
            <<<grid, block, 0, st>>>(f, prm, starts, out, ctl);
        return cuda_fail(cudaGetLastError(), "fast BFGS launch");
      } else {
        set_error("fast BFGS: dim %d has no layout built", D);
        return ZEUS_E_UNSUPPORTED;
      }
    });
  }

} // namespace zb
