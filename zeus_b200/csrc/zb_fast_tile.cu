// Tile-per-run fast BFGS launcher (2 <= D <= 32, tile widths 2..32).
#include "zb_bfgs_coop.cuh"
#include "zb_objective_visit.cuh"

namespace zb {

  namespace {
    template <class F, int D, int TS>
    int
    launch_ts(const F& f, bool adjoint, const BfgsParams& prm,
              const double* starts, const RunOut& out, Control* ctl,
              cudaStream_t st)
    {
      constexpr int TPB = kTileBlock / TS;
      const unsigned grid = (unsigned)((prm.n + TPB - 1) / TPB);
      const size_t smem = sizeof(double) * TPB * tile_smem_doubles<D, TS>();
      // the cycle timers are compiled in only where they are asked for
      const bool timed = out.cycles != nullptr;
      if (adjoint && timed)
        bfgs_tile_kernel<F, D, TS, true, true>
          <<<grid, kTileBlock, smem, st>>>(f, prm, starts, out, ctl);
      else if (adjoint)
        bfgs_tile_kernel<F, D, TS, true>
          <<<grid, kTileBlock, smem, st>>>(f, prm, starts, out, ctl);
      else if (timed)
        bfgs_tile_kernel<F, D, TS, false, true>
          <<<grid, kTileBlock, smem, st>>>(f, prm, starts, out, ctl);
      else
        bfgs_tile_kernel<F, D, TS, false>
          <<<grid, kTileBlock, smem, st>>>(f, prm, starts, out, ctl);
      return cuda_fail(cudaGetLastError(), "tile-layout BFGS launch");
    }
  } // namespace

  unsigned
  tile_widths(int kind, int dim)
  {
    return builtin_supported(kind, dim) ? tile_widths_for(kind, dim) : 0u;
  }

  int
  launch_tile(const Objective& o, const zeus_bfgs_config& c, int tile,
              const BfgsParams& prm, const double* starts, const RunOut& out,
              Control* ctl, cudaStream_t st)
  {
    const bool adjoint = c.gradient == ZEUS_GRAD_ADJOINT;
    return visit_objective(o, [&](auto f) -> int {
      using F = decltype(f);
      constexpr int D = (int)F::arity;
      constexpr unsigned W = tile_widths_for(F::kind, D);
      switch (tile) {
#define ZB_TS(K)                                                               \
  case (1 << K):                                                               \
    if constexpr ((W >> K) & 1u)                                               \
      return launch_ts<F, D, (1 << K)>(f, adjoint, prm, starts, out, ctl, st); \
    break;
        ZB_TS(1)
        ZB_TS(2)
        ZB_TS(3)
        ZB_TS(4)
        ZB_TS(5)
#undef ZB_TS
      }
      set_error("tile layout: width %d not built for dim %d", tile, D);
      return ZEUS_E_UNSUPPORTED;
    });
  }

} // namespace zb
