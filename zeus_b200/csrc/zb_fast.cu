// Fast-mode dispatcher: picks the layout for (objective, dimension) unless
// the configuration names one (the autotuner sweeps them that way).
#include "zb_objective_visit.cuh"

namespace zb {

  // The layout by dimension when neither the configuration nor the
  // autotuner names one: a thread per run with H in registers for D <= 8, a
  // warp per run (H rows in lane registers) up to D = 32, a block per run
  // with H in shared memory above.
  void
  default_layout(int kind, int dim, int* layout, int* tile)
  {
    *tile = 0;
    if (dim <= 8 && thread_layout_supported(kind, dim)) {
      *layout = ZEUS_LAYOUT_THREAD;
      return;
    }
    const unsigned w = tile_widths(kind, dim);
    if (w) {
      for (int k = 5; k >= 1; --k) // the widest built, a warp when it is
        if ((w >> k) & 1u) {
          *tile = 1 << k;
          break;
        }
      *layout = ZEUS_LAYOUT_TILE;
      return;
    }
    if (cta_layout_supported(kind, dim)) {
      *layout = ZEUS_LAYOUT_CTA;
      return;
    }
    *layout = thread_layout_supported(kind, dim) ? ZEUS_LAYOUT_THREAD : -1;
  }

  bool
  fast_supported(int kind, int dim, int gradient)
  {
    (void)gradient;
    return builtin_supported(kind, dim) &&
           (thread_layout_supported(kind, dim) || tile_widths(kind, dim) != 0 ||
            cta_layout_supported(kind, dim) || rows_layout_supported(kind, dim));
  }

  // Only the CTA and row layouts need one: their run queue, and past about
  // D = 160 the CTA blocks' H slices.
  size_t
  fast_workspace_bytes(const Objective& o, const zeus_bfgs_config& c,
                       int64_t n)
  {
    (void)c;
    return cta_workspace_bytes(o.dim, n);
  }

  int
  launch_fast(const Objective& o, const zeus_bfgs_config& c,
              const BfgsParams& prm, const double* starts, const RunOut& out,
              Control* ctl, void* ws, size_t ws_bytes, cudaStream_t st)
  {
    if (prm.n <= 0)
      return ZEUS_OK;
    int layout = c.layout, tile = c.tile;
    if (layout == ZEUS_LAYOUT_AUTO &&
        !zeus_autotune_lookup(o.kind, o.dim, c.gradient, &layout, &tile))
      default_layout(o.kind, o.dim, &layout, &tile);
    switch (layout) {
      case ZEUS_LAYOUT_THREAD:
        if (!thread_layout_supported(o.kind, o.dim))
          break;
        return launch_thread(o, c, prm, starts, out, ctl, st);
      case ZEUS_LAYOUT_TILE: {
        const unsigned w = tile_widths(o.kind, o.dim);
        if (tile == 0) {
          int l2;
          default_layout(o.kind, o.dim, &l2, &tile);
          if (l2 != ZEUS_LAYOUT_TILE)
            tile = 0;
        }
        if (tile < 2 || tile > 32 || (tile & (tile - 1)) ||
            !((w >> __builtin_ctz((unsigned)tile)) & 1u))
          break;
        return launch_tile(o, c, tile, prm, starts, out, ctl, st);
      }
      case ZEUS_LAYOUT_CTA:
        if (!cta_layout_supported(o.kind, o.dim))
          break;
        return launch_cta(o, c, prm, starts, out, ctl, ws, ws_bytes, st);
      case ZEUS_LAYOUT_ROWS:
        if (!rows_layout_supported(o.kind, o.dim))
          break;
        return launch_rows(o, c, prm, starts, out, ctl, ws, ws_bytes, st);
      default:
        break;
    }
    set_error("fast BFGS: layout %d (tile %d) is not built for kind %d dim %d",
              layout, tile, o.kind, o.dim);
    return ZEUS_E_UNSUPPORTED;
  }

} // namespace zb
