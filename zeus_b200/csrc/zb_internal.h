// Host-side interface between the library's translation units:
//   zb_exact.cu  (-fmad=false): exact-mode BFGS and PSO launchers
//   zb_fast.cu   : fast-mode BFGS launchers (thread / tile / CTA layouts)
//   zb_runtime.cu: the C ABI (include/zeus_b200.h), reductions, orchestration
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "zeus_b200.h"
#include "zb_common.cuh"

namespace zb {

  // A built-in objective with its data resolved to device pointers.
  struct Objective {
    int kind;
    int dim;
    const double* data;    // Gaussian C / NLL centres
    const int* idata;      // NLL counts
    int ndata;             // NLL bins
    int flags;             // bit 0: Gaussian C is symmetric
    const double* nll_bins; // NLL {ln x, ln(1-x), k, lgamma(k+1)} per bin
  };

  void set_error(const char* fmt, ...);
  int cuda_fail(cudaError_t e, const char* what);
  int sm_count();

  // exact mode (zb_exact.cu)
  bool exact_supported(int kind, int dim);
  size_t exact_workspace_bytes(const Objective& o, int64_t n);
  int launch_exact(const Objective& o, const BfgsParams& prm,
                   const double* starts, const RunOut& out, Control* ctl,
                   void* ws, size_t ws_bytes, cudaStream_t st);

  // PSO (zb_exact.cu)
  bool pso_supported(int kind, int dim);
  size_t pso_workspace_bytes(int64_t n, int dim);
  int launch_pso(const Objective& o, uint64_t seed, int64_t n, double lower,
                 double upper, int iters, double w, double c1, double c2,
                 double* pbx, double* pbf, double* gbest, void* ws,
                 size_t ws_bytes, cudaStream_t st,
                 const uint32_t* sobol = nullptr);

  // Tile widths built for an objective and dimension (bit k: width 2^k):
  // H rows per lane R*D <= 64 doubles; up to 4*D lanes (the spare lanes
  // evaluate line-search trials in parallel), any width where the
  // cooperative evaluation splits something other than the coordinates (the
  // NLL's bins, the Gaussian's C x).
  constexpr unsigned
  tile_widths_for(int kind, int d)
  {
    unsigned m = 0;
    if (d > 32)
      return 0;
    const bool wide = kind == ZEUS_OBJ_POISSON_NLL || kind == ZEUS_OBJ_GAUSSIAN;
    for (int k = 1; k <= 5; ++k) {
      const int ts = 1 << k;
      const int r = (d + ts - 1) / ts;
      if (r * d <= 64 && (wide || ts <= 4 * d))
        m |= 1u << k;
    }
    return m;
  }

  // fast-mode layouts (zb_fast_thread.cu, zb_fast_tile.cu, zb_fast_cta.cu)
  bool thread_layout_supported(int kind, int dim);
  int launch_thread(const Objective& o, const zeus_bfgs_config& c,
                    const BfgsParams& prm, const double* starts,
                    const RunOut& out, Control* ctl, cudaStream_t st);
  // tile widths built for dim (bit k set: width 2^k available)
  unsigned tile_widths(int kind, int dim);
  int launch_tile(const Objective& o, const zeus_bfgs_config& c, int tile,
                  const BfgsParams& prm, const double* starts,
                  const RunOut& out, Control* ctl, cudaStream_t st);
  bool cta_layout_supported(int kind, int dim);
  int launch_cta(const Objective& o, const zeus_bfgs_config& c,
                 const BfgsParams& prm, const double* starts,
                 const RunOut& out, Control* ctl, void* ws, size_t ws_bytes,
                 cudaStream_t st);
  // the row layout (zb_bfgs_rows.cuh): one run per group of S*dim threads,
  // H rows in registers
  bool rows_layout_supported(int kind, int dim);
  int launch_rows(const Objective& o, const zeus_bfgs_config& c,
                  const BfgsParams& prm, const double* starts,
                  const RunOut& out, Control* ctl, void* ws, size_t ws_bytes,
                  cudaStream_t st);
  // workspace of a CTA- or row-layout launch: the run queue, and past about
  // D = 160 the CTA blocks' H slices
  size_t cta_workspace_bytes(int dim, int64_t n);
  // default layout / tile width for (kind, dim): ZEUS_LAYOUT_* and width
  void default_layout(int kind, int dim, int* layout, int* tile);

  // fast mode dispatcher (zb_fast.cu)
  bool fast_supported(int kind, int dim, int gradient);
  size_t fast_workspace_bytes(const Objective& o, const zeus_bfgs_config& c,
                              int64_t n);
  int launch_fast(const Objective& o, const zeus_bfgs_config& c,
                  const BfgsParams& prm, const double* starts,
                  const RunOut& out, Control* ctl, void* ws, size_t ws_bytes,
                  cudaStream_t st);

  // gradient evaluation at given points (zb_grad.cu): path ZEUS_GRADPATH_*
  int launch_gradient(const Objective& o, int path, int gradient, int width,
                      const double* x, const double* p, double alpha,
                      int64_t n, double* fo, double* go, cudaStream_t st);

  inline size_t
  align_up(size_t v, size_t a = 256)
  {
    return (v + a - 1) / a * a;
  }

} // namespace zb
