// Exact-mode BFGS and PSO launchers.  Compiled with -fmad=false (see
// zeus_b200/build.py): no multiply-add contraction, so every basic
// operation rounds as in the reference built for the host.
#include "zb_bfgs_exact.cuh"
#include "zb_objective_visit.cuh"
#include "zb_pso.cuh"
#include "zb_pso_dmma.cuh"

namespace zb {

  namespace {
    constexpr int kExactBlock = 128;

    int
    exact_grid(int64_t n)
    {
      const int64_t g = (int64_t)sm_count() * 4;
      return (int)(n < g ? n : g);
    }
  } // namespace

  bool
  exact_supported(int kind, int dim)
  {
    return builtin_supported(kind, dim);
  }

  size_t
  exact_workspace_bytes(const Objective& o, int64_t n)
  {
    if (n <= 0)
      return 0;
    return sizeof(double) * 2 * (size_t)o.dim * o.dim * exact_grid(n);
  }

  int
  launch_exact(const Objective& o, const BfgsParams& prm,
               const double* starts, const RunOut& out, Control* ctl,
               void* ws, size_t ws_bytes, cudaStream_t st)
  {
    if (prm.n <= 0)
      return ZEUS_OK;
    const size_t need = exact_workspace_bytes(o, prm.n);
    if (ws_bytes < need || !ws) {
      set_error("exact BFGS needs %zu workspace bytes, got %zu", need,
                ws_bytes);
      return ZEUS_E_WORKSPACE;
    }
    const bool traj = out.traj_x && out.traj_f && out.traj_g &&
                      out.traj_status;
    return visit_objective(o, [&](auto f) -> int {
      using F = decltype(f);
      constexpr int D = (int)F::arity;
      const int grid = exact_grid(prm.n);
      const size_t smem = exact_smem_bytes<D>();
      double* scratch = static_cast<double*>(ws);
      if (traj)
        bfgs_exact_kernel<F, D, true>
          <<<grid, kExactBlock, smem, st>>>(f, prm, starts, out, ctl, scratch);
      else
        bfgs_exact_kernel<F, D, false>
          <<<grid, kExactBlock, smem, st>>>(f, prm, starts, out, ctl, scratch);
      return cuda_fail(cudaGetLastError(), "exact BFGS launch");
    });
  }

  bool
  pso_supported(int kind, int dim)
  {
    return builtin_supported(kind, dim);
  }

  size_t
  pso_workspace_bytes(int64_t n, int dim)
  {
    const int64_t blocks = pso_blocks(n, dim);
    size_t b = 0;
    b += align_up(sizeof(double) * (size_t)n * dim); // X
    b += align_up(sizeof(double) * (size_t)n * dim); // V
    b += align_up(sizeof(unsigned long long) * (size_t)blocks);
    b += align_up(sizeof(int) * (size_t)blocks);
    b += align_up(sizeof(unsigned int));
    return b;
  }

  int
  launch_pso(const Objective& o, uint64_t seed, int64_t n, double lower,
             double upper, int iters, double w, double c1, double c2,
             double* pbx, double* pbf, double* gbest, void* ws,
             size_t ws_bytes, cudaStream_t st, const uint32_t* sobol)
  {
    if (n <= 0)
      return ZEUS_OK;
    const size_t need = pso_workspace_bytes(n, o.dim);
    if (!ws || ws_bytes < need) {
      set_error("PSO needs %zu workspace bytes, got %zu", need, ws_bytes);
      return ZEUS_E_WORKSPACE;
    }
    const int64_t blocks = pso_blocks(n, o.dim);
    char* p = static_cast<char*>(ws);
    PsoWork wk;
    wk.X = reinterpret_cast<double*>(p);
    p += align_up(sizeof(double) * (size_t)n * o.dim);
    wk.V = reinterpret_cast<double*>(p);
    p += align_up(sizeof(double) * (size_t)n * o.dim);
    wk.part_key = reinterpret_cast<unsigned long long*>(p);
    p += align_up(sizeof(unsigned long long) * (size_t)blocks);
    wk.part_idx = reinterpret_cast<int*>(p);
    p += align_up(sizeof(int) * (size_t)blocks);
    wk.counter = reinterpret_cast<unsigned int*>(p);
    wk.gbest = gbest;
    wk.sobol = sobol;
    return visit_objective(o, [&](auto f) -> int {
      using F = decltype(f);
      constexpr int D = (int)F::arity;
      pso_reset_kernel<D><<<1, 256, 0, st>>>(wk);
      if constexpr (D >= kPsoCoopMinDim && D <= kPsoDmmaMaxDim &&
                    F::kind == ZEUS_OBJ_GAUSSIAN) {
        // f = 0.5 x^T C x for 8 particles per warp on the FP64 tensor cores
        const unsigned b8 = (unsigned)pso_dmma_blocks(n);
        pso_init_dmma_kernel<D><<<b8, kPsoBlock, 0, st>>>(f, n, lower, upper, seed,
                                                          wk, pbx, pbf);
        for (int t = 1; t <= iters; ++t)
          pso_iter_dmma_kernel<D><<<b8, kPsoBlock, 0, st>>>(f, n, w, c1, c2, seed, t,
                                                            wk, pbx, pbf);
      } else if constexpr (D >= kPsoCoopMinDim) {
        pso_init_coop_kernel<F, D><<<(unsigned)blocks, kPsoBlock, 0, st>>>(
          f, n, lower, upper, seed, wk, pbx, pbf);
        for (int t = 1; t <= iters; ++t)
          pso_iter_coop_kernel<F, D><<<(unsigned)blocks, kPsoBlock, 0, st>>>(
            f, n, w, c1, c2, seed, t, wk, pbx, pbf);
      } else {
        pso_init_kernel<F, D><<<(unsigned)blocks, kPsoBlock, 0, st>>>(
          f, n, lower, upper, seed, wk, pbx, pbf);
        for (int t = 1; t <= iters; ++t)
          pso_iter_kernel<F, D><<<(unsigned)blocks, kPsoBlock, 0, st>>>(
            f, n, w, c1, c2, seed, t, wk, pbx, pbf);
      }
      return cuda_fail(cudaGetLastError(), "PSO launch");
    });
  }

} // namespace zb
