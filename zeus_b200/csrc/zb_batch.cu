// Persistent batched BFGS kernel and its C ABI (zeus_batch_*).
#include <algorithm>
#include <vector>

#include "zb_batch.cuh"
#include "zb_objective_visit.cuh"
#include "zb_reduce.cuh"

namespace zb {

  namespace {

    // Device-side (kind, dim) -> functor, for the dimensions the library is
    // built for (the same sets as visit_objective).
    template <class Fn>
    __device__ __forceinline__ void
    batch_visit(const BatchClass& c, Fn&& fn)
    {
      switch (c.kind) {
        case ZEUS_OBJ_ROSENBROCK:
          switch (c.dim) {
#define ZB_CASE(D)                                                             \
  case D:                                                                      \
    fn(zeus::Rosenbrock<D>{});                                                 \
    return;
            ZB_ROSENBROCK_DIMS(ZB_CASE)
#undef ZB_CASE
          }
          return;
        case ZEUS_OBJ_RASTRIGIN:
          switch (c.dim) {
#define ZB_CASE(D)                                                             \
  case D:                                                                      \
    fn(zeus::Rastrigin<D>{});                                                  \
    return;
            ZB_RASTRIGIN_DIMS(ZB_CASE)
#undef ZB_CASE
          }
          return;
        case ZEUS_OBJ_ACKLEY:
          switch (c.dim) {
#define ZB_CASE(D)                                                             \
  case D:                                                                      \
    fn(zeus::Ackley<D>{});                                                     \
    return;
            ZB_ACKLEY_DIMS(ZB_CASE)
#undef ZB_CASE
          }
          return;
        case ZEUS_OBJ_GAUSSIAN:
          switch (c.dim) {
#define ZB_CASE(D)                                                             \
  case D: {                                                                    \
    zeus::Gaussian<D> g;                                                       \
    g.C = c.data;                                                              \
    g.symmetric = (c.flags & 1) != 0;                                          \
    fn(g);                                                                     \
    return;                                                                    \
  }
            ZB_GAUSSIAN_DIMS(ZB_CASE)
#undef ZB_CASE
          }
          return;
        case ZEUS_OBJ_POISSON_NLL:
          if (c.dim == 4) {
            zeus::PoissonNLL p;
            p.centres = c.data;
            p.counts = c.idata;
            p.bins = c.nll_bins;
            p.nbins = c.ndata;
            fn(p);
          }
          return;
      }
    }

    template <class F>
    __device__ __forceinline__ F
    instance_for(const F& f, const BatchClass& c, int64_t run)
    {
      return c.runs_per_instance > 0 ? with_instance(f, c, run / c.runs_per_instance)
                                     : f;
    }

    template <class F, int D, int TS>
    __device__ __forceinline__ void
    drain_tile_class(const F& f, const BatchClass& c, const BfgsParams& prm,
                     double* warp_buf)
    {
      auto tile = cg::tiled_partition<TS>(cg::this_thread_block());
      const int tin = (int)(threadIdx.x & 31) / TS;
      double* buf = warp_buf + tin * (4 * D + TS);
      for (;;) {
        unsigned long long r = 0;
        if (tile.thread_rank() == 0)
          r = atomicAdd(c.queue, 1ull);
        r = tile.shfl(r, 0);
        if ((int64_t)r >= c.n)
          break;
        tile_run<F, D, TS, true>(instance_for(f, c, (int64_t)r), tile, buf, prm,
                                 c.starts + (int64_t)r * D, (int64_t)r, c.out,
                                 c.ctl);
      }
    }

  } // namespace

  __global__ void __launch_bounds__(kBatchBlock, 1)
    bfgs_batch_kernel(const __grid_constant__ BatchTable bt)
  {
    const int ncls = bt.ncls;
    const BatchClass* classes = bt.c;
    extern __shared__ double sm[];
    __shared__ unsigned long long sh_run;

    // phase A: CTA-layout classes, one run per block at a time
    for (int ci = 0; ci < ncls; ++ci) {
      const BatchClass c = classes[ci];
      if (c.layout != ZEUS_LAYOUT_CTA)
        continue;
      const BfgsParams prm{c.n, bt.max_iter, c.required, bt.tol, bt.flags};
      for (;;) {
        if (threadIdx.x == 0)
          sh_run = atomicAdd(c.queue, 1ull);
        __syncthreads();
        const int64_t r = (int64_t)sh_run;
        __syncthreads();
        if (r >= c.n)
          break;
        batch_visit(c, [&](auto f) {
          using F = decltype(f);
          constexpr int D = (int)F::arity;
          if constexpr (D >= kBatchCtaMinDim &&
                        sizeof(double) * cta_smem_doubles<F, D, true>(kBatchBlock) <=
                          227 * 1024)
            cta_run<F, D, true, kBatchBlock>(instance_for(f, c, r), sm, prm,
                                             c.starts + r * D, r, c.out, c.ctl);
        });
      }
    }
    __syncthreads();

    // phase B: each warp drains the tile / thread classes
    double* warp_buf = nullptr;
    {
      // per-warp buffers follow each other; sized by the host for the
      // widest class of the batch
      const int warp = threadIdx.x >> 5;
      size_t stride = 0;
      for (int ci = 0; ci < ncls; ++ci)
        if (classes[ci].layout == ZEUS_LAYOUT_TILE)
          stride = stride > batch_tile_buf_doubles(classes[ci].dim, classes[ci].tile)
                     ? stride
                     : batch_tile_buf_doubles(classes[ci].dim, classes[ci].tile);
      warp_buf = sm + (size_t)warp * stride;
    }
    for (int ci = 0; ci < ncls; ++ci) {
      const BatchClass c = classes[ci];
      if (c.layout == ZEUS_LAYOUT_CTA)
        continue;
      const BfgsParams prm{c.n, bt.max_iter, c.required, bt.tol, bt.flags};
      batch_visit(c, [&](auto f) {
        using F = decltype(f);
        constexpr int D = (int)F::arity;
        if (c.layout == ZEUS_LAYOUT_THREAD) {
          if constexpr (D <= kBatchThreadMaxDim) {
            for (;;) {
              const int64_t r = (int64_t)atomicAdd(c.queue, 1ull);
              if (r >= c.n)
                break;
              thread_run<F, D, true>(instance_for(f, c, r), prm,
                                     c.starts + r * D, r, c.out, c.ctl);
            }
          }
        } else if constexpr (D < kBatchCtaMinDim) {
          constexpr unsigned W = batch_widths(F::kind, D);
          switch (c.tile) {
#define ZB_TS(K)                                                               \
  case (1 << K):                                                               \
    if constexpr ((W >> K) & 1u)                                               \
      drain_tile_class<F, D, (1 << K)>(f, c, prm, warp_buf);                   \
    break;
            ZB_TS(1)
            ZB_TS(2)
            ZB_TS(3)
            ZB_TS(4)
            ZB_TS(5)
#undef ZB_TS
          }
        }
      });
      __syncwarp();
    }
  }

  namespace {
    // shared memory of a CTA-layout class (the Gaussian's trials carry the
    // gradient and need no per-warp trial points)
    size_t
    cta_doubles_rt(int kind, int d, int block)
    {
      return cta_smem_doubles_rt(d, block, kind != ZEUS_OBJ_GAUSSIAN);
    }

    bool
    batch_layout_ok(int kind, int dim, int layout, int tile)
    {
      if (!builtin_supported(kind, dim))
        return false;
      if (layout == ZEUS_LAYOUT_THREAD)
        return dim <= kBatchThreadMaxDim;
      if (layout == ZEUS_LAYOUT_TILE)
        return tile >= 2 && tile <= 32 && !(tile & (tile - 1)) &&
               ((batch_widths(kind, dim) >> __builtin_ctz((unsigned)tile)) & 1u);
      if (layout == ZEUS_LAYOUT_CTA)
        return dim >= kBatchCtaMinDim &&
               cta_doubles_rt(kind, dim, kBatchBlock) * sizeof(double) <= 227 * 1024;
      return false;
    }

    void
    batch_default(int kind, int dim, int gradient, int* layout, int* tile)
    {
      *tile = 0;
      int l = 0, t = 0;
      if (zeus_autotune_lookup(kind, dim, gradient, &l, &t) &&
          batch_layout_ok(kind, dim, l, t)) {
        *layout = l;
        *tile = t;
        return;
      }
      if (dim <= kBatchThreadMaxDim) {
        *layout = ZEUS_LAYOUT_THREAD;
        return;
      }
      if (dim < kBatchCtaMinDim) {
        const unsigned w = batch_widths(kind, dim);
        for (int k = 1; k <= 5; ++k)
          if ((w >> k) & 1u) {
            *layout = ZEUS_LAYOUT_TILE;
            *tile = 1 << k;
            return;
          }
      }
      *layout = ZEUS_LAYOUT_CTA;
    }

    int64_t
    instances(const zeus_batch_class& c)
    {
      return c.runs_per_instance > 0
               ? (c.n + c.runs_per_instance - 1) / c.runs_per_instance
               : 1;
    }

    size_t
    ws_layout(const zeus_batch_class* cls, int ncls, size_t* off_queue,
              std::vector<size_t>* off_bins)
    {
      size_t b = 0;
      *off_queue = b;
      b += align_up(sizeof(unsigned long long) * (size_t)ncls);
      off_bins->assign(ncls, 0);
      for (int i = 0; i < ncls; ++i)
        if (cls[i].problem.kind == ZEUS_OBJ_POISSON_NLL) {
          (*off_bins)[i] = b;
          b += align_up(sizeof(double) * 4 * (size_t)cls[i].problem.ndata *
                        instances(cls[i]));
        }
      return b;
    }
  } // namespace

} // namespace zb

using namespace zb;

extern "C" {

size_t
zeus_batch_workspace_size(const zeus_batch_class* classes, int32_t n_classes)
{
  if (!classes || n_classes <= 0)
    return 0;
  size_t oq;
  std::vector<size_t> ob;
  return ws_layout(classes, n_classes, &oq, &ob);
}

int
zeus_batch_device(const zeus_batch_class* classes, int32_t n_classes,
                  const zeus_bfgs_config* config, void* d_workspace,
                  size_t workspace_bytes, void* stream)
{
  if (!classes || n_classes <= 0 || n_classes > kMaxBatchClasses || !config) {
    set_error("zeus_batch_device: 1..%d classes and a config are required",
              kMaxBatchClasses);
    return ZEUS_E_INVALID;
  }
  if (config->mode != ZEUS_MODE_FAST || config->gradient != ZEUS_GRAD_ADJOINT) {
    set_error("zeus_batch_device runs fast mode with adjoint gradients");
    return ZEUS_E_INVALID;
  }
  if (config->max_iter < 0 || !(config->tolerance >= 0.0)) {
    set_error("zeus_batch_device: max_iter >= 0 and tolerance >= 0 required");
    return ZEUS_E_INVALID;
  }
  size_t off_q;
  std::vector<size_t> off_b;
  const size_t need = ws_layout(classes, n_classes, &off_q, &off_b);
  if (!d_workspace || workspace_bytes < need) {
    set_error("zeus_batch_device: workspace of %zu bytes needed, got %zu", need,
              workspace_bytes);
    return ZEUS_E_WORKSPACE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = static_cast<char*>(d_workspace);
  auto* queues = reinterpret_cast<unsigned long long*>(ws + off_q);
  std::vector<BatchClass> hc;
  hc.reserve(n_classes);
  size_t smem_cta = 0, smem_tile = 0;
  for (int i = 0; i < n_classes; ++i) {
    const zeus_batch_class& c = classes[i];
    const zeus_problem& p = c.problem;
    if (!builtin_supported(p.kind, p.dim) || c.n < 0 ||
        (c.n > 0 && (!c.d_starts || !c.d_control)) ||
        (p.kind == ZEUS_OBJ_GAUSSIAN && !p.data) ||
        (p.kind == ZEUS_OBJ_POISSON_NLL && (!p.data || !p.idata || p.ndata <= 0))) {
      set_error("zeus_batch_device: class %d is invalid or not built", i);
      return ZEUS_E_INVALID;
    }
    int layout = c.layout, tile = c.tile;
    if (layout == ZEUS_LAYOUT_AUTO)
      batch_default(p.kind, p.dim, config->gradient, &layout, &tile);
    if (!batch_layout_ok(p.kind, p.dim, layout, tile)) {
      set_error("zeus_batch_device: class %d layout %d tile %d not built", i,
                layout, tile);
      return ZEUS_E_UNSUPPORTED;
    }
    BatchClass b{};
    b.kind = p.kind;
    b.dim = p.dim;
    b.layout = layout;
    b.tile = tile;
    b.n = c.n;
    b.starts = c.d_starts;
    b.out = RunOut{c.out.fval,   c.out.status, c.out.iter,   c.out.gnorm,
                   c.out.x,      c.out.counters, nullptr,     nullptr,
                   nullptr,      nullptr};
    b.ctl = reinterpret_cast<Control*>(c.d_control);
    b.data = p.data;
    b.idata = p.idata;
    b.ndata = p.ndata;
    b.flags = p.flags;
    b.runs_per_instance = c.runs_per_instance;
    b.queue = queues + i;
    b.required = c.required_converged;
    if (p.kind == ZEUS_OBJ_POISSON_NLL) {
      double* bins = reinterpret_cast<double*>(ws + off_b[i]);
      const int64_t nb = (int64_t)p.ndata * instances(c);
      nll_bins_kernel<<<(unsigned)((nb + 127) / 128), 128, 0, st>>>(
        p.data, p.idata, (int)nb, bins);
      int rc = cuda_fail(cudaGetLastError(), "NLL bins launch");
      if (rc)
        return rc;
      b.nll_bins = bins;
    }
    if (layout == ZEUS_LAYOUT_CTA)
      smem_cta = std::max(smem_cta, cta_doubles_rt(p.kind, p.dim, kBatchBlock));
    if (layout == ZEUS_LAYOUT_TILE)
      smem_tile = std::max(smem_tile, batch_tile_buf_doubles(p.dim, tile));
    hc.push_back(b);
  }
  // biggest work first: CTA classes by dimension, then the rest by dimension
  std::stable_sort(hc.begin(), hc.end(), [](const BatchClass& a, const BatchClass& b) {
    const int ka = a.layout == ZEUS_LAYOUT_CTA, kb = b.layout == ZEUS_LAYOUT_CTA;
    if (ka != kb)
      return ka > kb;
    return a.dim > b.dim;
  });
  int rc = cuda_fail(cudaMemsetAsync(queues, 0,
                                     sizeof(unsigned long long) * n_classes, st),
                     "batch queue reset");
  if (rc)
    return rc;
  BatchTable bt{};
  bt.ncls = n_classes;
  bt.max_iter = config->max_iter;
  bt.tol = config->tolerance;
  bt.flags = config->flags;
  for (int i = 0; i < n_classes; ++i)
    bt.c[i] = hc[i];
  const size_t smem =
    sizeof(double) * std::max(smem_cta, smem_tile * (kBatchBlock / 32));
  rc = cuda_fail(cudaFuncSetAttribute(bfgs_batch_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem),
                 "batch shared memory attribute");
  if (rc)
    return rc;
  int per_sm = 0;
  rc = cuda_fail(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                   &per_sm, bfgs_batch_kernel, kBatchBlock, smem),
                 "batch occupancy");
  if (rc)
    return rc;
  if (per_sm < 1) {
    set_error("batch kernel does not fit on an SM (%zu bytes of shared memory)",
              smem);
    return ZEUS_E_UNSUPPORTED;
  }
  bfgs_batch_kernel<<<sm_count() * per_sm, kBatchBlock, smem, st>>>(bt);
  return cuda_fail(cudaGetLastError(), "batch BFGS launch");
}

} // extern "C"
