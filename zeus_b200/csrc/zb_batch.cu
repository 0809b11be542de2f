// Host side of the persistent batched BFGS (zeus_batch_*): validates the
// classes, picks layouts and the block size, and launches one of the kernel
// instantiations (zb_batch_512.cu, zb_batch_384.cu).
#include <algorithm>
#include <map>
#include <vector>

#include "zb_batch.cuh"
#include "zb_bfgs_rows.cuh"
#include "zb_objective_visit.cuh"
#include "zb_reduce.cuh"

namespace zb {

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
      if (layout == ZEUS_LAYOUT_ROWS) // H rows in registers, both block sizes
        return dim >= kBatchRowMinDim && kind != ZEUS_OBJ_GAUSSIAN &&
               kind != ZEUS_OBJ_POISSON_NLL && row_warps(dim, kBatchBlockSmall) > 0 &&
               row_warps(dim, kBatchBlockLarge) > 0;
      if (layout == ZEUS_LAYOUT_CTA) // H in shared memory only
        return dim >= kBatchCtaMinDim && !cta_h_global(dim, kBatchBlockSmall) &&
               !cta_h_global(dim, kBatchBlockLarge) &&
               cta_doubles_rt(kind, dim, kBatchBlockSmall) * sizeof(double) <=
                 227 * 1024;
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
        // one H row per lane (the narrowest such tile), else the widest built
        const unsigned w = batch_widths(kind, dim);
        int pick = 0;
        for (int k = 1; k <= 5; ++k)
          if ((w >> k) & 1u) {
            pick = k;
            if ((1 << k) >= dim)
              break;
          }
        if (pick) {
          *layout = ZEUS_LAYOUT_TILE;
          *tile = 1 << pick;
          return;
        }
      }
      *layout = batch_layout_ok(kind, dim, ZEUS_LAYOUT_ROWS, 0) ? ZEUS_LAYOUT_ROWS
                                                                 : ZEUS_LAYOUT_CTA;
    }

    // shared memory (doubles) of a row-layout class: its groups side by side
    size_t
    rows_doubles_rt(int d, int block)
    {
      const int nw = row_warps(d, block);
      return nw > 0 ? (size_t)(block / (32 * nw)) * row_smem_doubles_rt(d, nw) : 0;
    }

    int64_t
    instances(const zeus_batch_class& c)
    {
      return c.runs_per_instance > 0
               ? (c.n + c.runs_per_instance - 1) / c.runs_per_instance
               : 1;
    }

    // Companion classes: row-layout classes whose standalone kernel runs two
    // split groups an SM (D = 128: six warps each, part of H in shared
    // memory).  Inside the batch kernel those groups spill under its
    // register budget, and one 12-warp group runs the class at 3.3 us an
    // iteration per SM against 2.35 in the standalone kernel; so such a
    // class runs in its standalone kernel, launched right after the batch
    // kernel on a second stream: its blocks take each SM as the batch's
    // block there retires (most within a few ms; those holding runs that
    // iterate to MAX_ITER stay), and both end about together.
    constexpr int kCompanionQueueBytes = 256;

    bool
    companion_class(const zeus_problem& p, int layout, int block)
    {
      return layout == ZEUS_LAYOUT_ROWS && block == kBatchBlockSmall &&
             row_split_warps(p.dim, kBatchBlockSmall) > 0 &&
             rows_layout_supported(p.kind, p.dim);
    }

    // A second stream and a fork / join event pair per device and host
    // thread, made once (never destroyed: exit-safe).
    struct SideStream {
      cudaStream_t st = nullptr;
      cudaEvent_t fork = nullptr, join = nullptr;
    };

    int
    side_stream(SideStream** out)
    {
      thread_local std::map<int, SideStream> per_dev;
      int dev = 0;
      int rc = cuda_fail(cudaGetDevice(&dev), "current device");
      if (rc)
        return rc;
      SideStream& s = per_dev[dev];
      if (!s.st) {
        if ((rc = cuda_fail(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking),
                            "batch side stream")) ||
            (rc = cuda_fail(cudaEventCreateWithFlags(&s.fork, cudaEventDisableTiming),
                            "batch fork event")) ||
            (rc = cuda_fail(cudaEventCreateWithFlags(&s.join, cudaEventDisableTiming),
                            "batch join event"))) {
          s = SideStream{};
          return rc;
        }
      }
      *out = &s;
      return ZEUS_OK;
    }

    size_t
    ws_layout(const zeus_batch_class* cls, int ncls, size_t* off_queue,
              std::vector<size_t>* off_bins)
    {
      size_t b = 0;
      *off_queue = b;
      // the batch's per-class queues, then a standalone run queue per class
      // (used by companion classes)
      b += align_up(sizeof(unsigned long long) * (size_t)ncls);
      b += align_up((size_t)kCompanionQueueBytes * ncls);
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
  char* companion_ws =
    ws + off_q + align_up(sizeof(unsigned long long) * (size_t)n_classes);
  std::vector<BatchClass> hc;
  std::vector<int> hc_index; // each entry's position in `classes`
  hc.reserve(n_classes);
  size_t smem_tile = 0;
  double warp_runs = 0.0;
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
    if (c.out.cycles) {
      set_error("zeus_batch_device: class %d asks for cycles, which the batch kernel "
                "does not sample (zeus_bfgs_device does)", i);
      return ZEUS_E_UNSUPPORTED;
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
                   nullptr,      nullptr,        nullptr};
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
    if (layout == ZEUS_LAYOUT_TILE)
      smem_tile = std::max(smem_tile, batch_tile_buf_doubles(p.dim, tile));
    // warps' worth of phase-B runs (a tile of TS lanes is TS/32 of a warp)
    if (layout == ZEUS_LAYOUT_TILE)
      warp_runs += (double)c.n * tile / 32.0;
    else if (layout == ZEUS_LAYOUT_THREAD)
      warp_runs += (double)c.n / 32.0;
    hc.push_back(b);
    hc_index.push_back(i);
  }
  // Block size: 512 threads (16 warps per SM) for a throughput batch -- only
  // tile/thread classes, all of dimension 8 or less, more than two waves of
  // warps (the dijet batch: 403 -> 360 ms) -- else 384 (12 warps, 170
  // registers a thread instead of 128: faster per run, which is what a
  // batch of long-running runs waits on; the multimodal batch 29.7 -> 26.1
  // ms, the mixed one 23.1 -> 21.9 ms).  config->block forces one.
  bool small_warp_only = true;
  for (const BatchClass& b : hc)
    small_warp_only &= (b.layout == ZEUS_LAYOUT_TILE || b.layout == ZEUS_LAYOUT_THREAD) &&
                       b.dim <= 8;
  int block = config->block == kBatchBlockLarge || config->block == kBatchBlockSmall
                ? config->block
                : (small_warp_only && warp_runs > 2.0 * sm_count() * (kBatchBlockLarge / 32)
                     ? kBatchBlockLarge
                     : kBatchBlockSmall);
  for (const BatchClass& b : hc)
    if (b.layout == ZEUS_LAYOUT_CTA &&
        cta_doubles_rt(b.kind, b.dim, block) * sizeof(double) > 227 * 1024)
      block = kBatchBlockSmall; // its CTA classes fit at 384 (checked above)
  // companion classes leave the batch table for their standalone kernel
  std::vector<BatchClass> companions;
  std::vector<int> companion_index;
  {
    std::vector<BatchClass> keep;
    for (size_t k = 0; k < hc.size(); ++k) {
      if (companion_class(classes[hc_index[k]].problem, hc[k].layout, block)) {
        companions.push_back(hc[k]);
        companion_index.push_back(hc_index[k]);
      } else {
        keep.push_back(hc[k]);
      }
    }
    hc.swap(keep);
  }
  size_t smem_cta = 0;
  for (const BatchClass& b : hc) {
    if (b.layout == ZEUS_LAYOUT_CTA)
      smem_cta = std::max(smem_cta, cta_doubles_rt(b.kind, b.dim, block));
    if (b.layout == ZEUS_LAYOUT_ROWS)
      smem_cta = std::max(smem_cta, rows_doubles_rt(b.dim, block));
  }
  // CTA classes first, smallest dimension (least work per run) first: a
  // batch lasts as long as its slowest run, and a class whose bulk finishes
  // early lets its stalled runs (those iterating to MAX_ITER) overlap the
  // bigger classes' bulk instead of starting after it (the mixed batch:
  // 44.0 ms largest-first, 40.0 ms smallest-first).  Row classes (all
  // light beside a companion 128-D class) largest dimension first: their
  // longest MAX_ITER runs, the 64-D ones (14.5 ms), then start at once (the
  // mixed batch 17.9 -> 17.2 / 18.1 ms in two runs: within its run-to-run
  // spread).  Then the tile/thread classes, largest dimension first.
  std::stable_sort(hc.begin(), hc.end(), [](const BatchClass& a, const BatchClass& b) {
    const int ka = a.layout == ZEUS_LAYOUT_CTA || a.layout == ZEUS_LAYOUT_ROWS;
    const int kb = b.layout == ZEUS_LAYOUT_CTA || b.layout == ZEUS_LAYOUT_ROWS;
    if (ka != kb)
      return ka > kb;
    if (a.layout == ZEUS_LAYOUT_ROWS && b.layout == ZEUS_LAYOUT_ROWS)
      return a.dim > b.dim;
    return ka ? a.dim < b.dim : a.dim > b.dim;
  });
  int rc = cuda_fail(cudaMemsetAsync(queues, 0,
                                     sizeof(unsigned long long) * n_classes, st),
                     "batch queue reset");
  if (rc)
    return rc;
  BatchTable bt{};
  bt.ncls = (int)hc.size();
  bt.max_iter = config->max_iter;
  bt.tol = config->tolerance;
  bt.flags = config->flags;
  // With CTA and tile/thread classes together, one block in kEarlyDiv
  // drains the tile/thread classes first (their bulk is small beside the
  // CTA classes', and what matters is that their longest runs start early)
  bool has_cta = false, has_warp = false;
  for (const BatchClass& b : hc) {
    const bool blockwide = b.layout == ZEUS_LAYOUT_CTA || b.layout == ZEUS_LAYOUT_ROWS;
    has_cta |= blockwide;
    has_warp |= !blockwide;
  }
  constexpr int kEarlyDiv = 16;
  bt.early_b = has_cta && has_warp ? std::max(1, sm_count() / kEarlyDiv) : 0;
  for (int i = 0; i < bt.ncls; ++i)
    bt.c[i] = hc[i];
  const size_t smem =
    sizeof(double) * std::max(smem_cta, smem_tile * (block / 32));
  const auto launch_batch = [&]() -> int {
    if (bt.ncls == 0)
      return ZEUS_OK;
    return block == kBatchBlockLarge ? launch_batch_512(bt, smem, st)
                                     : launch_batch_384(bt, smem, st);
  };
  if (companions.empty())
    return launch_batch();
  // the batch kernel first (its blocks take the SMs), then the companions
  // on the side stream, joined back into `st`
  SideStream* side = nullptr;
  if ((rc = side_stream(&side)) ||
      (rc = cuda_fail(cudaEventRecord(side->fork, st), "batch fork")) ||
      (rc = launch_batch()) ||
      (rc = cuda_fail(cudaStreamWaitEvent(side->st, side->fork, 0), "batch fork wait")))
    return rc;
  zeus_bfgs_config rows_cfg = *config;
  rows_cfg.layout = ZEUS_LAYOUT_ROWS;
  rows_cfg.tile = 0;
  for (size_t k = 0; k < companions.size(); ++k) {
    const BatchClass& b = companions[k];
    if (b.n <= 0)
      continue;
    const zeus_problem& p = classes[companion_index[k]].problem;
    const Objective o{p.kind, p.dim, p.data, p.idata, p.ndata, p.flags, nullptr};
    const BfgsParams prm{b.n, config->max_iter, b.required, config->tolerance,
                         config->flags};
    if ((rc = launch_rows(o, rows_cfg, prm, b.starts, b.out, b.ctl,
                          companion_ws + (size_t)companion_index[k] * kCompanionQueueBytes,
                          kCompanionQueueBytes, side->st)))
      break;
  }
  // join even after a failed launch, so that `st` is left consistent
  const int jrc = cuda_fail(cudaEventRecord(side->join, side->st), "batch join");
  const int wrc = cuda_fail(cudaStreamWaitEvent(st, side->join, 0), "batch join wait");
  return rc ? rc : jrc ? jrc : wrc;
}

} // extern "C"
