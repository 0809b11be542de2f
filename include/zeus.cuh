// zeus.cuh -- C++ drop-in for the reference's public API on B200 (sm_100a).
//
//   #include "zeus.cuh"       (nvcc -std=c++20 --expt-relaxed-constexpr
//                              -I include -I zeus_b200/csrc, link
//                              zeus_b200/libzeus_b200.so)
//   auto r = zeus::Zeus(f, lower, upper, N, MAX_ITER, PSO_ITER,
//                       requiredConverged, "name", tol, seed, run);
//
// Keeps the reference's call surface (include/zeus.cuh:341-375): the
// callable f is any functor with `template <class T> __host__ __device__ T
// operator()(std::array<T, D> const&) const`, its dimension D comes from
// zeus::FnTraits (static `arity`, or a Functor<D> template), it is validated
// by the ZeusObjective concept, objective data lives in Matrix<T> members
// read through .data(), and the result is zeus::Result<D> with the
// reference's field names and status codes (util.hpp:16-54).
//
// The kernels that evaluate f are templates instantiated here, in the
// caller's translation unit, from the library's own headers (PSO:
// zb_pso.cuh; BFGS layouts: zb_bfgs_thread.cuh / zb_bfgs_coop.cuh); the
// objective-independent work (argmin and status census) goes through the
// C ABI in zeus_b200.h.  Gradients are D forward dual passes unless the
// functor also has `double adjoint(const double* x, double* g) const`
// (hand-written gradient), which is then used.  Layout by dimension:
// thread-per-run (D <= 8), 32-lane tile (D <= 32), block-per-run with H in
// shared memory (up to D = 160).
#pragma once

#include <array>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <string_view>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

#include "zeus_b200.h"
#include "duals.cuh"
#include "matrix.hpp"
#include "traits.hpp"
#include "zb_bfgs_coop.cuh"
#include "zb_bfgs_exact.cuh"
#include "zb_bfgs_thread.cuh"
#include "zb_dual.cuh"
#include "zb_pso.cuh"

namespace zeus {

  // ---- results (util.hpp:16-54) -------------------------------------------
  struct Metrics {
    const char* label = "";
    double ms_per_call = 0.0;
    double calls_per_thread_mean = 0.0;
    double fraction_of_kernel = 0.0;
    double block95 = 0.0;
    double serialized = 0.0;
    double fraction_of_thread = 0.0;
  };
  struct Convergence {
    int actual = 0;
    int claimed = 0;
    int surrendered = 0;
    int stopped = 0;
  };
  template <std::size_t DIM>
  struct Result {
    int idx = -1;
    int status = -1; // 0 surrender, 1 converged, 2 stopped, 3 alloc, 4 CUDA, 5 non-finite
    double fval = 37.0;
    double gradientNorm = 0.0;
    double coordinates[DIM]{};
    int iter = 0;
    Convergence c;
    double ms_opt = 0.0;
    Metrics ad;
    Metrics bfgs;
  };

} // namespace zeus

namespace util {

  // The reference's util::setStackSize (src/utils.cu:52-99) raises the
  // device stack and malloc-heap limits its kernels need for heap-resident
  // Hessians.  Nothing here uses the device heap or deep stacks (H lives in
  // registers, shared memory or a workspace slice), so it changes no limit;
  // it is kept so that code written for the reference, which calls it
  // before zeus::Zeus, compiles and runs unchanged.
  inline void
  setStackSize()
  {}

} // namespace util

namespace zeus {

  namespace detail {

    // A call's device buffers and its own stream (the legacy stream cannot
    // be captured into a graph; it is used only if no stream can be made).
    struct DeviceBuffers {
      std::vector<void*> p;
      cudaStream_t st = nullptr;
      bool own = false;
      DeviceBuffers()
      {
        own = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
        if (!own) {
          cudaGetLastError();
          st = nullptr;
        }
      }
      ~DeviceBuffers()
      {
        for (void* q : p)
          cudaFreeAsync(q, st);
        cudaStreamSynchronize(st);
        if (own)
          cudaStreamDestroy(st);
      }
      DeviceBuffers(const DeviceBuffers&) = delete;
      DeviceBuffers& operator=(const DeviceBuffers&) = delete;
      template <class T>
      T*
      alloc(std::size_t n)
      {
        void* q = nullptr;
        const cudaError_t e = cudaMallocAsync(&q, n ? n * sizeof(T) : 1, st);
        if (e != cudaSuccess)
          throw e;
        p.push_back(q);
        return static_cast<T*>(q);
      }
    };

    // The PSO (the reference's zeus.cuh:64-92 with pso.cuh's kernels): a
    // thread per particle for D <= 32, a warp per particle above (its lanes
    // move the D coordinates of one particle, coalesced; the same random
    // counters and update expressions, so the same swarm).  The iterations
    // are captured into one CUDA graph and launched once.
    template <class Function, std::size_t D>
    cudaError_t
    run_pso(const Function& f, int64_t n, double lower, double upper, int iters,
            uint64_t seed, const zb::PsoWork& w, double* starts, double* pbf,
            cudaStream_t st, cudaEvent_t after_init)
    {
      const unsigned blocks = (unsigned)zb::pso_blocks(n, (int)D);
      constexpr bool coop = (int)D >= zb::kPsoCoopMinDim;
      zb::pso_reset_kernel<(int)D><<<1, 256, 0, st>>>(w);
      if constexpr (coop)
        zb::pso_init_coop_kernel<Function, (int)D>
          <<<blocks, zb::kPsoBlock, 0, st>>>(f, n, lower, upper, seed, w, starts, pbf);
      else
        zb::pso_init_kernel<Function, (int)D>
          <<<blocks, zb::kPsoBlock, 0, st>>>(f, n, lower, upper, seed, w, starts, pbf);
      cudaError_t e = cudaGetLastError();
      cudaEventRecord(after_init, st);
      if (e != cudaSuccess || iters <= 0)
        return e;
      const auto iterations = [&] {
        for (int t = 1; t <= iters; ++t) {
          if constexpr (coop)
            zb::pso_iter_coop_kernel<Function, (int)D><<<blocks, zb::kPsoBlock, 0, st>>>(
              f, n, 0.5, 1.2, 1.5, seed, t, w, starts, pbf);
          else
            zb::pso_iter_kernel<Function, (int)D><<<blocks, zb::kPsoBlock, 0, st>>>(
              f, n, 0.5, 1.2, 1.5, seed, t, w, starts, pbf);
        }
      };
      if (!st) {
        iterations();
        return cudaGetLastError();
      }
      if ((e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return e;
      iterations();
      cudaGraph_t g = nullptr;
      cudaGraphExec_t ge = nullptr;
      e = cudaStreamEndCapture(st, &g);
      if (e == cudaSuccess)
        e = cudaGraphInstantiate(&ge, g, 0);
      if (e == cudaSuccess)
        e = cudaGraphLaunch(ge, st);
      if (ge)
        cudaGraphExecDestroy(ge); // freed once the launch completes
      if (g)
        cudaGraphDestroy(g);
      return e;
    }

    // The reference's per-timer report lines (bfgs_sequential.cuh:345-360),
    // from zeus_cycle_metrics' values.
    inline void
    print_metrics(const char* label, float ms_opt, const double m[8])
    {
      std::printf("[%s] Kernel wall time: %.3f ms\n", label, ms_opt);
      std::printf("[%s] Avg cycles/thread: %.3f ; avg ms/thread: %.6f\n", label, m[6],
                  m[7]);
      std::printf("[%s] Calls/thread \u2248 %.2f; ms/call \u2248 %.6f\n", label, m[1],
                  m[0]);
      std::printf("[%s] Heuristic fraction: %.3f%%\n", label, 100.0 * m[5]);
      std::printf("[%s] Serialized sum: %.3f ms; fraction vs kernel: %.3f%%\n", label,
                  m[4] * ms_opt, 100.0 * m[4]);
      std::printf("[%s] Block-level fraction p95: %.3f%%\n", label, 100.0 * m[3]);
    }

    // hws: for the CTA layout past about D = 160, a device buffer of
    // cta_h_slices(n) * D * D doubles holding each block's H
    inline int64_t
    cta_h_slices(int64_t n)
    {
      int dev = 0, sms = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      return n < 2 * (int64_t)sms ? n : 2 * (int64_t)sms;
    }

    template <class F, std::size_t D>
    cudaError_t
    launch_bfgs(const F& f, const zb::BfgsParams& prm, const double* starts,
                const zb::RunOut& out, zb::Control* ctl, cudaStream_t st,
                double* hws = nullptr, unsigned long long* queue = nullptr)
    {
      constexpr bool kAdj = zb::HasAdjoint<F>;
      if constexpr (D <= 8) {
        const unsigned grid = (unsigned)((prm.n + 127) / 128);
        zb::bfgs_thread_kernel<F, (int)D, kAdj, true>
          <<<grid, 128, 0, st>>>(f, prm, starts, out, ctl);
      } else if constexpr (D <= 32) {
        constexpr int TS = 32, TPB = zb::kTileBlock / TS;
        const unsigned grid = (unsigned)((prm.n + TPB - 1) / TPB);
        const size_t smem =
          sizeof(double) * TPB * zb::tile_smem_doubles<(int)D, TS>();
        zb::bfgs_tile_kernel<F, (int)D, TS, kAdj, true>
          <<<grid, zb::kTileBlock, smem, st>>>(f, prm, starts, out, ctl);
      } else {
        static_assert(D <= 1024, "dimensions above 1024 are not supported");
        constexpr int B = D <= 64 ? 256 : 512;
        const size_t smem =
          sizeof(double) * zb::cta_smem_doubles<F, (int)D, kAdj>(B);
        auto k = zb::bfgs_cta_kernel<F, (int)D, kAdj, B, true>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, B, smem);
        int64_t cap = (int64_t)sms * (per_sm > 0 ? per_sm : 1);
        if constexpr (zb::cta_h_global((int)D, B)) {
          const int64_t slices = cta_h_slices(prm.n);
          cap = cap < slices ? cap : slices;
        }
        if (queue)
          cudaMemsetAsync(queue, 0, sizeof *queue, st);
        k<<<(unsigned)(prm.n < cap ? prm.n : cap), B, smem, st>>>(f, prm, starts,
                                                                  out, ctl, hws, queue);
      }
      return cudaGetLastError();
    }

  } // namespace detail

  // The reference's entry point (include/zeus.cuh:341-375).  prng_type
  // picks the start positions' generator: Philox4x32-10 for XORWOW and
  // PHILOX, a digitally shifted Sobol' sequence for SOBOL (starts, or the
  // PSO's initial swarm; velocities and r1/r2 stay on Philox).  parallel and
  // nzerosteps are accepted for source compatibility: the layout follows the
  // dimension, and the zero-step limit cannot trigger (the reference's line
  // search never returns 0, utils.cuh:395-411).  With a trajectory_file (.tsv) the BFGS
  // runs in exact mode, one run per block in the reference's operation
  // order, recording every iteration (N * MAX_ITER steps, as the reference
  // allocates them), and the file is written in the reference's layout
  // (zeus.cuh:62-103, 189-239; src/utils.cu:128-176); a file that cannot be
  // written is reported on stderr and the result is still returned, as the
  // reference does.  Like the reference, every call with N > 0 appends its
  // row to zeus_<D>d_results.tsv in the working directory and prints the
  // census line.
  template <typename Function, std::size_t ZEUS_DIM = FnTraits<Function>::arity>
    requires ZeusObjective<Function, ZEUS_DIM>
  Result<ZEUS_DIM>
  Zeus(Function const& f, double lower, double upper, std::size_t N,
       int MAX_ITER, int PSO_ITER, int requiredConverged,
       std::string_view fun_name, double tolerance, int seed, int run,
       bool parallel = true, PRNGType prng_type = PRNGType::XORWOW,
       std::string_view trajectory_file = {}, int nzerosteps = 0)
  {
    (void)parallel;
    (void)nzerosteps;
    const int32_t prng = prng_type == PRNGType::SOBOL    ? ZEUS_PRNG_SOBOL
                         : prng_type == PRNGType::PHILOX ? ZEUS_PRNG_PHILOX
                                                         : ZEUS_PRNG_XORWOW;
    constexpr std::size_t D = ZEUS_DIM;
    Result<D> best;
    if (N == 0)
      return best; // zeus.cuh:58-60
    detail::DeviceBuffers b;
    cudaEvent_t e0, e1, p0, p1, p2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&p0);
    cudaEventCreate(&p1);
    cudaEventCreate(&p2);
    try {
      const int64_t n = (int64_t)N;
      double* starts = b.alloc<double>(N * D);
      double* fval = b.alloc<double>(N);
      int32_t* status = b.alloc<int32_t>(N);
      int32_t* iter = b.alloc<int32_t>(N);
      double* gnorm = b.alloc<double>(N);
      double* x = b.alloc<double>(N * D);
      int32_t* ctl = b.alloc<int32_t>(2);
      zeus_census* cen = b.alloc<zeus_census>(1);
      cudaMemsetAsync(ctl, 0, 2 * sizeof(int32_t), b.st);
      if (PSO_ITER >= 0) {
        const int64_t blocks = zb::pso_blocks(n, (int)D);
        zb::PsoWork w;
        w.X = b.alloc<double>(N * D);
        w.V = b.alloc<double>(N * D);
        w.part_key = b.alloc<unsigned long long>(blocks);
        w.part_idx = b.alloc<int>(blocks);
        w.counter = b.alloc<unsigned int>(1);
        w.gbest = b.alloc<double>(D + 1);
        if (prng == ZEUS_PRNG_SOBOL &&
            zeus_sobol_device_table(&w.sobol) != ZEUS_OK)
          throw cudaErrorLaunchFailure;
        double* pbf = b.alloc<double>(N);
        cudaEventRecord(p0, b.st);
        const cudaError_t pe = detail::run_pso<Function, D>(
          f, n, lower, upper, PSO_ITER, (uint64_t)seed, w, starts, pbf, b.st, p1);
        if (pe != cudaSuccess)
          throw pe;
        cudaEventRecord(p2, b.st);
      } else if (zeus_starts((uint64_t)seed, prng, n, (int32_t)D, lower, upper,
                             starts, b.st) != ZEUS_OK) {
        throw cudaErrorLaunchFailure;
      }
      zb::BfgsParams prm{n, MAX_ITER, requiredConverged, tolerance, 0};
      // per-run counters and the AD / BFGS / total cycle timers of the
      // reference's metrics (bfgs_sequential.cuh:447-470)
      int64_t* counters = b.alloc<int64_t>(N * 3);
      int64_t* cycles = b.alloc<int64_t>(N * 3);
      zb::RunOut out{fval,   status,  iter,    gnorm,   x,
                     counters, nullptr, nullptr, nullptr, nullptr, cycles};
      const bool traj = !trajectory_file.empty() && MAX_ITER > 0;
      const size_t steps = traj ? (size_t)N * (size_t)MAX_ITER : 0;
      if (traj) {
        out.traj_x = b.alloc<double>(steps * D);
        out.traj_f = b.alloc<double>(steps);
        out.traj_g = b.alloc<double>(steps);
        out.traj_status = b.alloc<int8_t>(steps);
        // all-ones bytes: NaN doubles and status -1 (the reference's fill)
        cudaMemsetAsync(out.traj_x, 0xff, steps * D * sizeof(double), b.st);
        cudaMemsetAsync(out.traj_f, 0xff, steps * sizeof(double), b.st);
        cudaMemsetAsync(out.traj_g, 0xff, steps * sizeof(double), b.st);
        cudaMemsetAsync(out.traj_status, 0xff, steps, b.st);
      }
      cudaEventRecord(e0, b.st);
      cudaError_t e;
      if (traj) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int64_t grid = n < (int64_t)sms * 4 ? n : (int64_t)sms * 4;
        double* scratch = b.alloc<double>((size_t)grid * 2 * D * D);
        zb::bfgs_exact_kernel<Function, (int)D, true>
          <<<(unsigned)grid, 128, zb::exact_smem_bytes<(int)D>(), b.st>>>(
            f, prm, starts, out, reinterpret_cast<zb::Control*>(ctl), scratch);
        e = cudaGetLastError();
      } else {
        double* hws = nullptr;
        unsigned long long* queue = nullptr;
        if constexpr (D > 32) {
          queue = b.alloc<unsigned long long>(1); // the blocks' run queue
          if constexpr (zb::cta_h_global((int)D, D <= 64 ? 256 : 512))
            hws = b.alloc<double>((size_t)detail::cta_h_slices(n) * D * D);
        }
        e = detail::launch_bfgs<Function, D>(
          f, prm, starts, out, reinterpret_cast<zb::Control*>(ctl), b.st, hws, queue);
      }
      cudaEventRecord(e1, b.st);
      if (e != cudaSuccess)
        throw e;
      if (traj) {
        std::vector<double> hx(steps * D), hf(steps), hg(steps);
        std::vector<int8_t> hs(steps);
        cudaMemcpyAsync(hx.data(), out.traj_x, hx.size() * sizeof(double),
                        cudaMemcpyDeviceToHost, b.st);
        cudaMemcpyAsync(hf.data(), out.traj_f, hf.size() * sizeof(double),
                        cudaMemcpyDeviceToHost, b.st);
        cudaMemcpyAsync(hg.data(), out.traj_g, hg.size() * sizeof(double),
                        cudaMemcpyDeviceToHost, b.st);
        cudaMemcpyAsync(hs.data(), out.traj_status, hs.size(),
                        cudaMemcpyDeviceToHost, b.st);
        if ((e = cudaStreamSynchronize(b.st)) != cudaSuccess)
          throw e;
        const std::string path(trajectory_file);
        if (zeus_write_trajectory_tsv(path.c_str(), hx.data(), hf.data(), hg.data(),
                                      hs.data(), nullptr, n, MAX_ITER,
                                      (int32_t)D) != ZEUS_OK)
          std::fprintf(stderr, "Error: %s\n", zeus_last_error());
      }
      std::vector<double> km;
      if (fun_name == "rosenbrock")
        km.assign(D, 1.0);
      if (zeus_census_device(fval, status, x, n, (int32_t)D,
                             km.empty() ? nullptr : km.data(), cen, b.st) != ZEUS_OK)
        throw cudaErrorLaunchFailure;
      zeus_census hc{};
      cudaMemcpyAsync(&hc, cen, sizeof hc, cudaMemcpyDeviceToHost, b.st);
      if ((e = cudaStreamSynchronize(b.st)) != cudaSuccess)
        throw e;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      best.ms_opt = ms;
      double met[2][8] = {};
      {
        std::vector<int64_t> hcy((size_t)N * 3), hct((size_t)N * 3);
        cudaMemcpy(hcy.data(), cycles, hcy.size() * sizeof(int64_t),
                   cudaMemcpyDeviceToHost);
        cudaMemcpy(hct.data(), counters, hct.size() * sizeof(int64_t),
                   cudaMemcpyDeviceToHost);
        int dev = 0, khz = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev);
        const char* label[2] = {"AD", "BFGS"};
        Metrics* dst[2] = {&best.ad, &best.bfgs};
        for (int w = 0; w < 2; ++w) {
          if (zeus_cycle_metrics(hcy.data(), hct.data(), n, w, (double)khz, ms,
                                 128, met[w]) != ZEUS_OK)
            continue;
          detail::print_metrics(label[w], ms, met[w]);
          *dst[w] = Metrics{label[w], met[w][0], met[w][1], met[w][5],
                            met[w][3], met[w][4], met[w][2]};
        }
      }
      best.c = Convergence{hc.actual, hc.claimed, hc.surrendered, hc.stopped};
      if (hc.best_idx >= 0) {
        const int i = hc.best_idx;
        cudaMemcpy(&best.fval, fval + i, sizeof(double), cudaMemcpyDeviceToHost);
        cudaMemcpy(&best.status, status + i, sizeof(int), cudaMemcpyDeviceToHost);
        cudaMemcpy(&best.iter, iter + i, sizeof(int), cudaMemcpyDeviceToHost);
        cudaMemcpy(&best.gradientNorm, gnorm + i, sizeof(double),
                   cudaMemcpyDeviceToHost);
        cudaMemcpy(best.coordinates, x + (size_t)i * D, sizeof(double) * D,
                   cudaMemcpyDeviceToHost);
        best.idx = i;
      }
      // the reference's per-call results row and census line
      // (zeus.cuh:170-183, util.hpp:79-136)
      float ms_init = 0.f, ms_pso = 0.f;
      if (PSO_ITER >= 0) {
        cudaEventElapsedTime(&ms_init, p0, p1);
        cudaEventElapsedTime(&ms_pso, p1, p2);
      }
      const std::string fn(fun_name);
      const double err = zeus_euclidean_error(fn.c_str(), best.coordinates, (int32_t)D);
      const zeus_result zr{best.idx, best.status, best.fval, best.gradientNorm,
                           best.iter, 0};
      const zeus_census zc{hc.actual, hc.claimed, hc.surrendered, hc.stopped,
                           hc.best_idx, 0};
      const double tsv_metrics[10] = {met[0][0], met[0][1], met[0][2], met[0][3],
                                      met[0][4], met[1][0], met[1][1], met[1][2],
                                      met[1][3], met[1][4]};
      if (zeus_append_results_tsv(nullptr, fn.c_str(), run, n, (int32_t)D, ms_init,
                                  ms_pso, ms, 0.f, MAX_ITER, PSO_ITER, err, &zr, &zc,
                                  best.coordinates, tsv_metrics) != ZEUS_OK)
        std::fprintf(stderr, "Error: %s\n", zeus_last_error());
      std::printf("claimed: %d\tactual : %d\tsurrendered: %d\tstopped: %d\n",
                  hc.claimed, hc.actual, hc.surrendered, hc.stopped);
    } catch (cudaError_t e) { // zeus.cuh:112-116: 3 allocation, 4 runtime
      best = Result<D>{};
      best.status = (e == cudaErrorMemoryAllocation) ? 3 : 4;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(p0);
    cudaEventDestroy(p1);
    cudaEventDestroy(p2);
    return best;
  }

} // namespace zeus
