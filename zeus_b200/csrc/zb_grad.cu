// f and grad f at given points through each gradient path the BFGS layouts
// step on (zeus_gradient_device):
//   thread    one thread per point: the objective's adjoint(), or the D
//             forward dual passes of the plain form (fast_gradient);
//   tile      a tile of TS lanes per point: coop_gradient (adjoint_coop, the
//             value with the gradient) or coop_gradient_only (gradient_coop
//             where the objective has one) -- what tile_run calls;
//   cta       a block per point, the same two forms on a CtaGroup -- what
//             cta_run and the persistent batch call (the dual form is the
//             CTA plain form's per-member passes);
//   quadratic the CTA line search of a symmetric quadratic form: from one
//             ctx2_coop pass over C at (x, p), the carried value
//             f(x) + a g.p + a^2 f(p) and gradient C x + a C p at x + a p.
// The kernels call the same device functions as the BFGS kernels, so a
// point checked here checks the gradient those kernels use.
#include <cmath>

#include "zb_bfgs_coop.cuh"
#include "zb_objective_visit.cuh"

namespace zb {

  namespace {

    constexpr int kGradThreadBlock = 128;

    __device__ __forceinline__ double
    nan_value()
    {
      return __longlong_as_double(0x7ff8000000000000ll);
    }

    template <class F, int D, bool Adjoint>
    __global__ void __launch_bounds__(kGradThreadBlock)
      grad_thread_kernel(F f, const double* __restrict__ x, int64_t n,
                         double* __restrict__ fo, double* __restrict__ go)
    {
      const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
      if (i >= n)
        return;
      double xl[D], gl[D];
#pragma unroll
      for (int d = 0; d < D; ++d)
        xl[d] = x[i * D + d];
      double v;
      if constexpr (Adjoint) {
        v = f.adjoint(xl, gl);
      } else {
        fast_gradient<F, D, false>(f, xl, gl);
        v = fast_value<F, D>(f, xl);
      }
      fo[i] = v;
#pragma unroll
      for (int d = 0; d < D; ++d)
        go[i * D + d] = gl[d];
    }

    // per tile: x[D] | g[D] | scratch[TS]
    template <int D, int TS>
    __host__ __device__ constexpr int
    grad_tile_doubles()
    {
      return ((2 * D + TS) + 1) & ~1;
    }

    template <class F, int D, int TS, bool Adjoint, bool GradOnly>
    __global__ void __launch_bounds__(kTileBlock)
      grad_tile_kernel(F f, const double* __restrict__ x, int64_t n,
                       double* __restrict__ fo, double* __restrict__ go)
    {
      constexpr int TPB = kTileBlock / TS;
      extern __shared__ __align__(16) double sm[];
      auto tile = cg::tiled_partition<TS>(cg::this_thread_block());
      const int tslot = threadIdx.x / TS;
      const int64_t i = (int64_t)blockIdx.x * TPB + tslot;
      if (i >= n)
        return; // the whole tile leaves together
      double* xs = sm + tslot * grad_tile_doubles<D, TS>();
      double* gs = xs + D;
      TileGroup<TS> grp(tile, gs + D);
      for (int d = grp.rank(); d < D; d += TS)
        xs[d] = x[i * D + d];
      grp.sync();
      double v = nan_value();
      if constexpr (GradOnly) {
        coop_gradient_only<F, D, Adjoint>(f, grp, xs, gs);
        v = coop_value<F, D>(f, grp, xs);
      } else {
        v = coop_gradient<F, D, Adjoint>(f, grp, xs, gs);
        if constexpr (!Adjoint)
          v = coop_value<F, D>(f, grp, xs);
      }
      grp.sync();
      if (grp.rank() == 0)
        fo[i] = v;
      for (int d = grp.rank(); d < D; d += TS)
        go[i * D + d] = gs[d];
    }

    // x[D] | g[D] | reductions | scratch[blockDim] (D rounded up to even so
    // the later arrays stay 16-byte aligned)
    __host__ __device__ constexpr size_t
    grad_cta_doubles(int d, int block)
    {
      const size_t de = (size_t)((d + 1) & ~1);
      return 2 * de + kCtaRedDoubles + (size_t)block;
    }

    // blocks of up to 512 threads, the widest the BFGS kernels launch
    constexpr int kGradMaxBlock = 512;

    template <class F, int D, bool Adjoint, bool GradOnly>
    __global__ void __launch_bounds__(kGradMaxBlock)
    grad_cta_kernel(F f, const double* __restrict__ x, double* __restrict__ fo,
                    double* __restrict__ go)
    {
      extern __shared__ __align__(16) double sm[];
      constexpr int DE = (D + 1) & ~1;
      double* xs = sm;
      double* gs = xs + DE;
      double* red = gs + DE;
      CtaGroup grp{red, red + kCtaRedDoubles};
      const int64_t i = blockIdx.x;
      for (int d = threadIdx.x; d < D; d += blockDim.x)
        xs[d] = x[i * D + d];
      __syncthreads();
      double v = nan_value();
      if constexpr (GradOnly) {
        coop_gradient_only<F, D, Adjoint>(f, grp, xs, gs);
        v = coop_value<F, D>(f, grp, xs);
      } else {
        v = coop_gradient<F, D, Adjoint>(f, grp, xs, gs);
        if constexpr (!Adjoint) {
          __syncthreads();
          v = coop_value<F, D>(f, grp, xs);
        }
      }
      __syncthreads();
      if (threadIdx.x == 0)
        fo[i] = v;
      for (int d = threadIdx.x; d < D; d += blockDim.x)
        go[i * D + d] = gs[d];
    }

    // partial-sum arrays of ctx2_coop: the even-D pair form writes
    // (block / (D/2)) * D doubles each, the column form at most block
    __host__ __device__ constexpr size_t
    quad_part_doubles(int d, int block)
    {
      const size_t pair = d % 2 == 0 && block >= d / 2
                            ? (size_t)(block / (d / 2)) * d
                            : 0;
      const size_t col = (size_t)block;
      return ((pair > col ? pair : col) + 1) & ~(size_t)1;
    }
    // x[D] | p[D] | C^T x [D] | C^T p [D] | reductions | sx | sp
    __host__ __device__ constexpr size_t
    grad_quad_doubles(int d, int block)
    {
      const size_t de = (size_t)((d + 1) & ~1);
      return 4 * de + kCtaRedDoubles + 2 * quad_part_doubles(d, block);
    }

    template <class F, int D>
    __global__ void __launch_bounds__(kGradMaxBlock)
    grad_quad_kernel(F f, const double* __restrict__ x,
                     const double* __restrict__ p, double alpha,
                     double* __restrict__ fo, double* __restrict__ go)
    {
      extern __shared__ __align__(16) double sm[];
      constexpr int DE = (D + 1) & ~1;
      double* xs = sm;
      double* ps = xs + DE;
      double* rx = ps + DE;
      double* rp = rx + DE;
      double* red = rp + DE;
      double* sx = red + kCtaRedDoubles;
      double* sp = sx + quad_part_doubles(D, blockDim.x);
      CtaGroup grp{red, sx};
      const int64_t i = blockIdx.x;
      const int t = threadIdx.x;
      for (int d = t; d < D; d += blockDim.x) {
        xs[d] = x[i * D + d];
        ps[d] = p[i * D + d];
      }
      __syncthreads();
      // the CTA line search's arithmetic (cta_run, symmetric quadratic form)
      f.ctx2_coop(grp, xs, ps, rx, rp, sx, sp);
      double v3[3] = {0.0, 0.0, 0.0};
      if (t < D) { // blockDim.x >= D: one term per thread, as cta_run forms them
        v3[0] = xs[t] * rx[t];
        v3[1] = ps[t] * rp[t];
        v3[2] = rx[t] * ps[t];
      }
      grp.template sum<3>(v3);
      const double f0 = 0.5 * v3[0], fp = 0.5 * v3[1], gp = v3[2];
      if (t == 0)
        fo[i] = f0 + alpha * fma(alpha, fp, gp);
      for (int d = t; d < D; d += blockDim.x)
        go[i * D + d] = fma(alpha, rp[d], rx[d]);
    }

    template <class K>
    int
    set_smem(K kern, size_t bytes)
    {
      if (bytes <= 48 * 1024)
        return ZEUS_OK;
      return cuda_fail(cudaFuncSetAttribute(
                         kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)bytes),
                       "gradient kernel shared memory attribute");
    }

    template <class F, int D, int TS, bool Adjoint, bool GradOnly>
    int
    launch_tile_grad(const F& f, const double* x, int64_t n, double* fo,
                     double* go, cudaStream_t st)
    {
      constexpr int TPB = kTileBlock / TS;
      const unsigned grid = (unsigned)((n + TPB - 1) / TPB);
      const size_t smem = sizeof(double) * TPB * grad_tile_doubles<D, TS>();
      auto kern = grad_tile_kernel<F, D, TS, Adjoint, GradOnly>;
      if (int rc = set_smem(kern, smem))
        return rc;
      kern<<<grid, kTileBlock, smem, st>>>(f, x, n, fo, go);
      return cuda_fail(cudaGetLastError(), "tile gradient launch");
    }

  } // namespace

  int
  launch_gradient(const Objective& o, int path, int gradient, int width,
                  const double* x, const double* p, double alpha, int64_t n,
                  double* fo, double* go, cudaStream_t st)
  {
    const bool adj = gradient == ZEUS_GRAD_ADJOINT;
    return visit_objective(o, [&](auto f) -> int {
      using F = decltype(f);
      constexpr int D = (int)F::arity;
      switch (path) {
        case ZEUS_GRADPATH_THREAD: {
          if constexpr (D <= 32) {
            const unsigned grid =
              (unsigned)((n + kGradThreadBlock - 1) / kGradThreadBlock);
            if (adj)
              grad_thread_kernel<F, D, true>
                <<<grid, kGradThreadBlock, 0, st>>>(f, x, n, fo, go);
            else
              grad_thread_kernel<F, D, false>
                <<<grid, kGradThreadBlock, 0, st>>>(f, x, n, fo, go);
            return cuda_fail(cudaGetLastError(), "thread gradient launch");
          }
          set_error("thread gradient path: dim %d > 32 is not built", D);
          return ZEUS_E_UNSUPPORTED;
        }
        case ZEUS_GRADPATH_TILE:
        case ZEUS_GRADPATH_TILE_GRAD: {
          constexpr unsigned W = tile_widths_for(F::kind, D);
          const bool gonly = path == ZEUS_GRADPATH_TILE_GRAD;
          if (gonly && !adj) {
            set_error("the gradient-only tile form is the adjoint's");
            return ZEUS_E_INVALID;
          }
          switch (width) {
#define ZB_TS(K)                                                               \
  case (1 << K):                                                               \
    if constexpr ((W >> K) & 1u) {                                             \
      if (gonly)                                                               \
        return launch_tile_grad<F, D, (1 << K), true, true>(f, x, n, fo, go,   \
                                                            st);               \
      if (adj)                                                                 \
        return launch_tile_grad<F, D, (1 << K), true, false>(f, x, n, fo, go,  \
                                                             st);              \
      return launch_tile_grad<F, D, (1 << K), false, false>(f, x, n, fo, go,   \
                                                            st);               \
    }                                                                          \
    break;
            ZB_TS(1)
            ZB_TS(2)
            ZB_TS(3)
            ZB_TS(4)
            ZB_TS(5)
#undef ZB_TS
          }
          set_error("tile gradient path: width %d not built for dim %d", width,
                    D);
          return ZEUS_E_UNSUPPORTED;
        }
        case ZEUS_GRADPATH_CTA:
        case ZEUS_GRADPATH_CTA_GRAD: {
          const bool gonly = path == ZEUS_GRADPATH_CTA_GRAD;
          if (gonly && !adj) {
            set_error("the gradient-only CTA form is the adjoint's");
            return ZEUS_E_INVALID;
          }
          const size_t smem = sizeof(double) * grad_cta_doubles(D, width);
          auto launch = [&](auto kern) -> int {
            if (int rc = set_smem(kern, smem))
              return rc;
            kern<<<(unsigned)n, width, smem, st>>>(f, x, fo, go);
            return cuda_fail(cudaGetLastError(), "CTA gradient launch");
          };
          if (gonly)
            return launch(grad_cta_kernel<F, D, true, true>);
          if (adj)
            return launch(grad_cta_kernel<F, D, true, false>);
          return launch(grad_cta_kernel<F, D, false, false>);
        }
        case ZEUS_GRADPATH_QUADRATIC: {
          if constexpr (QuadraticForm<F>) {
            if (!f.symmetric) {
              set_error("quadratic gradient path: C must be symmetric");
              return ZEUS_E_INVALID;
            }
            if (!adj) {
              set_error("the quadratic path carries the adjoint's gradient");
              return ZEUS_E_INVALID;
            }
            const size_t smem = sizeof(double) * grad_quad_doubles(D, width);
            auto kern = grad_quad_kernel<F, D>;
            if (int rc = set_smem(kern, smem))
              return rc;
            kern<<<(unsigned)n, width, smem, st>>>(f, x, p, alpha, fo, go);
            return cuda_fail(cudaGetLastError(), "quadratic gradient launch");
          }
          set_error("quadratic gradient path: objective %d is not a quadratic "
                    "form",
                    F::kind);
          return ZEUS_E_UNSUPPORTED;
        }
      }
      set_error("unknown gradient path %d", path);
      return ZEUS_E_INVALID;
    });
  }

} // namespace zb
