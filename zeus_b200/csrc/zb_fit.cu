// Implicit-function adjoint of a binned Poisson fit: d(argmin)/d(counts).
//
// No counterpart in the reference (its fit example stops at the minimum,
// examples/fit_dijet_spectrum.cu:162-221).  At the fitted parameters p of a
// toy, grad_p NLL = sum_i (lambda_i - k_i) J_i = 0 with
// J_i = d ln lambda_i / dp = (1/a, ln(1-x_i), -ln x_i, -(ln x_i)^2); the
// implicit function theorem on k_j gives
//     dp/dk_j = H^-1 J_j,
//     H = sum_i lambda_i J_i J_i^T - (sum_i (lambda_i - k_i)) / a^2 e_a e_a^T
// (the exact Hessian of the NLL; the second term vanishes at an exact
// minimum).  One warp per toy: pick the toy's best run (lowest fval, lowest
// index on ties, as the census does), accumulate H over the bins in lanes,
// factor it (4x4 Cholesky), and solve for every bin.
#include "zb_internal.h"

namespace zb {

  namespace {

    __device__ __forceinline__ double
    warp_sum(double v)
    {
#pragma unroll
      for (int m = 16; m > 0; m >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, m);
      return v;
    }

    // d p / d k for every bin of every toy; best[toy] = {fval, p0..p3, run}
    __global__ void __launch_bounds__(128)
      nll_sensitivity_kernel(const double* __restrict__ centres,
                             const int* __restrict__ counts, int nbins,
                             int64_t ntoys, int64_t per_toy,
                             const double* __restrict__ fval,
                             const double* __restrict__ x,
                             double* __restrict__ best,
                             double* __restrict__ sens)
    {
      const int64_t toy = (int64_t)blockIdx.x * 4 + (threadIdx.x >> 5);
      const int lane = threadIdx.x & 31;
      if (toy >= ntoys)
        return;
      // best run of the toy: lowest fval, lowest index on ties
      unsigned long long key = ~0ull;
      long long arg = 0x7fffffffffffffffll;
      for (int64_t r = lane; r < per_toy; r += 32) {
        const long long run = (long long)(toy * per_toy + r);
        const unsigned long long k = order_key(fval[run]);
        if (k < key || (k == key && run < arg)) {
          key = k;
          arg = run;
        }
      }
#pragma unroll
      for (int m = 16; m > 0; m >>= 1) {
        const unsigned long long k2 = __shfl_xor_sync(0xffffffffu, key, m);
        const long long a2 = __shfl_xor_sync(0xffffffffu, arg, m);
        if (k2 < key || (k2 == key && a2 < arg)) {
          key = k2;
          arg = a2;
        }
      }
      double* b = best + toy * 6;
      double* S = sens + toy * 4 * (int64_t)nbins;
      if (arg == 0x7fffffffffffffffll) { // no run: NaN sensitivities
        for (int i = lane; i < 4 * nbins; i += 32)
          S[i] = __longlong_as_double(0x7ff8000000000000ll);
        if (lane == 0)
          for (int q = 0; q < 6; ++q)
            b[q] = __longlong_as_double(0x7ff8000000000000ll);
        return;
      }
      const double a = x[arg * 4 + 0], bb = x[arg * 4 + 1];
      const double c = x[arg * 4 + 2], d = x[arg * 4 + 3];
      const double la = ::log(a);
      const double* xc = centres + toy * nbins;
      const int* kc = counts + toy * nbins;
      // H: 10 unique entries, plus sum (lambda - k)
      double h[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int i = lane; i < nbins; i += 32) {
        const double lx = ::log(xc[i]), l1 = ::log(1.0 - xc[i]);
        const double ll = la + fma(bb, l1, -fma(d, lx, c) * lx);
        const double lam = ::exp(ll);
        const double J[4] = {1.0 / a, l1, -lx, -lx * lx};
        int e = 0;
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int q = r; q < 4; ++q)
            h[e++] += lam * J[r] * J[q];
        h[10] += lam - (double)kc[i];
      }
#pragma unroll
      for (int e = 0; e < 11; ++e)
        h[e] = warp_sum(h[e]);
      double A[4][4];
      {
        int e = 0;
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int q = r; q < 4; ++q) {
            A[r][q] = h[e];
            A[q][r] = h[e];
            ++e;
          }
        A[0][0] -= h[10] / (a * a);
      }
      // Cholesky A = L L^T (every lane the same factor)
      double L[4][4] = {};
#pragma unroll
      for (int r = 0; r < 4; ++r) {
#pragma unroll
        for (int q = 0; q <= r; ++q) {
          double s = A[r][q];
#pragma unroll
          for (int m = 0; m < q; ++m)
            s -= L[r][m] * L[q][m];
          L[r][q] = (r == q) ? ::sqrt(s) : s / L[q][q];
        }
      }
      for (int i = lane; i < nbins; i += 32) {
        const double lx = ::log(xc[i]), l1 = ::log(1.0 - xc[i]);
        double z[4] = {1.0 / a, l1, -lx, -lx * lx};
#pragma unroll
        for (int r = 0; r < 4; ++r) { // L z' = J
#pragma unroll
          for (int m = 0; m < r; ++m)
            z[r] -= L[r][m] * z[m];
          z[r] /= L[r][r];
        }
#pragma unroll
        for (int r = 3; r >= 0; --r) { // L^T s = z'
#pragma unroll
          for (int m = r + 1; m < 4; ++m)
            z[r] -= L[m][r] * z[m];
          z[r] /= L[r][r];
        }
#pragma unroll
        for (int r = 0; r < 4; ++r)
          S[(int64_t)r * nbins + i] = z[r];
      }
      if (lane == 0) {
        b[0] = fval[arg];
        b[1] = a;
        b[2] = bb;
        b[3] = c;
        b[4] = d;
        b[5] = (double)arg;
      }
    }

  } // namespace

} // namespace zb

using namespace zb;

extern "C" {

int
zeus_nll_sensitivity_device(const zeus_problem* problem, int64_t n_instances,
                            int64_t runs_per_instance, const double* d_fval,
                            const double* d_x, double* d_best, double* d_sens,
                            void* stream)
{
  if (!problem || problem->kind != ZEUS_OBJ_POISSON_NLL || problem->dim != 4 ||
      !problem->data || !problem->idata || problem->ndata <= 0 ||
      n_instances < 0 || runs_per_instance <= 0 ||
      (n_instances > 0 && (!d_fval || !d_x || !d_best || !d_sens))) {
    set_error("zeus_nll_sensitivity_device: a Poisson NLL problem, "
              "runs_per_instance > 0 and device buffers are required");
    return ZEUS_E_INVALID;
  }
  if (n_instances == 0)
    return ZEUS_OK;
  const unsigned grid = (unsigned)((n_instances + 3) / 4);
  nll_sensitivity_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(
    problem->data, problem->idata, problem->ndata, n_instances,
    runs_per_instance, d_fval, d_x, d_best, d_sens);
  return cuda_fail(cudaGetLastError(), "NLL sensitivity launch");
}

} // extern "C"
