// Trajectory files: the per-iteration records of exact-mode runs written in
// the reference's tab-separated layout (util::writeTrajectoryDataTSV,
// src/utils.cu:128-176).  Host code only.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "zb_internal.h"

using namespace zb;

namespace {

  // "%.17e" (what the reference's std::scientific, setprecision(17) stream
  // prints), "NaN" where the reference tests std::isnan
  void
  put_value(std::string& line, double v, bool nan_word)
  {
    char b[40];
    if (nan_word && std::isnan(v)) {
      line += "\tNaN";
      return;
    }
    const int k = std::snprintf(b, sizeof b, "\t%.17e", v);
    line.append(b, (size_t)k);
  }

  bool
  ends_with(const char* s, const char* suffix)
  {
    const size_t a = std::strlen(s), b = std::strlen(suffix);
    return a >= b && std::strcmp(s + a - b, suffix) == 0;
  }

} // namespace

extern "C" {

int
zeus_write_trajectory_tsv(const char* path, const double* coords,
                          const double* fval, const double* gnorm,
                          const int8_t* status, const double* alpha, int64_t n,
                          int32_t max_iter, int32_t dim)
{
  if (!path || n < 0 || max_iter < 0 || dim <= 0 ||
      (n > 0 && max_iter > 0 && (!coords || !fval || !gnorm || !status))) {
    set_error("zeus_write_trajectory_tsv: path, n >= 0, max_iter >= 0, dim > 0 "
              "and the four trajectory arrays are required");
    return ZEUS_E_INVALID;
  }
  if (!ends_with(path, ".tsv")) {
    set_error("zeus_write_trajectory_tsv: %s: only .tsv trajectory files are "
              "written (the reference's .nc form needs NetCDF, not built here)",
              path);
    return ZEUS_E_UNSUPPORTED;
  }
  std::FILE* fp = std::fopen(path, "w");
  if (!fp) {
    set_error("zeus_write_trajectory_tsv: cannot open %s for writing", path);
    return ZEUS_E_INVALID;
  }
  std::string line = "traj\tstep\tfval\tgrad\tstatus\talpha";
  for (int d = 0; d < dim; ++d)
    line += "\tx" + std::to_string(d);
  line += "\n";
  bool ok = std::fwrite(line.data(), 1, line.size(), fp) == line.size();
  const size_t N = (size_t)n;
  std::string chunk;
  chunk.reserve(1 << 20);
  for (size_t i = 0; ok && i < N; ++i) {
    for (size_t it = 0; it < (size_t)max_iter; ++it) {
      line = std::to_string(i) + "\t" + std::to_string(it);
      put_value(line, fval[it * N + i], true);
      put_value(line, gnorm[it * N + i], true);
      line += "\t" + std::to_string((int)status[it * N + i]);
      put_value(line, alpha ? alpha[it * N + i] : 0.0, false);
      for (size_t d = 0; d < (size_t)dim; ++d)
        put_value(line, coords[it * (size_t)dim * N + d * N + i], true);
      line += "\n";
      chunk += line;
      if (chunk.size() > (1u << 20) - 4096) {
        ok = std::fwrite(chunk.data(), 1, chunk.size(), fp) == chunk.size();
        chunk.clear();
      }
    }
  }
  if (ok && !chunk.empty())
    ok = std::fwrite(chunk.data(), 1, chunk.size(), fp) == chunk.size();
  if (std::fclose(fp) != 0)
    ok = false;
  if (!ok) {
    set_error("zeus_write_trajectory_tsv: write to %s failed", path);
    return ZEUS_E_INVALID;
  }
  return ZEUS_OK;
}

} // extern "C"

// ---- the per-call results file (util::appendResultsToTsv,
// include/util.hpp:79-136 / src/util.cpp:44-108; error from
// util::calculateEuclideanError, src/util.cpp:12-41)
extern "C" {

double
zeus_euclidean_error(const char* fun_name, const double* x, int32_t dim)
{
  if (!x || dim <= 0)
    return NAN;
  const std::string name = fun_name ? fun_name : "";
  double ss = 0.0;
  if (name == "rosenbrock") {
    for (int i = 0; i < dim; ++i) {
      const double d = x[i] - 1.0;
      ss += d * d;
    }
  } else if (name == "goldstein_price") {
    if (dim != 2)
      return NAN;
    const double dx = x[0] - 0.0, dy = x[1] - (-1.0);
    ss = dx * dx + dy * dy;
  } else {
    for (int i = 0; i < dim; ++i)
      ss += x[i] * x[i];
  }
  return std::sqrt(ss);
}

int
zeus_append_results_tsv(const char* dir, const char* fun_name, int32_t run,
                        int64_t n, int32_t dim, float ms_init, float ms_pso,
                        float ms_opt, float ms_rand, int32_t max_iter,
                        int32_t pso_iter, double error, const zeus_result* best,
                        const zeus_census* census, const double* coords,
                        const double* metrics)
{
  if (!best || !census || dim <= 0 || !coords) {
    set_error("zeus_append_results_tsv: best, census, dim > 0 and coords are required");
    return ZEUS_E_INVALID;
  }
  std::string path = dir && *dir ? std::string(dir) + "/" : std::string();
  path += "zeus_" + std::to_string(dim) + "d_results.tsv";
  std::FILE* fp = std::fopen(path.c_str(), "a");
  if (!fp) {
    set_error("zeus_append_results_tsv: cannot open %s", path.c_str());
    return ZEUS_E_INVALID;
  }
  std::string out;
  std::fseek(fp, 0, SEEK_END);
  if (std::ftell(fp) == 0) { // a new or empty file gets the header
    out = "fun\trun\tN\tkernel"
          "\tad_ms_per_call\tad_calls_per_thread_mean\tad_fraction\tad_block95"
          "\tad_serialized"
          "\tbfgs_ms_per_call\tbfgs_calls_per_thread_mean\tbfgs_fraction"
          "\tbfgs_block95\tbfgs_serialized"
          "\tclaimed\tactual\tsurrender\tstopped\tidx\tstatus\tbfgs_iter"
          "\tpso_iter\ttime\terror\tfval\tnorm";
    for (int i = 0; i < dim; ++i)
      out += "\tcoord_" + std::to_string(i);
    out += "\n";
  }
  char b[64];
  // the stream's default floating format is %g (precision 6) until
  // std::scientific switches it to %.6e for error, fval, norm and the
  // coordinates
  auto g = [&](double v) {
    std::snprintf(b, sizeof b, "%g", v);
    out += b;
  };
  auto e = [&](double v) {
    std::snprintf(b, sizeof b, "%e", v);
    out += b;
  };
  out += std::string(fun_name ? fun_name : "") + "\t" + std::to_string(run) + "\t" +
         std::to_string(n) + "\t";
  g(ms_opt);
  // metrics: AD then BFGS, each {ms_per_call, calls_per_thread_mean,
  // fraction_of_thread, block95, serialized}; this library does not sample
  // per-call cycle counts, so its callers pass NULL (zeros)
  for (int k = 0; k < 10; ++k) {
    out += "\t";
    g(metrics ? metrics[k] : 0.0);
  }
  out += "\t" + std::to_string(census->claimed) + "\t" + std::to_string(census->actual) +
         "\t" + std::to_string(census->surrendered) + "\t" +
         std::to_string(census->stopped) + "\t" + std::to_string(best->idx) + "\t" +
         std::to_string(best->status) + "\t" + std::to_string(max_iter) + "\t" +
         std::to_string(pso_iter) + "\t";
  const double t = pso_iter > 0 ? (double)ms_init + ms_pso + ms_opt + ms_rand
                                : (double)ms_opt + ms_rand;
  g(t);
  out += "\t";
  e(error);
  out += "\t";
  e(best->fval);
  out += "\t";
  e(best->gradient_norm);
  out += "\t";
  for (int i = 0; i < dim; ++i) {
    e(coords[i]);
    if (i < dim - 1)
      out += "\t";
  }
  out += "\n";
  const bool ok = std::fwrite(out.data(), 1, out.size(), fp) == out.size();
  if (std::fclose(fp) != 0 || !ok) {
    set_error("zeus_append_results_tsv: write to %s failed", path.c_str());
    return ZEUS_E_INVALID;
  }
  return ZEUS_OK;
}

int
zeus_cycle_metrics(const int64_t* cycles, const int64_t* counters, int64_t n,
                   int32_t which, double sm_clock_khz, float ms_opt,
                   int32_t runs_per_block, double metrics[8])
{
  if (!cycles || !counters || !metrics || n <= 0 || (which != 0 && which != 1) ||
      !(sm_clock_khz > 0.0) || runs_per_block <= 0) {
    set_error("zeus_cycle_metrics: cycles, counters, metrics, n > 0, which 0/1, "
              "a clock and runs_per_block > 0 are required");
    return ZEUS_E_INVALID;
  }
  // the timer's cycles and calls per run: AD = gradient evaluations, BFGS =
  // updates (one after each gradient evaluation but the first)
  const int cyc_col = which == 0 ? 0 : 1;
  const double hz = sm_clock_khz * 1000.0;
  unsigned long long sum_cycles = 0ULL;
  long long sum_calls = 0LL;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t grads = counters[3 * i + 2];
    sum_cycles += (unsigned long long)cycles[3 * i + cyc_col];
    sum_calls += which == 0 ? grads : (grads > 0 ? grads - 1 : 0);
  }
  const double avg_cycles = double(sum_cycles) / double(n);
  const double avg_calls = sum_calls > 0 ? double(sum_calls) / double(n) : 0.0;
  const double avg_cycles_per_call = avg_calls > 0 ? avg_cycles / avg_calls : 0.0;
  const double ms_per_call = avg_cycles_per_call / hz * 1e3;
  const double serialized_ms = double(sum_cycles) / hz * 1e3;
  const double serialized = ms_opt > 0.0 ? serialized_ms / ms_opt : 0.0;
  // mean over runs of this timer's share of the run's cycles
  long double acc = 0.0L;
  long long cnt = 0;
  for (int64_t i = 0; i < n; ++i) {
    const double tot = (double)cycles[3 * i + 2];
    if (tot > 0.0) {
      acc += (long double)((double)cycles[3 * i + cyc_col] / tot);
      ++cnt;
    }
  }
  const double frac_thread = cnt > 0 ? (double)(acc / (long double)cnt) : 0.0;
  // 95th percentile of the per-block summed time over ms_opt
  const int64_t blocks = (n + runs_per_block - 1) / runs_per_block;
  std::vector<long double> bc((size_t)blocks, 0.0L);
  for (int64_t i = 0; i < n; ++i)
    bc[(size_t)(i / runs_per_block)] += (long double)cycles[3 * i + cyc_col];
  std::vector<double> fb((size_t)blocks);
  for (int64_t b = 0; b < blocks; ++b)
    fb[(size_t)b] = (double)(bc[(size_t)b] / hz * 1e3L) / (double)ms_opt;
  std::sort(fb.begin(), fb.end());
  const size_t i95 = std::min<size_t>(
    fb.size() - 1, (size_t)std::ceil(0.95 * (double)fb.size()) - 1);
  const double ms_per_thread = avg_cycles / hz * 1e3;
  metrics[0] = ms_per_call;
  metrics[1] = avg_calls;
  metrics[2] = frac_thread;
  metrics[3] = fb[i95];
  metrics[4] = serialized;
  metrics[5] = ms_per_thread > 0.0 && ms_opt > 0.0 ? ms_per_thread / ms_opt : 0.0;
  metrics[6] = avg_cycles;
  metrics[7] = ms_per_thread;
  return ZEUS_OK;
}

} // extern "C"
