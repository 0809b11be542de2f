// Trajectory files: the per-iteration records of exact-mode runs written in
// the reference's tab-separated layout (util::writeTrajectoryDataTSV,
// src/utils.cu:128-176).  Host code only.
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
