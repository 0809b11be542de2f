// Runs zeus::Zeus on objective classes written for the reference, included
// unchanged from its examples tree: the dense Gaussian 0.5 x^T C x of
// examples/gaussian.hpp (a Matrix<double> member read through data()) and
// the binned Poisson likelihood of examples/simulation/fitting/LogLikelihood.h
// (std::vector and Matrix<int> members, a user specialisation of
// zeus::FnTraits).  Built against this library's include/ by
// zeus_b200/build.py; the checks against the oracle are in
// tests/test_gpu_reference_examples.py.
//
//   ref_objectives_test gaussian <dim 8|150> <N> <pso_iter> <max_iter> <seed>
//   ref_objectives_test nll <counts_and_centres.tsv> <N> <pso_iter> <max_iter> <seed>
//
// Prints one line: RESULT <status> <fval> <gradient norm> <iter> <x_0> ...
// with 17 significant digits.
#include <array>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "zeus.cuh"
#include "gaussian.hpp"
#include "simulation/fitting/LogLikelihood.h"

namespace {

  template <std::size_t D>
  void
  print(const zeus::Result<D>& r)
  {
    std::printf("RESULT %d %.17g %.17g %d", r.status, r.fval, r.gradientNorm, r.iter);
    for (std::size_t i = 0; i < D; ++i)
      std::printf(" %.17g", r.coordinates[i]);
    std::printf("\n");
  }

  // C_ii = 1 + (D - 1) / 2, C_ij = 1/2: the reference's Gaussian example
  template <std::size_t D>
  int
  gaussian(std::size_t n, int pso, int max_iter, int seed)
  {
    auto C = std::make_unique<std::array<std::array<double, D>, D>>();
    for (std::size_t i = 0; i < D; ++i)
      for (std::size_t j = 0; j < D; ++j)
        (*C)[i][j] = i == j ? 1.0 + 0.5 * (double)(D - 1) : 0.5;
    Gaussian<D> g(*C);
    const auto r = zeus::Zeus(g, -5.0, 5.0, n, max_iter, pso, (int)n + 1, "gaussian",
                              1e-8, seed, 0);
    print(r);
    return r.status == 1 ? 0 : 2;
  }

} // namespace

int
main(int argc, char** argv)
{
  if (argc < 7) {
    std::fprintf(stderr, "usage: %s gaussian|nll <dim|file> N pso max_iter seed\n",
                 argv[0]);
    return 1;
  }
  const std::string what = argv[1];
  const std::size_t n = std::strtoul(argv[3], nullptr, 10);
  const int pso = std::atoi(argv[4]), max_iter = std::atoi(argv[5]);
  const int seed = std::atoi(argv[6]);
  util::setStackSize();
  if (what == "gaussian") {
    const int dim = std::atoi(argv[2]);
    if (dim == 8)
      return gaussian<8>(n, pso, max_iter, seed);
    if (dim == 150)
      return gaussian<150>(n, pso, max_iter, seed);
    std::fprintf(stderr, "gaussian: dim 8 or 150\n");
    return 1;
  }
  if (what == "nll") {
    std::ifstream in(argv[2]);
    std::vector<int> counts;
    std::vector<double> centres;
    int k;
    double x;
    while (in >> k >> x) {
      counts.push_back(k);
      centres.push_back(x);
    }
    if (counts.empty()) {
      std::fprintf(stderr, "nll: no bins read from %s\n", argv[2]);
      return 1;
    }
    LogLikelihood ll(counts, centres);
    const auto r = zeus::Zeus(ll, 0.0, 10.0, n, max_iter, pso, (int)n + 1, "poisson",
                              1e-8, seed, 0);
    print(r);
    return 0;
  }
  std::fprintf(stderr, "unknown objective %s\n", what.c_str());
  return 1;
}
