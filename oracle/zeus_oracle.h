/*
 * zeus_oracle.h -- CPU restatement of the reference hot path, used ONLY as
 * the checker by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg.  The product (zeus_b200/) never links or calls it.
 *
 * Parity pin: every BFGS entry here is compared bit for bit against the
 * reference's own sequential kernel body compiled for the host
 * (oracle/_ref/libzeus_ref.so, built by oracle/Makefile from the reference
 * sources), and against the known answers of the reference's tests
 * (test/bfgs_tests.cu, test/fun_tests.cu, test/dual_tests.cu,
 * test/pso_tests.cu) in tests/test_oracle.py.
 *
 * Arithmetic: plain IEEE double, no FMA contraction (-ffp-contract=off),
 * glibc libm for transcendentals -- the same as the reference's host build.
 */
#ifndef ZEUS_ORACLE_H
#define ZEUS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Objective kinds (shared numbering with the product's C-ABI). */
enum {
  ZOR_ROSENBROCK = 0,
  ZOR_RASTRIGIN = 1,
  ZOR_ACKLEY = 2,
  ZOR_GAUSSIAN = 3,
  ZOR_POISSON_NLL = 4
};

#define ZOR_MAX_DIM 256

/* Objective description: data = Gaussian C (dim*dim, row-major) or NLL bin
 * centres (ndata); idata = NLL bin counts (ndata). */
typedef struct {
  int kind;
  int dim;
  const double* data;
  const int* idata;
  int ndata;
} zor_objective;

/* f(x), reference double path. */
double zor_value(const zor_objective* o, const double* x);
/* f(x) and grad by D forward dual passes (duals.cuh:241-266). */
double zor_value_grad_dual(const zor_objective* o, const double* x,
                           double* grad);
/* Hand-derived analytic gradient (the adjoint's mathematics). */
double zor_value_grad_analytic(const zor_objective* o, const double* x,
                               double* grad);
/* Reference digamma (src/duals.cu:10-39). */
double zor_digamma(double x);

/* Reference backtracking line search (utils.cuh:376-412). */
double zor_line_search(const zor_objective* o, double f0, const double* x,
                       const double* p, const double* g);
/* Reference BFGS inverse update, O(D^3) with the m-sum hoisted; bit-identical
 * to the O(D^4) loop of utils.cuh:245-287 / 312-340. */
void zor_bfgs_update(int dim, double* H, const double* s, const double* y,
                     double sTy);

/* The reference's sequential BFGS (bfgs_sequential.cuh:46-234) over n runs in
 * index order, sharing one converged counter / stop flag.  Same signature as
 * zref_bfgs() in oracle/_ref.  Trajectory layout [iter][dim][run] and
 * [iter][run]; caller prefills NaN / -1.  Returns 0 or -1 (bad arguments). */
int zor_bfgs(int kind, int dim, const double* data, const int* idata,
             int ndata, const double* starts, int n, double lower,
             double upper, int max_iter, int required, double tol,
             double* fval, int* status, int* iter, double* gnorm,
             double* x_out, double* traj_x, double* traj_f, double* traj_g,
             signed char* traj_status, int nthreads);

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), 10 rounds. */
void zor_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2],
                       uint32_t out[4]);
/* The product's uniform double in [0,1): 53 bits of one Philox block.
 * stream tags: 1 = BFGS starts, 2 = PSO positions, 3 = PSO velocities,
 * 16+t = PSO iteration t (r1 at index 2d, r2 at 2d+1). */
double zor_uniform(uint64_t seed, uint32_t tag, uint64_t run, uint32_t index);
/* Uniform starts in [lower, upper): out[i*dim+d], tag 1. */
void zor_uniform_starts(uint64_t seed, int n, int dim, double lower,
                        double upper, double* out);

/* Sobol' points (the product's quasi-random starts, PRNGType::SOBOL of
 * traits.hpp:67-71 in own construction).  Direction numbers of dimensions
 * [0, ndim): dirs[d*32 + k] = v_(k+1) as a 32-bit fraction, from
 * polynomials poly[d] (bit i = coefficient of x^i; poly[0] unused) and
 * initial numbers minit[d*maxdeg + k] = m_(k+1). */
void zor_sobol_directions(int ndim, const uint32_t* poly,
                          const uint32_t* minit, int maxdeg, uint32_t* dirs);
/* The product's polynomials and initial numbers; -1 if maxdeg is too
 * small for ndim. */
int zor_sobol_params(int ndim, uint32_t* poly, uint32_t* minit, int maxdeg);
/* Shifted point `run`, coordinate d, in (0, 1). */
double zor_sobol01(const uint32_t* dirs, uint64_t seed, uint64_t run,
                   uint32_t d);
/* Starts in [lower, upper): Sobol' when sobol != NULL, else Philox tag 1. */
void zor_starts(uint64_t seed, const uint32_t* sobol, int n, int dim,
                double lower, double upper, double* out);

/* Synchronous PSO (pso.cuh:17-155 with gBest fixed at iteration boundaries,
 * ties to the lowest index).  Writes the BFGS starts (pBestX, n*dim) and the
 * per-particle best values.  Returns 0. */
int zor_pso(const zor_objective* o, uint64_t seed, int n, double lower,
            double upper, int iters, double w, double c1, double c2,
            double* pbest_x, double* pbest_f, double* gbest_x,
            double* gbest_f);
/* zor_pso with the initial positions from Sobol' directions `sobol` (NULL:
 * Philox, as zor_pso). */
int zor_pso_sobol(const zor_objective* o, uint64_t seed, const uint32_t* sobol,
                  int n, double lower, double upper, int iters, double w,
                  double c1, double c2, double* pbest_x, double* pbest_f,
                  double* gbest_x, double* gbest_f);

/* One reference PSO step for given r1/r2 (pso.cuh:104-119). */
void zor_pso_step(int dim, double w, double c1, double c2, const double* r1,
                  const double* r2, double* x, double* v, const double* pb,
                  const double* gb);

#ifdef __cplusplus
}
#endif
#endif
