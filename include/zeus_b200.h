/*
 * zeus_b200.h -- C ABI of the B200 (sm_100a) global optimiser.
 *
 * Plain C: pointers, sizes, PODs; no exceptions cross it; every entry point
 * returns ZEUS_OK (0) or a negative ZEUS_E* code, with a message available
 * from zeus_last_error() on the calling host thread.  Device pointers are
 * marked d_; streams are cudaStream_t passed as void* (NULL = legacy default
 * stream).  All device entry points are asynchronous on that stream unless
 * stated otherwise.
 *
 * The reference (fnal-numerics/zeus) is a header-only C++ template library
 * with no FFI of its own; each entry point below replaces the reference
 * function named in its comment (file:line in the reference tree), so a C,
 * ctypes, cgo or JNI caller binds these in place of instantiating the
 * templates.  The C++ drop-in (include/zeus.cuh, zeus::Zeus) is built on the
 * same kernels.
 */
#ifndef ZEUS_B200_H
#define ZEUS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ---------------------------------------------------- */
#define ZEUS_OK 0
#define ZEUS_E_INVALID (-1)     /* bad argument */
#define ZEUS_E_UNSUPPORTED (-2) /* (objective, dim, layout) not built */
#define ZEUS_E_CUDA (-3)        /* CUDA runtime error (launch or sync) */
#define ZEUS_E_NOMEM (-4)       /* device allocation failed */
#define ZEUS_E_WORKSPACE (-5)   /* workspace too small */

/* ---- per-run status, the reference's Result::status (util.hpp:39-44,
 * bfgs_common.cuh:110-273) ------------------------------------------------- */
#define ZEUS_STATUS_UNSET (-1)
#define ZEUS_STATUS_SURRENDER 0 /* MAX_ITER reached */
#define ZEUS_STATUS_CONVERGED 1 /* ||grad|| < tol */
#define ZEUS_STATUS_STOPPED 2   /* required_converged reached elsewhere */
#define ZEUS_STATUS_NOMEM 3     /* allocation failure (whole call) */
#define ZEUS_STATUS_KERNEL 4    /* launch / runtime failure (whole call) */
#define ZEUS_STATUS_NONFINITE 5 /* non-finite f or ||grad|| */

/* ---- built-in objectives (examples/rosenbrock.hpp, rastrigin.hpp,
 * ackley.hpp, gaussian.hpp, simulation/fitting/LogLikelihood.h) ---------- */
#define ZEUS_OBJ_ROSENBROCK 0
#define ZEUS_OBJ_RASTRIGIN 1
#define ZEUS_OBJ_ACKLEY 2
#define ZEUS_OBJ_GAUSSIAN 3    /* 0.5 x^T C x, data = C (dim*dim) */
#define ZEUS_OBJ_POISSON_NLL 4 /* dim 4, data = bin centres, idata = counts */

#define ZEUS_PROBLEM_SYMMETRIC 1 /* zeus_problem.flags: Gaussian C = C^T */

/* ---- arithmetic mode ---------------------------------------------------
 * EXACT: the reference's operation order (O(D^3) hoisted update that equals
 *        its O(D^4) loop, no FMA contraction, dual gradients): per-iterate
 *        identical to the reference for polynomial objectives.
 * FAST:  O(D^2) symmetric rank-2 update with FMA, layout by dimension,
 *        dual or adjoint gradients.                                        */
#define ZEUS_MODE_EXACT 0
#define ZEUS_MODE_FAST 1

#define ZEUS_GRAD_DUAL 0    /* D forward dual passes (duals.cuh:241-266) */
#define ZEUS_GRAD_ADJOINT 1 /* hand-written reverse-mode gradient */

/* zeus_bfgs_config.flags
 * NO_FIXED_POINT: keep iterating a run whose iteration changed nothing.  By
 *   default a run whose step was rejected (f_new >= best) AND whose update
 *   was skipped (|s.y| < 1e-14) ends at once with status 0 and iter =
 *   max_iter: its state (x, g, H, best) is unchanged, so every remaining
 *   iteration would repeat it bit for bit and the reference would return
 *   exactly that result at MAX_ITER (with stop-early on, it is the result the
 *   reference gives when the run reaches MAX_ITER before the stop flag).
 *   Trajectory recording always iterates to the end. */
#define ZEUS_FLAG_NO_FIXED_POINT 1

#define ZEUS_LAYOUT_AUTO 0
#define ZEUS_LAYOUT_THREAD 1 /* one run per thread, H in registers */
#define ZEUS_LAYOUT_TILE 2   /* one run per 2..32-lane tile, H rows per lane */
#define ZEUS_LAYOUT_CTA 3    /* one run per CTA, H in shared memory */
#define ZEUS_LAYOUT_ROWS 4   /* one run per group of S*dim threads, each holding
                                a segment of one row of H in registers; several
                                groups per block (dim 64: 128 threads; dim 128:
                                384 or 512) */

typedef struct zeus_problem {
  int32_t kind;         /* ZEUS_OBJ_* */
  int32_t dim;          /* number of parameters D */
  const double* data;   /* Gaussian C (row-major dim*dim) or NLL centres */
  const int32_t* idata; /* NLL counts */
  int32_t ndata;        /* NLL bins */
  int32_t flags;        /* ZEUS_PROBLEM_SYMMETRIC: data matrix is symmetric */
} zeus_problem;

typedef struct zeus_bfgs_config {
  int32_t max_iter;           /* MAX_ITER */
  int32_t required_converged; /* stop-early threshold (> n disables) */
  double tolerance;           /* ||grad||_2 < tolerance => converged */
  int32_t mode;               /* ZEUS_MODE_* */
  int32_t gradient;           /* ZEUS_GRAD_* */
  int32_t layout;             /* ZEUS_LAYOUT_* */
  int32_t tile;               /* lanes per run for TILE (0 = auto) */
  int32_t block;              /* threads per block (0 = auto) */
  int32_t flags;              /* ZEUS_FLAG_* */
  int32_t prng;               /* ZEUS_PRNG_*: start positions (zeus_optimize) */
} zeus_bfgs_config;

/* Per-run outputs, all device pointers; NULL members are not written.
 * x is row-major [run][dim].  counters (optional) receives per run
 * {BFGS iterations, f evaluations, gradient evaluations} as int64[3].
 * Trajectories use the reference layout [iter][dim][run] and [iter][run]
 * (bfgs_sequential.cuh:100-109); they must hold max_iter steps and be
 * prefilled by the caller (NaN, status -1).  cycles (optional) receives per
 * run {gradient cycles, update cycles, whole-run cycles} as int64[3]: the
 * reference's ad_cycles / bfgs_cycles / total_cycles clock64 timers
 * (bfgs_sequential.cuh:40-44, 222-232), sampled only when it is non-NULL.
 * The update span includes the new search direction where a layout forms
 * both in one pass over H.  Calls per run follow from counters' gradient
 * evaluations (see zeus_cycle_metrics).  zeus_bfgs_device samples them
 * (its kernels are built with and without the timers, so asking costs
 * nothing when not asked); the persistent batch does not and rejects a class
 * whose cycles are set. */
typedef struct zeus_run_outputs {
  double* fval;
  int32_t* status;
  int32_t* iter;
  double* gnorm;
  double* x;
  int64_t* counters;
  double* traj_x;
  double* traj_f;
  double* traj_g;
  int8_t* traj_status;
  int64_t* cycles;
} zeus_run_outputs;

/* The reference's Result<D> minus the coordinate array (util.hpp:36-54). */
typedef struct zeus_result {
  int32_t idx;
  int32_t status;
  double fval;
  double gradient_norm;
  int32_t iter;
  int32_t reserved;
} zeus_result;

/* The reference's Convergence census (util.hpp:27-32, 151-200). */
typedef struct zeus_census {
  int32_t actual;      /* status 1 and within 0.5 of the known minimum */
  int32_t claimed;     /* status 1 */
  int32_t surrendered; /* any status other than 1 and 2 */
  int32_t stopped;     /* status 2 */
  int32_t best_idx;    /* argmin fval (lowest index on ties) */
  int32_t reserved;
} zeus_census;

/* ---- runtime -------------------------------------------------------- */
/* Message of the last failing call on this host thread ("" if none). */
const char* zeus_last_error(void);
/* Library version string. */
const char* zeus_version(void);
/* 1 if (problem kind, dim) has built kernels for (mode, gradient). */
int zeus_supported(int32_t kind, int32_t dim, int32_t mode, int32_t gradient);

/* ---- start-position generators (the reference's PRNGType,
 * traits.hpp:67-71) ------------------------------------------------------
 * XORWOW, PHILOX: Philox4x32-10, counter-based, no per-run state (cuRAND's
 *   XORWOW, the reference's default, is not reproduced; Philox takes its
 *   place).
 * SOBOL: start positions (and the PSO's initial swarm) are points of a
 *   Sobol' sequence, run i = point i, coordinate d = dimension d (d < 1024),
 *   digitally shifted by the seed: the starts of any 2^m consecutive runs
 *   are stratified in every coordinate.  Velocities and the PSO's r1/r2 stay
 *   on Philox.  Own direction numbers: primitive polynomials in order of
 *   degree then value, initial numbers from a fixed splitmix64 stream. */
#define ZEUS_PRNG_XORWOW 0
#define ZEUS_PRNG_PHILOX 1
#define ZEUS_PRNG_SOBOL 2

/* ---- starts ---------------------------------------------------------
 * Starts in [lower, upper): d_out[i*dim+d] = lower + (upper - lower) * u
 * with u from the generator `prng`, run index i.  Replaces the reference's
 * in-kernel cuRAND draws when PSO is off (bfgs_sequential.cuh:73-77,
 * utils.cuh:353-358).  The first SOBOL call on a device copies the direction
 * table to it (synchronous): make it before any stream capture. */
int zeus_starts(uint64_t seed, int32_t prng, int64_t n, int32_t dim,
                double lower, double upper, double* d_out, void* stream);
/* zeus_starts with ZEUS_PRNG_PHILOX. */
int zeus_starts_uniform(uint64_t seed, int64_t n, int32_t dim, double lower,
                        double upper, double* d_out, void* stream);
/* Host copy of the Sobol' direction numbers of dimensions [0, ndim), ndim
 * <= 1024: out[d*32 + k] = v_{k+1} of dimension d, a 32-bit binary
 * fraction.  Host only; no device is touched. */
int zeus_sobol_directions(int32_t ndim, uint32_t* out);
/* Device address of the full direction table (1024 x 32 uint32) on the
 * current device, copied there on the first call (synchronous). */
int zeus_sobol_device_table(const uint32_t** d_table);

/* ---- PSO seeding ----------------------------------------------------
 * Replaces pso::launch (pso.cuh:194-345; kernels 17-155): init plus `iters`
 * synchronous PSO steps (gBest fixed at each iteration boundary by a
 * deterministic argmin, ties to the lowest index), all launched on `stream`
 * with no host round trip.  Outputs the per-particle best positions (the
 * BFGS starts, d_pbest_x[n*dim]) and values; d_gbest receives {f, x[dim]}.
 * Workspace: zeus_pso_workspace_size() bytes of device memory. */
size_t zeus_pso_workspace_size(int64_t n, int32_t dim);
int zeus_pso_device(const zeus_problem* problem, uint64_t seed, int64_t n,
                    double lower, double upper, int32_t iters, double w,
                    double c1, double c2, double* d_pbest_x,
                    double* d_pbest_f, double* d_gbest, void* d_workspace,
                    size_t workspace_bytes, void* stream);
/* zeus_pso_device with the initial positions from generator `prng`
 * (ZEUS_PRNG_*; zeus_pso_device is ZEUS_PRNG_PHILOX), as the reference's
 * pso::launch takes its cuRAND state type (pso.cuh:194-210). */
int zeus_pso_device_prng(const zeus_problem* problem, uint64_t seed,
                         int32_t prng, int64_t n, double lower, double upper,
                         int32_t iters, double w, double c1, double c2,
                         double* d_pbest_x, double* d_pbest_f,
                         double* d_gbest, void* d_workspace,
                         size_t workspace_bytes, void* stream);

/* No counterpart in the reference (its pso::launch allocates its buffers
 * itself, pso.cuh:211-241).  zeus_pso_device without the workspace, for
 * callers that cannot allocate device memory where they seed a swarm (an
 * allocator owned by another framework, allocation-free real-time loops,
 * hosts that must not let an allocation synchronize the device).  The swarm
 * state lives in one 8 MiB array compiled into the library, which every GPU
 * that loads the library keeps until the process exits; calls needing more
 * (zeus_pso_workspace_size(n, dim) > 8 MiB) are rejected with
 * ZEUS_E_WORKSPACE.  The first call on a device looks the array's device
 * address up (cudaGetSymbolAddress), so make that first call before any
 * stream capture.  All calls share the array and it keeps the last call's
 * contents; each call clears what must start at zero, but calls that
 * overlap on the GPU race on it: serialize them.  Outputs as for
 * zeus_pso_device (Philox positions, as ZEUS_PRNG_PHILOX). */
int zeus_pso_device_noalloc(const zeus_problem* problem, uint64_t seed,
                            int64_t n, double lower, double upper,
                            int32_t iters, double w, double c1, double c2,
                            double* d_pbest_x, double* d_pbest_f,
                            double* d_gbest, void* stream);

/* ---- BFGS -----------------------------------------------------------
 * Replaces bfgs::sequential::launch / bfgs::parallel::launch
 * (bfgs_sequential.cuh:384-589, bfgs_parallel.cuh:301-472) and their
 * kernels: one FP64 BFGS per start d_starts[i*dim+d], with the reference's
 * line search, update skip, accept-if-better and termination protocol.
 * d_control: 2 int32 {stop flag, converged count}, zeroed by the caller
 * before the first launch (the reference's BFGSContext, context.hpp:7-10).
 * Workspace: zeus_bfgs_workspace_size() bytes: none for the thread and tile
 * layouts; the CTA layout (dim > 32) keeps its blocks' run queue there (a
 * block that finishes a run takes the next unstarted one) and, past about
 * dim 160, each block's H. */
size_t zeus_bfgs_workspace_size(const zeus_problem* problem,
                                const zeus_bfgs_config* config, int64_t n);
int zeus_bfgs_device(const zeus_problem* problem,
                     const zeus_bfgs_config* config, const double* d_starts,
                     int64_t n, const zeus_run_outputs* out,
                     int32_t* d_control, void* d_workspace,
                     size_t workspace_bytes, void* stream);

/* ---- persistent batch -----------------------------------------------
 * No single reference counterpart: the reference runs one objective per
 * zeus::Zeus call (zeus.cuh:341-375), one kernel launch per call.  This
 * runs up to 16 classes -- each an objective and dimension with its own
 * runs, starts, outputs and stop-early control, as one Zeus call would --
 * in ONE persistent kernel launch.  Slots are refilled from per-class
 * atomic queues as runs finish; CTA-layout classes (dim > 32) go first,
 * smallest dimension first, then the warp-sized ones (one block in 16 takes
 * the warp-sized ones first).  A class may carry several data instances
 * stored one
 * after another (Gaussian: dim*dim doubles each; NLL: ndata centres and
 * ndata counts each), run r using instance r / runs_per_instance.
 * Fast mode with adjoint gradients only (config->mode, ->gradient);
 * config->max_iter, ->tolerance and ->flags apply to every class;
 * config->block picks the kernel's block size, 512 or 384 threads (0: 512
 * when the tile/thread classes hold more than two waves of warps, else
 * 384, whose threads get more registers). */
typedef struct zeus_batch_class {
  zeus_problem problem;       /* data on the device */
  int64_t n;                  /* runs */
  int64_t runs_per_instance;  /* 0: every run uses the one instance */
  const double* d_starts;     /* n*dim, row-major */
  zeus_run_outputs out;       /* per-run outputs (trajectories ignored) */
  int32_t* d_control;         /* 2 int32 {stop, converged}, zeroed */
  int32_t required_converged; /* stop-early threshold of this class */
  int32_t layout;             /* ZEUS_LAYOUT_* (AUTO: autotuned/default) */
  int32_t tile;               /* tile width for ZEUS_LAYOUT_TILE */
  int32_t reserved;
} zeus_batch_class;

size_t zeus_batch_workspace_size(const zeus_batch_class* classes,
                                 int32_t n_classes);
int zeus_batch_device(const zeus_batch_class* classes, int32_t n_classes,
                      const zeus_bfgs_config* config, void* d_workspace,
                      size_t workspace_bytes, void* stream);

/* ---- persistent batch with host buffers --------------------------------
 * The reference runs one objective per zeus::Zeus call, with host inputs
 * and a host Result back (zeus.cuh:341-375; the best run by
 * bfgs_common.cuh:280-319).  A batch plan does that for up to 16 classes in
 * one persistent kernel launch: it owns the device copies of every class's
 * objective data and starts, the per-run outputs and the batch workspace,
 * allocated once at creation on the current device.  Each run copies the
 * classes' HOST inputs to the device (objective data, and starts when given;
 * without host starts a class draws them on the device from `seed`: PSO
 * when pso_iter >= 0, as pso::launch, else uniform Philox starts in
 * [lower, upper)), runs zeus_batch_device, reduces every class (argmin with
 * ties to the lowest index, census as zeus_census_device) and returns per
 * class the best run (best[c]), its coordinates (best_x: the classes'
 * coordinates one after another, sum of dims doubles) and the census
 * (census[c], may be NULL), with one device-to-host copy and one
 * synchronisation of `stream`.  Runs must use the plan's device and class
 * shapes (kind, dim, ndata, n, runs_per_instance, host-or-device starts);
 * the data and starts may change between runs.  Errors set every
 * best[c].status to 3 (allocation) or 4 (CUDA), as zeus_optimize does. */
typedef struct zeus_host_class {
  zeus_problem problem;       /* data / idata: HOST pointers to every instance */
  int64_t n;                  /* runs */
  int64_t runs_per_instance;  /* 0: every run uses the one instance */
  const double* starts;       /* HOST n*dim starts, or NULL: drawn on the device */
  uint64_t seed;              /* starts == NULL: the generator's seed */
  double lower;               /* starts == NULL: bounds of the draw / swarm */
  double upper;
  int32_t pso_iter;           /* starts == NULL: >= 0 PSO iterations, < 0 uniform */
  int32_t required_converged; /* stop-early threshold of this class */
  int32_t layout;             /* ZEUS_LAYOUT_* */
  int32_t tile;               /* tile width for ZEUS_LAYOUT_TILE */
} zeus_host_class;

typedef struct zeus_batch_plan zeus_batch_plan;
int zeus_batch_plan_create(const zeus_host_class* classes, int32_t n_classes,
                           const zeus_bfgs_config* config, zeus_batch_plan** plan);
int zeus_batch_plan_run(zeus_batch_plan* plan, const zeus_host_class* classes,
                        zeus_result* best, double* best_x, zeus_census* census,
                        void* stream);
/* Bytes the last run copied host-to-device, and the bytes every run copies
 * back. */
int zeus_batch_plan_traffic(const zeus_batch_plan* plan, size_t* h2d_bytes,
                            size_t* d2h_bytes);
int zeus_batch_plan_destroy(zeus_batch_plan* plan);

/* ---- fit sensitivities ----------------------------------------------------
 * No counterpart in the reference (its dijet fit stops at the minimum,
 * examples/fit_dijet_spectrum.cu:162-221).  For a Poisson NLL batch with
 * n_instances toy spectra (problem->data / idata: ndata centres and counts
 * per toy, one toy after another) and runs_per_instance runs per toy
 * (d_fval and d_x hold n_instances * runs_per_instance runs):
 * picks each toy's best run (lowest fval, lowest index on ties) and writes
 * d_best[toy*6 + {0..5}] = {fval, a, b, c, d, run index} and the implicit-
 * function derivatives of the fitted parameters with respect to the bin
 * counts, d_sens[(toy*4 + param)*ndata + bin] = d p_param / d k_bin
 * = (H^-1 J_bin)_param, H the exact Hessian of the NLL at the fit, J_bin =
 * d ln lambda_bin / dp. */
int zeus_nll_sensitivity_device(const zeus_problem* problem,
                                int64_t n_instances, int64_t runs_per_instance,
                                const double* d_fval, const double* d_x,
                                double* d_best, double* d_sens, void* stream);

/* ---- layout autotuner -------------------------------------------------
 * No reference counterpart (the reference fixes thread-per-run or a tile
 * of min(32, 2^floor(log2 D)) lanes, bfgs_parallel.cuh:57-65).  Times every
 * built layout / tile width for (problem, config) on n_sample uniform
 * starts in [lower, upper), and one run's iteration alone (200 iterations
 * that neither converge nor stop early); a layout's estimate is the longer
 * of the sample's time and max_iter of those iterations (a batch lasts as
 * long as its slowest run, one that iterates to max_iter).  Records the
 * layout with the lowest estimate in a per-process table keyed by (device,
 * kind, dim, gradient); ZEUS_LAYOUT_AUTO launches and batches then use it.
 * Synchronous.  *best_ms is the winner's estimate. */
int zeus_autotune(const zeus_problem* problem, const zeus_bfgs_config* config,
                  int64_t n_sample, uint64_t seed, double lower, double upper,
                  int32_t* best_layout, int32_t* best_tile, float* best_ms,
                  void* stream);
/* 1 and the recorded choice if (kind, dim, gradient) is in the table for
 * the current device, else 0. */
int zeus_autotune_lookup(int32_t kind, int32_t dim, int32_t gradient,
                         int32_t* layout, int32_t* tile);
/* Records a choice (e.g. from a previous process) for the current device. */
int zeus_autotune_record(int32_t kind, int32_t dim, int32_t gradient,
                         int32_t layout, int32_t tile);

/* ---- gradient evaluation ----------------------------------------------
 * Replaces dual::calculateGradientUsingAD (duals.cuh:241-266) as a call of
 * its own, for checking every gradient path of the BFGS layouts at given
 * points: writes f(x_i) to d_f[i] and grad f(x_i) to d_g[i*dim + d] for the
 * n points d_x[i*dim + d] (row-major), evaluated by the device functions the
 * BFGS kernels step on.  `gradient` is ZEUS_GRAD_DUAL (the plain form's D
 * forward dual passes) or ZEUS_GRAD_ADJOINT (the hand-written reverse-mode
 * gradient); `path` picks the layout:
 *   THREAD     one thread per point (dim <= 32; the thread layout);
 *   TILE       a tile of `width` lanes per point, value and gradient in one
 *              cooperative call (a width zeus_tile_widths reports);
 *   TILE_GRAD  the tile's gradient-only form (adjoint only; f from the
 *              cooperative value) -- the form tile_run calls;
 *   CTA        a block of `width` threads per point (a multiple of 32, at
 *              most 512), the CTA layout's and the persistent batch's calls;
 *   CTA_GRAD   the block's gradient-only form (adjoint only);
 *   QUADRATIC  Gaussian with symmetric C (adjoint only, width >= dim): the
 *              CTA line search's carried point x_i + alpha p_i, from one
 *              pass over C at (x_i, p_i) (d_p: n*dim directions): d_f =
 *              f(x) + alpha grad f(x).p + alpha^2 f(p), d_g = C x + alpha C p.
 * Workspace: zeus_gradient_workspace_size() bytes (the NLL's per-bin
 * constants; 0 otherwise). */
#define ZEUS_GRADPATH_THREAD 0
#define ZEUS_GRADPATH_TILE 1
#define ZEUS_GRADPATH_TILE_GRAD 2
#define ZEUS_GRADPATH_CTA 3
#define ZEUS_GRADPATH_CTA_GRAD 4
#define ZEUS_GRADPATH_QUADRATIC 5
size_t zeus_gradient_workspace_size(const zeus_problem* problem);
int zeus_gradient_device(const zeus_problem* problem, int32_t path,
                         int32_t gradient, int32_t width, const double* d_x,
                         const double* d_p, double alpha, int64_t n,
                         double* d_f, double* d_g, void* d_workspace,
                         size_t workspace_bytes, void* stream);
/* Bit k set: the tile layout is built with 2^k lanes per run for
 * (kind, dim); 0 if it has no tile layout. */
uint32_t zeus_tile_widths(int32_t kind, int32_t dim);

/* ---- reduction ------------------------------------------------------
 * Replaces bfgs::launchReduction + util::dumpDataToFile's census
 * (bfgs_common.cuh:280-319, util.hpp:151-200): argmin of fval (lowest index
 * on ties, NaN never wins) and status counts, in one kernel.  known_min is a
 * HOST pointer to dim doubles (NULL: origin) used for `actual`. */
int zeus_census_device(const double* d_fval, const int32_t* d_status,
                       const double* d_x, int64_t n, int32_t dim,
                       const double* known_min, zeus_census* d_census,
                       void* stream);

/* ---- whole call with host buffers -------------------------------------
 * The drop-in for zeus::Zeus (zeus.cuh:341-375) on a built-in objective:
 * problem data in HOST memory, PSO (pso_iter >= 0; pso_iter < 0 draws
 * uniform starts), BFGS, argmin and census; synchronous.  Copies the best
 * run into *best / best_x (host, dim doubles) and, when per_run_* are not
 * NULL, every run's fval/status (host arrays of n).  Returns ZEUS_OK, or an
 * error code with best->status set to 3 (allocation) or 4 (CUDA), as the
 * reference does (zeus.cuh:112-116). */
int zeus_optimize(const zeus_problem* host_problem, double lower,
                  double upper, int64_t n, int32_t max_iter, int32_t pso_iter,
                  int32_t required_converged, double tolerance, uint64_t seed,
                  const zeus_bfgs_config* config, zeus_result* best,
                  double* best_x, zeus_census* census, double* per_run_fval,
                  int32_t* per_run_status, void* stream);

/* ---- trajectory files -------------------------------------------------
 * Replaces util::writeTrajectoryData's TSV form (src/utils.cu:128-176,
 * 258-286): writes `path` (must end in .tsv) with the header
 * "traj step fval grad status alpha x0 .. x{dim-1}" (tab-separated) and one
 * row per run and step, all max_iter steps of every run, values as %.17e
 * (the reference's scientific, precision 17), NaN printed "NaN".  The
 * arrays are HOST copies of an exact-mode run's trajectory buffers
 * (zeus_run_outputs layouts: coords[step][dim][run], fval / gnorm /
 * status[step][run]); alpha (same layout) may be NULL for zeros, which is
 * what the reference's sequential path writes.  The reference's .nc form
 * needs NetCDF and is not built: such paths return ZEUS_E_UNSUPPORTED. */
int zeus_write_trajectory_tsv(const char* path, const double* coords,
                              const double* fval, const double* gnorm,
                              const int8_t* status, const double* alpha,
                              int64_t n, int32_t max_iter, int32_t dim);

/* ---- the per-call results file ---------------------------------------
 * Replaces util::calculateEuclideanError (src/util.cpp:12-41): distance of
 * x from the known minimum by function name -- (1, ..., 1) for
 * "rosenbrock", (0, -1) for "goldstein_price" (dim 2 only, else NaN), the
 * origin otherwise. */
double zeus_euclidean_error(const char* fun_name, const double* x, int32_t dim);
/* Replaces util::appendResultsToTsv (src/util.cpp:44-108), which every
 * zeus::Zeus call runs: appends one row to zeus_<dim>d_results.tsv in
 * `dir` (NULL or "": the current directory), writing the reference's header
 * first when the file is new or empty.  Columns and number formats are the
 * reference's: times and metrics as %g, error / fval / norm / coordinates
 * as %e; `time` is ms_init + ms_pso + ms_opt + ms_rand when pso_iter > 0,
 * else ms_opt + ms_rand.  `metrics` holds the AD then BFGS
 * {ms_per_call, calls_per_thread_mean, fraction_of_thread, block95,
 * serialized} (10 doubles, see zeus_cycle_metrics) or NULL for zeros. */
int zeus_append_results_tsv(const char* dir, const char* fun_name, int32_t run,
                            int64_t n, int32_t dim, float ms_init, float ms_pso,
                            float ms_opt, float ms_rand, int32_t max_iter,
                            int32_t pso_iter, double error,
                            const zeus_result* best, const zeus_census* census,
                            const double* coords, const double* metrics);

/* Replaces bfgs::sequential::report_metrics_and_cleanup
 * (bfgs_sequential.cuh:236-373) for one of its two timers, from HOST
 * copies of zeus_run_outputs' cycles and counters (n runs each): `which` 0
 * is the AD timer (gradient cycles; calls = gradient evaluations), 1 the
 * BFGS timer (update cycles; calls = updates, one after every gradient
 * evaluation but the first).  With the SM clock in kHz (the
 * device's clockRate, which the reference uses) and the launch's ms_opt,
 * fills by the reference's formulas, a run standing for its thread,
 * metrics[8] = {ms_per_call, calls_per_thread_mean, fraction_of_thread,
 * block95, serialized (the results file's five, in its order),
 * fraction_of_kernel, avg_cycles_per_thread, avg_ms_per_thread}:
 * fraction_of_thread is the mean of cycles / whole-run cycles, block95 the
 * 95th percentile over consecutive groups of `runs_per_block` runs of their
 * summed time / ms_opt, serialized the summed time / ms_opt.  Does not
 * print. */
int zeus_cycle_metrics(const int64_t* cycles, const int64_t* counters, int64_t n,
                       int32_t which, double sm_clock_khz, float ms_opt,
                       int32_t runs_per_block, double metrics[8]);

/* ---- measurement ----------------------------------------------------
 * No counterpart in the reference: a roofline probe.  Runs `iters`
 * iterations of 8 independent FP64 FMA chains per thread on a grid sized to
 * fill every SM, and writes one double per thread to d_sink (grid*block
 * doubles, see zeus_probe_fp64_shape) so the work cannot be elided.  Flops =
 * grid * block * iters * 8 * 2; time it with events on `stream`. */
void zeus_probe_fp64_shape(int32_t* grid, int32_t* block);
int zeus_probe_fp64(int64_t iters, double* d_sink, void* stream);

#ifdef __cplusplus
}
#endif
#endif
