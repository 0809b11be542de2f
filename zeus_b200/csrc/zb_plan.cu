// Host-buffer persistent batch (zeus_batch_plan_*): the zeus_optimize of a
// batch.  A plan owns, per class, the device copies of the objective data
// and starts, the per-run outputs and the stop-early control, plus the
// batch workspace and a pinned staging buffer, all allocated once.  Each
// run copies the host inputs in, draws device-side starts (Philox or PSO)
// where the class has no host starts, launches the one persistent batch
// kernel, reduces every class (argmin + census) and gathers each class's
// census and best run into one packed buffer that comes back with one
// device-to-host copy and one stream synchronisation.
#include <cstring>
#include <new>
#include <vector>

#include "zb_internal.h"

namespace {

  // the batch kernel's class limit (zeus_batch_device)
  constexpr int kMaxPlanClasses = 16;

  // per class in the packed result: census (3 doubles of 6 int32), then
  // fval, gradient norm, status, iter, idx, then x[dim]
  constexpr int kPackHead = 3 + 5;

  struct PlanClass {
    zeus_host_class shape; // as given at creation (host pointers unused)
    int64_t instances = 1;
    size_t data_bytes = 0, idata_bytes = 0;
    double* d_data = nullptr;
    int32_t* d_idata = nullptr;
    double* d_starts = nullptr;
    double* d_fval = nullptr;
    int32_t* d_status = nullptr;
    int32_t* d_iter = nullptr;
    double* d_gnorm = nullptr;
    double* d_x = nullptr;
    int32_t* d_ctl = nullptr;
    zeus_census* d_cen = nullptr;
    // PSO (device-drawn starts with pso_iter >= 0)
    double* d_pbf = nullptr;
    double* d_gbest = nullptr;
    void* d_pso_ws = nullptr;
    size_t pso_ws_bytes = 0;
    size_t pack_off = 0; // doubles
  };

  struct GatherEntry {
    const zeus_census* cen;
    const double* fval;
    const double* gnorm;
    const int32_t* status;
    const int32_t* iter;
    const double* x;
    int dim;
    int64_t pack_off;
  };
  struct GatherTable {
    int n;
    GatherEntry e[kMaxPlanClasses];
  };

  // one block per class: the census and the best run (census best_idx)
  __global__ void
  gather_kernel(GatherTable t, double* __restrict__ pack)
  {
    const GatherEntry g = t.e[blockIdx.x];
    double* out = pack + g.pack_off;
    const zeus_census c = *g.cen;
    const int b = c.best_idx;
    if (threadIdx.x == 0) {
      int32_t* ci = reinterpret_cast<int32_t*>(out);
      ci[0] = c.actual;
      ci[1] = c.claimed;
      ci[2] = c.surrendered;
      ci[3] = c.stopped;
      ci[4] = c.best_idx;
      ci[5] = 0;
      out[3] = b >= 0 ? g.fval[b] : 37.0;
      out[4] = b >= 0 ? g.gnorm[b] : 0.0;
      out[5] = b >= 0 ? (double)g.status[b] : -1.0;
      out[6] = b >= 0 ? (double)g.iter[b] : 0.0;
      out[7] = (double)b;
    }
    for (int d = threadIdx.x; d < g.dim; d += blockDim.x)
      out[kPackHead + d] = b >= 0 ? g.x[(size_t)b * g.dim + d] : 0.0;
  }

} // namespace

struct zeus_batch_plan {
  int device = 0;
  zeus_bfgs_config cfg{};
  std::vector<PlanClass> cls;
  std::vector<zeus_batch_class> bcls;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  double* d_pack = nullptr;
  double* h_pack = nullptr;
  size_t pack_doubles = 0;
  size_t h2d_last = 0;
  std::vector<void*> allocs;

  ~zeus_batch_plan()
  {
    for (void* p : allocs)
      cudaFree(p);
    if (h_pack)
      cudaFreeHost(h_pack);
  }
  template <class T>
  int
  alloc(T** p, size_t count)
  {
    *p = nullptr;
    if (count == 0)
      return ZEUS_OK;
    void* q = nullptr;
    const int rc = zb::cuda_fail(cudaMalloc(&q, count * sizeof(T)), "plan allocation");
    if (rc == ZEUS_OK) {
      allocs.push_back(q);
      *p = static_cast<T*>(q);
    }
    return rc;
  }
};

namespace {

  int
  check_class(const zeus_host_class& c, int i)
  {
    const zeus_problem& p = c.problem;
    if (!zeus_supported(p.kind, p.dim, ZEUS_MODE_FAST, ZEUS_GRAD_ADJOINT) || c.n <= 0 ||
        c.n > 0x7fffffffLL || c.runs_per_instance < 0 ||
        (p.kind == ZEUS_OBJ_GAUSSIAN && !p.data) ||
        (p.kind == ZEUS_OBJ_POISSON_NLL && (!p.data || !p.idata || p.ndata <= 0)) ||
        (!c.starts && !(c.upper >= c.lower))) {
      zb::set_error("zeus_batch_plan: class %d is invalid or not built", i);
      return ZEUS_E_INVALID;
    }
    return ZEUS_OK;
  }

  bool
  same_shape(const zeus_host_class& a, const zeus_host_class& b)
  {
    return a.problem.kind == b.problem.kind && a.problem.dim == b.problem.dim &&
           a.problem.ndata == b.problem.ndata && a.n == b.n &&
           a.runs_per_instance == b.runs_per_instance &&
           (a.starts == nullptr) == (b.starts == nullptr) &&
           (a.starts != nullptr || a.pso_iter == b.pso_iter);
  }

  bool
  is_symmetric(const double* C, int d)
  {
    for (int i = 0; i < d; ++i)
      for (int j = i + 1; j < d; ++j)
        if (C[(size_t)i * d + j] != C[(size_t)j * d + i])
          return false;
    return true;
  }

} // namespace

extern "C" {

int
zeus_batch_plan_create(const zeus_host_class* classes, int32_t n_classes,
                       const zeus_bfgs_config* config, zeus_batch_plan** plan)
{
  if (!plan) {
    zb::set_error("zeus_batch_plan_create: plan is NULL");
    return ZEUS_E_INVALID;
  }
  *plan = nullptr;
  if (!classes || n_classes <= 0 || n_classes > kMaxPlanClasses ||
      !config) {
    zb::set_error("zeus_batch_plan_create: 1..%d classes and a config are required",
                  kMaxPlanClasses);
    return ZEUS_E_INVALID;
  }
  if (config->mode != ZEUS_MODE_FAST || config->gradient != ZEUS_GRAD_ADJOINT) {
    zb::set_error("zeus_batch_plan_create: the batch runs fast mode with adjoint "
                  "gradients");
    return ZEUS_E_INVALID;
  }
  for (int i = 0; i < n_classes; ++i)
    if (int rc = check_class(classes[i], i))
      return rc;
  auto* P = new (std::nothrow) zeus_batch_plan();
  if (!P) {
    zb::set_error("zeus_batch_plan_create: host allocation failed");
    return ZEUS_E_NOMEM;
  }
  int rc = zb::cuda_fail(cudaGetDevice(&P->device), "current device");
  P->cfg = *config;
  P->cls.resize(n_classes);
  P->bcls.resize(n_classes);
  size_t pack = 0;
  for (int i = 0; i < n_classes && rc == ZEUS_OK; ++i) {
    const zeus_host_class& c = classes[i];
    PlanClass& k = P->cls[i];
    k.shape = c;
    const int dim = c.problem.dim;
    k.instances = c.runs_per_instance > 0
                    ? (c.n + c.runs_per_instance - 1) / c.runs_per_instance
                    : 1;
    if (c.problem.kind == ZEUS_OBJ_GAUSSIAN)
      k.data_bytes = sizeof(double) * (size_t)dim * dim * k.instances;
    if (c.problem.kind == ZEUS_OBJ_POISSON_NLL) {
      k.data_bytes = sizeof(double) * (size_t)c.problem.ndata * k.instances;
      k.idata_bytes = sizeof(int32_t) * (size_t)c.problem.ndata * k.instances;
    }
    const size_t nd = (size_t)c.n * dim;
    if ((rc = P->alloc(&k.d_data, k.data_bytes / sizeof(double))) ||
        (rc = P->alloc(&k.d_idata, k.idata_bytes / sizeof(int32_t))) ||
        (rc = P->alloc(&k.d_starts, nd)) || (rc = P->alloc(&k.d_fval, (size_t)c.n)) ||
        (rc = P->alloc(&k.d_status, (size_t)c.n)) ||
        (rc = P->alloc(&k.d_iter, (size_t)c.n)) ||
        (rc = P->alloc(&k.d_gnorm, (size_t)c.n)) || (rc = P->alloc(&k.d_x, nd)) ||
        (rc = P->alloc(&k.d_ctl, 2)) || (rc = P->alloc(&k.d_cen, 1)))
      break;
    if (!c.starts && c.pso_iter >= 0) {
      k.pso_ws_bytes = zeus_pso_workspace_size(c.n, dim);
      char* w = nullptr;
      if ((rc = P->alloc(&k.d_pbf, (size_t)c.n)) ||
          (rc = P->alloc(&k.d_gbest, (size_t)dim + 1)) ||
          (rc = P->alloc(&w, k.pso_ws_bytes)))
        break;
      k.d_pso_ws = w;
    }
    zeus_batch_class& b = P->bcls[i];
    b = zeus_batch_class{};
    b.problem = c.problem;
    b.problem.data = k.d_data;
    b.problem.idata = k.d_idata;
    b.n = c.n;
    b.runs_per_instance = c.runs_per_instance;
    b.d_starts = k.d_starts;
    b.out.fval = k.d_fval;
    b.out.status = k.d_status;
    b.out.iter = k.d_iter;
    b.out.gnorm = k.d_gnorm;
    b.out.x = k.d_x;
    b.d_control = k.d_ctl;
    b.required_converged = c.required_converged;
    b.layout = c.layout;
    b.tile = c.tile;
    k.pack_off = pack;
    pack += kPackHead + (size_t)dim;
  }
  if (rc == ZEUS_OK) {
    P->ws_bytes = zeus_batch_workspace_size(P->bcls.data(), n_classes);
    char* w = nullptr;
    if ((rc = P->alloc(&w, P->ws_bytes)) == ZEUS_OK) {
      P->ws = w;
      P->pack_doubles = pack;
      if ((rc = P->alloc(&P->d_pack, pack)) == ZEUS_OK)
        rc = zb::cuda_fail(cudaMallocHost(&P->h_pack, pack * sizeof(double)),
                           "pinned staging");
    }
  }
  if (rc != ZEUS_OK) {
    delete P;
    return rc;
  }
  *plan = P;
  return ZEUS_OK;
}

int
zeus_batch_plan_run(zeus_batch_plan* P, const zeus_host_class* classes,
                    zeus_result* best, double* best_x, zeus_census* census,
                    void* stream)
{
  if (!P || !classes || !best) {
    zb::set_error("zeus_batch_plan_run: plan, classes and best are required");
    return ZEUS_E_INVALID;
  }
  const int nc = (int)P->cls.size();
  for (int i = 0; i < nc; ++i) {
    best[i] = zeus_result{-1, -1, 37.0, 0.0, 0, 0};
    if (census)
      census[i] = zeus_census{0, 0, 0, 0, -1, 0};
    if (!same_shape(classes[i], P->cls[i].shape) || check_class(classes[i], i)) {
      zb::set_error("zeus_batch_plan_run: class %d differs from the plan's", i);
      return ZEUS_E_INVALID;
    }
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev != P->device) {
    zb::set_error("zeus_batch_plan_run: the plan belongs to device %d", P->device);
    return ZEUS_E_INVALID;
  }
  cudaStream_t st = (cudaStream_t)stream;
  auto fail = [&](int code) {
    for (int i = 0; i < nc; ++i)
      best[i].status = code == ZEUS_E_NOMEM ? ZEUS_STATUS_NOMEM : ZEUS_STATUS_KERNEL;
    return code;
  };
  size_t h2d = 0;
  int rc = ZEUS_OK;
  for (int i = 0; i < nc; ++i) {
    const zeus_host_class& c = classes[i];
    PlanClass& k = P->cls[i];
    zeus_batch_class& b = P->bcls[i];
    const int dim = c.problem.dim;
    if (k.data_bytes &&
        (rc = zb::cuda_fail(cudaMemcpyAsync(k.d_data, c.problem.data, k.data_bytes,
                                            cudaMemcpyHostToDevice, st),
                            "H2D objective data")))
      return fail(rc);
    if (k.idata_bytes &&
        (rc = zb::cuda_fail(cudaMemcpyAsync(k.d_idata, c.problem.idata, k.idata_bytes,
                                            cudaMemcpyHostToDevice, st),
                            "H2D counts")))
      return fail(rc);
    h2d += k.data_bytes + k.idata_bytes;
    b.problem.flags = c.problem.flags;
    if (c.problem.kind == ZEUS_OBJ_GAUSSIAN) {
      bool sym = true;
      for (int64_t q = 0; q < k.instances && sym; ++q)
        sym = is_symmetric(c.problem.data + (size_t)q * dim * dim, dim);
      b.problem.flags = sym ? ZEUS_PROBLEM_SYMMETRIC : 0;
    }
    b.required_converged = c.required_converged;
    zeus_problem dp = b.problem;
    if (c.starts) {
      const size_t bytes = sizeof(double) * (size_t)c.n * dim;
      if ((rc = zb::cuda_fail(cudaMemcpyAsync(k.d_starts, c.starts, bytes,
                                              cudaMemcpyHostToDevice, st),
                              "H2D starts")))
        return fail(rc);
      h2d += bytes;
    } else if (c.pso_iter >= 0) {
      if (c.runs_per_instance > 0 && k.instances > 1) {
        zb::set_error("zeus_batch_plan_run: class %d: PSO over several data "
                      "instances is not built; pass host starts",
                      i);
        return fail(ZEUS_E_UNSUPPORTED);
      }
      if ((rc = zeus_pso_device(&dp, c.seed, c.n, c.lower, c.upper, c.pso_iter, 0.5,
                                1.2, 1.5, k.d_starts, k.d_pbf, k.d_gbest, k.d_pso_ws,
                                k.pso_ws_bytes, st)))
        return fail(rc);
    } else if ((rc = zeus_starts_uniform(c.seed, c.n, dim, c.lower, c.upper,
                                         k.d_starts, st))) {
      return fail(rc);
    }
    if ((rc = zb::cuda_fail(cudaMemsetAsync(k.d_ctl, 0, 2 * sizeof(int32_t), st),
                            "control reset")))
      return fail(rc);
  }
  if ((rc = zeus_batch_device(P->bcls.data(), nc, &P->cfg, P->ws, P->ws_bytes, st)))
    return fail(rc);
  GatherTable gt{};
  gt.n = nc;
  int maxdim = 32;
  for (int i = 0; i < nc; ++i) {
    const PlanClass& k = P->cls[i];
    const int dim = k.shape.problem.dim;
    std::vector<double> km;
    if (k.shape.problem.kind == ZEUS_OBJ_ROSENBROCK && dim <= 256)
      km.assign(dim, 1.0);
    if ((rc = zeus_census_device(k.d_fval, k.d_status, k.d_x, k.shape.n, dim,
                                 km.empty() ? nullptr : km.data(), k.d_cen, st)))
      return fail(rc);
    gt.e[i] = GatherEntry{k.d_cen, k.d_fval, k.d_gnorm, k.d_status, k.d_iter,
                          k.d_x,   dim,      (int64_t)k.pack_off};
    maxdim = dim > maxdim ? dim : maxdim;
  }
  gather_kernel<<<nc, maxdim < 256 ? 128 : 256, 0, st>>>(gt, P->d_pack);
  if ((rc = zb::cuda_fail(cudaGetLastError(), "result gather launch")) ||
      (rc = zb::cuda_fail(cudaMemcpyAsync(P->h_pack, P->d_pack,
                                          P->pack_doubles * sizeof(double),
                                          cudaMemcpyDeviceToHost, st),
                          "D2H results")) ||
      (rc = zb::cuda_fail(cudaStreamSynchronize(st), "batch run")))
    return fail(rc);
  P->h2d_last = h2d;
  size_t xoff = 0;
  for (int i = 0; i < nc; ++i) {
    const PlanClass& k = P->cls[i];
    const double* o = P->h_pack + k.pack_off;
    zeus_census cz;
    std::memcpy(&cz, o, sizeof cz);
    if (census)
      census[i] = cz;
    best[i].fval = o[3];
    best[i].gradient_norm = o[4];
    best[i].status = (int32_t)o[5];
    best[i].iter = (int32_t)o[6];
    best[i].idx = (int32_t)o[7];
    const int dim = k.shape.problem.dim;
    if (best_x)
      std::memcpy(best_x + xoff, o + kPackHead, sizeof(double) * dim);
    xoff += dim;
  }
  return ZEUS_OK;
}

int
zeus_batch_plan_traffic(const zeus_batch_plan* P, size_t* h2d_bytes,
                        size_t* d2h_bytes)
{
  if (!P) {
    zb::set_error("zeus_batch_plan_traffic: plan is NULL");
    return ZEUS_E_INVALID;
  }
  if (h2d_bytes)
    *h2d_bytes = P->h2d_last;
  if (d2h_bytes)
    *d2h_bytes = P->pack_doubles * sizeof(double);
  return ZEUS_OK;
}

int
zeus_batch_plan_destroy(zeus_batch_plan* P)
{
  delete P;
  return ZEUS_OK;
}

} // extern "C"
