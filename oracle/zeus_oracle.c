/*
 * zeus_oracle.c -- CPU restatement of the reference hot path (PSO seeding,
 * sequential FP64 BFGS with forward-mode dual gradients).  Test
 * infrastructure only; see zeus_oracle.h.  Compiled with -ffp-contract=off:
 * every expression below keeps the reference's evaluation order, including
 * the implicit double -> DualNumber conversions, so results are bit-identical
 * to the reference's host build for the same inputs.
 */
#include "zeus_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ dual */
/* DualNumber and its operators: include/duals.cuh:14-134. */
typedef struct {
  double r, d;
} dual;

static inline dual
D(double r, double d)
{
  dual z = {r, d};
  return z;
}
static inline dual
d_add(dual a, dual b) /* duals.cuh:76-80 */
{
  return D(a.r + b.r, a.d + b.d);
}
static inline dual
d_sub(dual a, dual b) /* duals.cuh:82-86 */
{
  return D(a.r - b.r, a.d - b.d);
}
static inline dual
d_mul(dual a, dual b) /* duals.cuh:88-92 */
{
  return D(a.r * b.r, a.d * b.r + a.r * b.d);
}
static inline dual
d_div(dual a, dual b) /* duals.cuh:94-100 */
{
  double denom = b.r * b.r;
  return D(a.r / b.r, (a.d * b.r - a.r * b.d) / denom);
}
static inline dual
d_lsub(double l, dual b) /* double - dual, duals.cuh:102-106 */
{
  return D(l - b.r, -b.d);
}
static inline dual
d_lmul(double l, dual b) /* double * dual, duals.cuh:108-112 */
{
  return D(l * b.r, l * b.d);
}
static inline dual
d_cos(dual x) /* duals.cuh:158-162 */
{
  return D(cos(x.r), -x.d * sin(x.r));
}
static inline dual
d_exp(dual x) /* duals.cuh:165-170 */
{
  double ex = exp(x.r);
  return D(ex, x.d * ex);
}
static inline dual
d_sqrt(dual x) /* duals.cuh:173-178 */
{
  double sr = sqrt(x.r);
  return D(sr, x.d / (2.0 * sr));
}
static inline dual
d_log(dual x) /* duals.cuh:190-195 */
{
  return D(log(x.r), x.d / x.r);
}
static inline dual
d_pow(dual base, dual ex) /* duals.cuh:198-208 */
{
  const double br = base.r, er = ex.r;
  const double pr = pow(br, er);
  const double pd = pr * (ex.d * log(br) + er * base.d / br);
  return D(pr, pd);
}
static inline dual
d_powd(dual base, double e) /* duals.cuh:211-220 */
{
  const double br = base.r;
  const double pr = pow(br, e);
  if (br == 0.0)
    return D(pr, e * pow(br, e - 1.0) * base.d);
  return D(pr, e * pr / br * base.d);
}
static inline dual
d_lgamma(dual x) /* duals.cuh:233-239 */
{
  const double lr = lgamma(x.r);
  const double dg = zor_digamma(x.r);
  return D(lr, x.d * dg);
}

/* src/duals.cu:10-39 */
double
zor_digamma(double x)
{
  const double pi = 3.14159265358979323846;
  if (x <= 0.0 && x == floor(x))
    return INFINITY;
  if (x < 0.5)
    return zor_digamma(1.0 - x) - pi / tan(pi * x);
  double acc = 0.0;
  while (x < 8.0) {
    acc -= 1.0 / x;
    x += 1.0;
  }
  const double inv = 1.0 / x;
  const double inv2 = inv * inv;
  const double s =
    inv2 *
    (-1.0 / 12.0 +
     inv2 * (1.0 / 120.0 +
             inv2 * (-1.0 / 252.0 +
                     inv2 * (1.0 / 240.0 +
                             inv2 * (-1.0 / 132.0 + inv2 * (691.0 / 32760.0))))));
  return acc + log(x) - 0.5 * inv + s;
}

static const double TWO_PI = 2.0 * 3.14159265358979323846;

/* ------------------------------------------------------------ objectives */
/* double paths: examples/rosenbrock.hpp:19-30, rastrigin.hpp:18-24,
 * ackley.hpp:26-39, gaussian.hpp:19-33, LogLikelihood.h:29-58 */
double
zor_value(const zor_objective* o, const double* x)
{
  const int n = o->dim;
  switch (o->kind) {
    case ZOR_ROSENBROCK: {
      double sum = 0.0;
      for (int i = 0; i < n - 1; ++i) {
        double t1 = 1.0 - x[i];
        double t2 = x[i + 1] - x[i] * x[i];
        sum += t1 * t1 + 100.0 * t2 * t2;
      }
      return sum;
    }
    case ZOR_RASTRIGIN: {
      double sum = 10.0 * n;
      for (int i = 0; i < n; ++i)
        sum += x[i] * x[i] - 10.0 * cos(TWO_PI * x[i]);
      return sum;
    }
    case ZOR_ACKLEY: {
      double sum_sq = 0.0, sum_cos = 0.0;
      for (int i = 0; i < n; ++i) {
        sum_sq += x[i] * x[i];
        sum_cos += cos(TWO_PI * x[i]);
      }
      double term1 = -20.0 * exp(-0.2 * sqrt(sum_sq / n));
      double term2 = -exp(sum_cos / n);
      return term1 + term2 + 20.0 + exp(1.0);
    }
    case ZOR_GAUSSIAN: {
      const double* C = o->data;
      double q = 0.0;
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
          q += x[i] * C[i * n + j] * x[j];
      return 0.5 * q;
    }
    case ZOR_POISSON_NLL: {
      const double a = x[0], b = x[1], c = x[2], d = x[3];
      double nll = 0.0;
      for (int i = 0; i < o->ndata; ++i) {
        double xc = o->data[i];
        int ki = o->idata[i];
        double mean = a * pow(1.0 - xc, b) / pow(xc, c + d * log(xc));
        double log_p = (double)ki * log(mean) - mean - lgamma((double)ki + 1.0);
        nll -= log_p;
      }
      return nll;
    }
  }
  return NAN;
}

/* DualNumber paths of the same objectives (T = dual::DualNumber). */
static dual
value_dual(const zor_objective* o, const dual* x)
{
  const int n = o->dim;
  switch (o->kind) {
    case ZOR_ROSENBROCK: { /* rosenbrock.hpp:6-17 */
      dual sum = D(0.0, 0.0);
      for (int i = 0; i < n - 1; ++i) {
        dual t1 = d_sub(D(1.0, 0.0), x[i]);
        dual t2 = d_sub(x[i + 1], d_mul(x[i], x[i]));
        sum = d_add(d_add(sum, d_mul(t1, t1)),
                    d_mul(d_mul(D(100.0, 0.0), t2), t2));
      }
      return sum;
    }
    case ZOR_RASTRIGIN: { /* rastrigin.hpp:6-16 */
      dual sum = D(10.0 * n, 0.0);
      for (int i = 0; i < n; ++i) {
        dual arg = d_mul(x[i], D(TWO_PI, 0.0));
        sum = d_add(sum, d_sub(d_mul(x[i], x[i]),
                               d_mul(D(10.0, 0.0), d_cos(arg))));
      }
      return sum;
    }
    case ZOR_ACKLEY: { /* ackley.hpp:10-24 */
      dual sum_sq = D(0.0, 0.0), sum_cos = D(0.0, 0.0);
      for (int i = 0; i < n; ++i) {
        sum_sq = d_add(sum_sq, d_powd(x[i], 2.0));
        sum_cos = d_add(sum_cos, d_cos(d_lmul(TWO_PI, x[i])));
      }
      dual dimv = D((double)n, 0.0);
      dual term1 = d_mul(D(-20.0, 0.0),
                         d_exp(d_lmul(-0.2, d_sqrt(d_div(sum_sq, dimv)))));
      dual term2 = d_sub(D(0.0, 0.0), d_exp(d_div(sum_cos, dimv)));
      return d_add(d_add(d_add(term1, term2), D(20.0, 0.0)),
                   d_exp(D(1.0, 0.0)));
    }
    case ZOR_GAUSSIAN: { /* gaussian.hpp:19-33 */
      const double* C = o->data;
      dual q = D(0.0, 0.0);
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
          q = d_add(q, d_mul(d_mul(x[i], D(C[i * n + j], 0.0)), x[j]));
      return d_mul(D(0.5, 0.0), q);
    }
    case ZOR_POISSON_NLL: { /* LogLikelihood.h:29-58 */
      const dual a = x[0], b = x[1], c = x[2], d = x[3];
      dual nll = D(0.0, 0.0);
      for (int i = 0; i < o->ndata; ++i) {
        dual xc = D(o->data[i], 0.0);
        int ki = o->idata[i];
        dual mean = d_div(d_mul(a, d_pow(d_sub(D(1.0, 0.0), xc), b)),
                          d_pow(xc, d_add(c, d_mul(d, d_log(xc)))));
        dual log_p = d_sub(d_sub(d_mul(D((double)ki, 0.0), d_log(mean)), mean),
                           d_lgamma(d_add(D((double)ki, 0.0), D(1.0, 0.0))));
        nll = d_sub(nll, log_p);
      }
      return nll;
    }
  }
  return D(NAN, NAN);
}

/* duals.cuh:241-266: one forward pass per coordinate. */
double
zor_value_grad_dual(const zor_objective* o, const double* x, double* grad)
{
  dual xd[ZOR_MAX_DIM];
  const int n = o->dim;
  for (int i = 0; i < n; ++i)
    xd[i] = D(x[i], 0.0);
  for (int i = 0; i < n; ++i) {
    xd[i].d = 1.0;
    grad[i] = value_dual(o, xd).d;
    xd[i].d = 0.0;
  }
  return zor_value(o, x);
}

/* Closed-form gradients: the mathematics the product's adjoint kernels
 * implement.  Checked against zor_value_grad_dual and central differences. */
double
zor_value_grad_analytic(const zor_objective* o, const double* x, double* g)
{
  const int n = o->dim;
  switch (o->kind) {
    case ZOR_ROSENBROCK:
      for (int i = 0; i < n; ++i) {
        double gi = 0.0;
        if (i < n - 1)
          gi += -2.0 * (1.0 - x[i]) - 400.0 * x[i] * (x[i + 1] - x[i] * x[i]);
        if (i > 0)
          gi += 200.0 * (x[i] - x[i - 1] * x[i - 1]);
        g[i] = gi;
      }
      break;
    case ZOR_RASTRIGIN:
      for (int i = 0; i < n; ++i)
        g[i] = 2.0 * x[i] + 10.0 * TWO_PI * sin(TWO_PI * x[i]);
      break;
    case ZOR_ACKLEY: {
      double s = 0.0, c = 0.0;
      for (int i = 0; i < n; ++i) {
        s += x[i] * x[i];
        c += cos(TWO_PI * x[i]);
      }
      double r = sqrt(s / n);
      double a = 4.0 * exp(-0.2 * r) / (n * r);
      double b = TWO_PI * exp(c / n) / n;
      for (int i = 0; i < n; ++i)
        g[i] = a * x[i] + b * sin(TWO_PI * x[i]);
      break;
    }
    case ZOR_GAUSSIAN: {
      const double* C = o->data;
      for (int i = 0; i < n; ++i) {
        double acc = 0.0;
        for (int j = 0; j < n; ++j)
          acc += 0.5 * (C[i * n + j] + C[j * n + i]) * x[j];
        g[i] = acc;
      }
      break;
    }
    case ZOR_POISSON_NLL: {
      double ga = 0, gb = 0, gc = 0, gd = 0;
      for (int i = 0; i < o->ndata; ++i) {
        double xc = o->data[i], lx = log(xc);
        double lam = x[0] * pow(1.0 - xc, x[1]) / pow(xc, x[2] + x[3] * lx);
        double w = lam - (double)o->idata[i];
        ga += w / x[0];
        gb += w * log(1.0 - xc);
        gc -= w * lx;
        gd -= w * lx * lx;
      }
      g[0] = ga;
      g[1] = gb;
      g[2] = gc;
      g[3] = gd;
      break;
    }
  }
  return zor_value(o, x);
}

/* ----------------------------------------------------------- BFGS pieces */
/* utils.cuh:111-119 */
static double
dot(const double* a, const double* b, int n)
{
  double sum = 0.0;
  for (int i = 0; i < n; ++i)
    sum += a[i] * b[i];
  return sum;
}
/* utils.cuh:137-146 */
static double
grad_norm(const double* g, int n)
{
  double s = 0.0;
  for (int i = 0; i < n; ++i)
    s += g[i] * g[i];
  return sqrt(s);
}

/* utils.cuh:376-412: alpha0 = 1, halve up to 20 times, accept on Armijo
 * (c1 = 0.1) AND strict decrease; never returns 0 (2^-20 after 20 misses). */
double
zor_line_search(const zor_objective* o, double f0, const double* x,
                const double* p, const double* g)
{
  const double c1 = 0.1;
  double alpha = 1.0;
  double ddir = dot(g, p, o->dim);
  double xt[ZOR_MAX_DIM];
  for (int i = 0; i < 20; i++) {
    for (int j = 0; j < o->dim; j++)
      xt[j] = x[j] + alpha * p[j];
    double f1 = zor_value(o, xt);
    if (f1 <= f0 + c1 * alpha * ddir && f1 < f0)
      break;
    alpha *= 0.5;
  }
  return alpha;
}

/* utils.cuh:245-287: H <- (I - rho s y^T) H (I - rho y s^T) + rho s s^T,
 * skipped when |s.y| < 1e-14.  The reference recomputes the inner m-sum
 * T[k][j] = sum_m H[k][m] (delta_mj - rho y_m s_j) for every i; it depends on
 * (k, j) only, so computing it once per (k, j) in the same m order gives the
 * same bits. */
void
zor_bfgs_update(int n, double* H, const double* s, const double* y,
                double sTy)
{
  if (fabs(sTy) < 1e-14)
    return;
  double rho = 1.0 / sTy;
  double* T = (double*)malloc(sizeof(double) * (size_t)n * n);
  double* Hn = (double*)malloc(sizeof(double) * (size_t)n * n);
  for (int k = 0; k < n; k++)
    for (int j = 0; j < n; j++) {
      double inner = 0.0;
      for (int m = 0; m < n; m++) {
        double B_mj = ((m == j) ? 1.0 : 0.0) - rho * y[m] * s[j];
        inner += H[k * n + m] * B_mj;
      }
      T[k * n + j] = inner;
    }
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      double sum = 0.0;
      for (int k = 0; k < n; k++) {
        double A_ik = ((i == k) ? 1.0 : 0.0) - rho * s[i] * y[k];
        sum += A_ik * T[k * n + j];
      }
      Hn[i * n + j] = sum + rho * s[i] * s[j];
    }
  memcpy(H, Hn, sizeof(double) * (size_t)n * n);
  free(T);
  free(Hn);
}

/* bfgs_sequential.cuh:46-234 for one run; ctx = {stopFlag, convergedCount}. */
static void
bfgs_one(const zor_objective* o, int idx, int N, const double* start,
         int max_iter, int required, double tol, int* ctx, double* r_fval,
         int* r_status, int* r_iter, double* r_gnorm, double* r_x,
         double* traj_x, double* traj_f, double* traj_g,
         signed char* traj_status)
{
  const int n = o->dim;
  double x[ZOR_MAX_DIM] = {0}, xn[ZOR_MAX_DIM], g[ZOR_MAX_DIM], gn[ZOR_MAX_DIM],
    p[ZOR_MAX_DIM], s[ZOR_MAX_DIM], y[ZOR_MAX_DIM];
  double* H = (double*)calloc((size_t)n * n, sizeof(double));
  for (int i = 0; i < n; ++i)
    H[i * n + i] = 1.0;
  for (int d = 0; d < n; ++d) {
    x[d] = start[d];
    g[d] = 0.0;
  }
  const int traj = traj_x && traj_f && traj_g && traj_status;
  double f0 = zor_value(o, x);
  double best = f0;
  zor_value_grad_dual(o, x, g);

  int status = -1, it_out = 0, done = 0, iter;
  double fval_out = 333777.0, gn_out = 69.0;
  double xo[ZOR_MAX_DIM];
  for (int d = 0; d < n; ++d)
    xo[d] = 7.0;

  for (iter = 0; iter < max_iter; ++iter) {
    if (traj) {
      for (int d = 0; d < n; ++d)
        traj_x[(size_t)iter * n * N + (size_t)d * N + idx] = x[d];
      traj_f[(size_t)iter * N + idx] = best;
      traj_g[(size_t)iter * N + idx] = grad_norm(g, n);
      traj_status[(size_t)iter * N + idx] = -1;
    }
    if (ctx[0] != 0) { /* bfgs_common.cuh:115-141, status 2 */
      status = 2;
      fval_out = zor_value(o, x);
      gn_out = grad_norm(g, n);
      it_out = iter;
      memcpy(xo, x, sizeof(double) * n);
      if (traj)
        traj_status[(size_t)iter * N + idx] = 2;
      done = 1;
      break;
    }
    for (int i = 0; i < n; i++) { /* p = -H g, utils.cuh:148-161 */
      double sum = 0.0;
      for (int j = 0; j < n; j++)
        sum += H[i * n + j] * g[j];
      p[i] = -sum;
    }
    double alpha = zor_line_search(o, best, x, p, g);
    for (int i = 0; i < n; ++i) {
      xn[i] = x[i] + alpha * p[i];
      s[i] = xn[i] - x[i];
    }
    double fnew = zor_value(o, xn);
    zor_value_grad_dual(o, xn, gn);
    for (int i = 0; i < n; ++i)
      y[i] = gn[i] - g[i];
    double sy = dot(s, y, n);
    zor_bfgs_update(n, H, s, y, sy);
    if (fnew < best) {
      best = fnew;
      memcpy(x, xn, sizeof(double) * n);
      memcpy(g, gn, sizeof(double) * n);
    }
    double gnrm = grad_norm(g, n);
    if (!isfinite(gnrm) || !isfinite(fnew)) { /* bfgs_common.cuh:145-164 */
      status = 5;
      fval_out = fnew;
      gn_out = gnrm;
      it_out = iter;
      memcpy(xo, x, sizeof(double) * n);
      if (traj)
        traj_status[(size_t)iter * N + idx] = 5;
      done = 1;
      break;
    }
    if (gnrm < tol) { /* bfgs_common.cuh:170-208 */
      int old = ctx[1]++;
      status = 1;
      fval_out = zor_value(o, x);
      gn_out = gnrm;
      it_out = iter;
      memcpy(xo, x, sizeof(double) * n);
      if (traj)
        traj_status[(size_t)iter * N + idx] = 1;
      if (old + 1 == required)
        ctx[0] = 1;
      done = 1;
      break;
    }
  }
  if (!done && iter == max_iter) { /* bfgs_common.cuh:213-238, status 0 */
    status = 0;
    fval_out = zor_value(o, x);
    gn_out = grad_norm(g, n);
    it_out = iter;
    memcpy(xo, x, sizeof(double) * n);
    if (traj && max_iter > 0)
      traj_status[(size_t)(max_iter - 1) * N + idx] = 0;
  }
  if (r_fval)
    r_fval[idx] = fval_out;
  if (r_status)
    r_status[idx] = status;
  if (r_iter)
    r_iter[idx] = it_out;
  if (r_gnorm)
    r_gnorm[idx] = gn_out;
  if (r_x)
    memcpy(r_x + (size_t)idx * n, xo, sizeof(double) * n);
  free(H);
}

int
zor_bfgs(int kind, int dim, const double* data, const int* idata, int ndata,
         const double* starts, int n, double lower, double upper,
         int max_iter, int required, double tol, double* fval, int* status,
         int* iter, double* gnorm, double* x_out, double* traj_x,
         double* traj_f, double* traj_g, signed char* traj_status,
         int nthreads)
{
  (void)lower;
  (void)upper;
  (void)nthreads;
  if (dim < 1 || dim > ZOR_MAX_DIM || n < 0 || !starts)
    return -1;
  zor_objective o = {kind, dim, data, idata, ndata};
  int ctx[2] = {0, 0};
  for (int i = 0; i < n; ++i)
    bfgs_one(&o, i, n, starts + (size_t)i * dim, max_iter, required, tol, ctx,
             fval, status, iter, gnorm, x_out, traj_x, traj_f, traj_g,
             traj_status);
  return 0;
}

/* ----------------------------------------------------------------- RNG */
static inline void
mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo)
{
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

/* Philox4x32 with 10 rounds: multipliers 0xD2511F53, 0xCD9E8D57 and Weyl
 * key increments 0x9E3779B9, 0xBB67AE85 as published by Salmon et al. */
void
zor_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2],
                  uint32_t out[4])
{
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c0, &hi0, &lo0);
    mulhilo32(0xCD9E8D57u, c2, &hi1, &lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* Counter = (run lo, index/2, tag, run hi), key = seed; the pair of words
 * (2*(index&1), 2*(index&1)+1) gives 64 bits, of which the top 53 make the
 * mantissa of a double in [0, 1). */
double
zor_uniform(uint64_t seed, uint32_t tag, uint64_t run, uint32_t index)
{
  uint32_t ctr[4] = {(uint32_t)run, index >> 1, tag, (uint32_t)(run >> 32)};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t out[4];
  zor_philox4x32_10(ctr, key, out);
  int w = (int)(index & 1u) * 2;
  uint64_t bits = ((uint64_t)out[w] << 32) | out[w + 1];
  return (double)(bits >> 11) * (1.0 / 9007199254740992.0);
}

void
zor_uniform_starts(uint64_t seed, int n, int dim, double lower, double upper,
                   double* out)
{
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < dim; ++d)
      out[(size_t)i * dim + d] =
        lower + (upper - lower) * zor_uniform(seed, 1u, (uint64_t)i, (uint32_t)d);
}

/* --------------------------------------------------------------- Sobol' */
/* Sobol' (1967) points with the Bratley-Fox recurrence (ACM TOMS 14 (1988)
 * 88-100): for the primitive polynomial x^s + a_1 x^(s-1) + ... + a_(s-1) x
 * + 1 and m_1..m_s, m_k = 2 a_1 m_(k-1) ^ 4 a_2 m_(k-2) ^ ... ^
 * 2^(s-1) a_(s-1) m_(k-s+1) ^ 2^s m_(k-s) ^ m_(k-s), and v_k = m_k / 2^k
 * (here as 32-bit fractions).  Dimension 0 is van der Corput (v_k = 2^-k). */
void
zor_sobol_directions(int ndim, const uint32_t* poly, const uint32_t* minit,
                     int maxdeg, uint32_t* dirs)
{
  for (int d = 0; d < ndim; ++d) {
    uint32_t* v = dirs + (size_t)d * 32;
    if (d == 0) {
      for (int k = 1; k <= 32; ++k)
        v[k - 1] = (uint32_t)1u << (32 - k);
      continue;
    }
    int s = 0;
    while ((poly[d] >> (s + 1)) != 0u)
      ++s;
    uint64_t m[33];
    for (int k = 1; k <= s; ++k)
      m[k] = minit[(size_t)d * maxdeg + (k - 1)];
    for (int k = s + 1; k <= 32; ++k) {
      uint64_t x = ((uint64_t)1 << s) * m[k - s] ^ m[k - s];
      for (int i = 1; i < s; ++i) {
        const uint64_t a = (poly[d] >> (s - i)) & 1u;
        x ^= a * (((uint64_t)1 << i) * m[k - i]);
      }
      m[k] = x;
    }
    for (int k = 1; k <= 32; ++k)
      v[k - 1] = (uint32_t)(m[k] << (32 - k));
  }
}

/* Order of x modulo p over GF(2) by repeated multiplication (p of degree s,
 * constant term 1); p is primitive iff the order is 2^s - 1. */
static int
sobol_primitive(uint32_t p, int s)
{
  const uint32_t top = (uint32_t)1u << s, full = top - 1u;
  uint32_t r = 1u;
  for (uint32_t k = 1; k <= full; ++k) {
    r <<= 1;
    if (r & top)
      r ^= p;
    if (r == 1u)
      return k == full;
  }
  return 0;
}

static uint64_t
sobol_splitmix(uint64_t* st)
{
  uint64_t z = (*st += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* The product's parameters: polynomials in order of degree then value;
 * m_k = (bits 32..63 of the k-th splitmix64 output of the stream seeded
 * 0x5A17B01D + 0x100000001B3 * d) mod 2^k, forced odd. */
int
zor_sobol_params(int ndim, uint32_t* poly, uint32_t* minit, int maxdeg)
{
  int d = 1;
  if (ndim > 0)
    poly[0] = 1u;
  for (int s = 1; d < ndim; ++s) {
    if (s > maxdeg || s > 30)
      return -1;
    for (uint32_t p = ((uint32_t)1u << s) + 1u; d < ndim && p < ((uint32_t)2u << s);
         p += 2u) {
      if (!sobol_primitive(p, s))
        continue;
      poly[d] = p;
      uint64_t st = 0x5A17B01Dull + 0x100000001B3ull * (uint64_t)d;
      for (int k = 1; k <= s; ++k)
        minit[(size_t)d * maxdeg + (k - 1)] =
          ((uint32_t)(sobol_splitmix(&st) >> 32) & (((uint32_t)1u << k) - 1u)) | 1u;
      ++d;
    }
  }
  return 0;
}

/* Point `run` (low 32 bits, natural order), coordinate d, XOR-shifted by
 * word 0 of Philox(counter (d, 0, 4, 0), key seed), at its cell midpoint. */
double
zor_sobol01(const uint32_t* dirs, uint64_t seed, uint64_t run, uint32_t d)
{
  uint32_t ctr[4] = {d, 0u, 4u, 0u};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t sh[4];
  zor_philox4x32_10(ctr, key, sh);
  uint32_t x = sh[0];
  const uint32_t n = (uint32_t)run;
  for (int k = 0; k < 32; ++k)
    if ((n >> k) & 1u)
      x ^= dirs[(size_t)d * 32 + k];
  return ((double)x + 0.5) / 4294967296.0;
}

void
zor_starts(uint64_t seed, const uint32_t* sobol, int n, int dim, double lower,
           double upper, double* out)
{
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < dim; ++d) {
      const double u = sobol ? zor_sobol01(sobol, seed, (uint64_t)i, (uint32_t)d)
                             : zor_uniform(seed, 1u, (uint64_t)i, (uint32_t)d);
      out[(size_t)i * dim + d] = lower + (upper - lower) * u;
    }
}

/* ----------------------------------------------------------------- PSO */
/* pso.cuh:104-119 */
void
zor_pso_step(int dim, double w, double c1, double c2, const double* r1,
             const double* r2, double* x, double* v, const double* pb,
             const double* gb)
{
  for (int d = 0; d < dim; ++d) {
    double nv = w * v[d] + c1 * r1[d] * (pb[d] - x[d]) + c2 * r2[d] * (gb[d] - x[d]);
    v[d] = nv;
    x[d] = x[d] + nv;
  }
}

/* pso.cuh:17-69 (init) and 72-155 (iterations), synchronous gBest. */
int
zor_pso(const zor_objective* o, uint64_t seed, int n, double lower,
        double upper, int iters, double w, double c1, double c2,
        double* pbx, double* pbf, double* gbx, double* gbf)
{
  return zor_pso_sobol(o, seed, NULL, n, lower, upper, iters, w, c1, c2, pbx,
                       pbf, gbx, gbf);
}

int
zor_pso_sobol(const zor_objective* o, uint64_t seed, const uint32_t* sobol,
              int n, double lower, double upper, int iters, double w,
              double c1, double c2, double* pbx, double* pbf, double* gbx,
              double* gbf)
{
  const int dim = o->dim;
  double* X = (double*)malloc(sizeof(double) * (size_t)n * dim);
  double* V = (double*)malloc(sizeof(double) * (size_t)n * dim);
  const double vr = (upper - lower) * 0.1;
  double gbest = INFINITY;
  int gidx = -1;
  for (int i = 0; i < n; ++i) {
    for (int d = 0; d < dim; ++d) {
      double ux = sobol ? zor_sobol01(sobol, seed, (uint64_t)i, (uint32_t)d)
                        : zor_uniform(seed, 2u, (uint64_t)i, (uint32_t)d);
      double uv = zor_uniform(seed, 3u, (uint64_t)i, (uint32_t)d);
      X[(size_t)i * dim + d] = lower + (upper - lower) * ux;
      V[(size_t)i * dim + d] = -vr + (vr - -vr) * uv;
      pbx[(size_t)i * dim + d] = X[(size_t)i * dim + d];
    }
    double f = zor_value(o, X + (size_t)i * dim);
    pbf[i] = f;
    if (f < gbest) {
      gbest = f;
      gidx = i;
    }
  }
  double gb[ZOR_MAX_DIM];
  for (int d = 0; d < dim; ++d)
    gb[d] = gidx >= 0 ? pbx[(size_t)gidx * dim + d] : 0.0;
  for (int t = 1; t <= iters; ++t) {
    double r1[ZOR_MAX_DIM], r2[ZOR_MAX_DIM];
    double nbest = gbest;
    int nidx = -1;
    for (int i = 0; i < n; ++i) {
      for (int d = 0; d < dim; ++d) {
        r1[d] = zor_uniform(seed, 16u + (uint32_t)t, (uint64_t)i, 2u * d);
        r2[d] = zor_uniform(seed, 16u + (uint32_t)t, (uint64_t)i, 2u * d + 1u);
      }
      double* xi = X + (size_t)i * dim;
      zor_pso_step(dim, w, c1, c2, r1, r2, xi, V + (size_t)i * dim,
                   pbx + (size_t)i * dim, gb);
      double f = zor_value(o, xi);
      if (f < pbf[i]) {
        pbf[i] = f;
        memcpy(pbx + (size_t)i * dim, xi, sizeof(double) * dim);
      }
      if (f < nbest) {
        nbest = f;
        nidx = i;
      }
    }
    if (nidx >= 0) {
      gbest = nbest;
      memcpy(gb, X + (size_t)nidx * dim, sizeof(double) * dim);
    }
  }
  if (gbx)
    memcpy(gbx, gb, sizeof(double) * dim);
  if (gbf)
    *gbf = gbest;
  free(X);
  free(V);
  return 0;
}
