// Maps a runtime (kind, dim) to a built-in objective functor and calls
// fn(functor).  The dimension sets are the ones the library is built for;
// anything else is ZEUS_E_UNSUPPORTED.
#pragma once

#include "zb_internal.h"
#include "zb_objectives.cuh"

namespace zb {

#define ZB_ROSENBROCK_DIMS(X) X(2) X(4) X(8) X(10) X(16) X(32) X(64) X(128) X(256)
#define ZB_RASTRIGIN_DIMS(X) X(2) X(10) X(16)
#define ZB_ACKLEY_DIMS(X) X(2) X(10) X(30)
#define ZB_GAUSSIAN_DIMS(X) X(2) X(8) X(32) X(150)

  template <class Fn>
  int
  visit_objective(const Objective& o, Fn&& fn)
  {
    switch (o.kind) {
      case ZEUS_OBJ_ROSENBROCK:
        switch (o.dim) {
#define ZB_CASE(D)                                                             \
  case D:                                                                      \
    return fn(zeus::Rosenbrock<D>{});
          ZB_ROSENBROCK_DIMS(ZB_CASE)
#undef ZB_CASE
        }
        break;
      case ZEUS_OBJ_RASTRIGIN:
        switch (o.dim) {
#define ZB_CASE(D)                                                             \
  case D:                                                                      \
    return fn(zeus::Rastrigin<D>{});
          ZB_RASTRIGIN_DIMS(ZB_CASE)
#undef ZB_CASE
        }
        break;
      case ZEUS_OBJ_ACKLEY:
        switch (o.dim) {
#define ZB_CASE(D)                                                             \
  case D:                                                                      \
    return fn(zeus::Ackley<D>{});
          ZB_ACKLEY_DIMS(ZB_CASE)
#undef ZB_CASE
        }
        break;
      case ZEUS_OBJ_GAUSSIAN:
        switch (o.dim) {
#define ZB_CASE(D)                                                             \
  case D: {                                                                    \
    zeus::Gaussian<D> g;                                                       \
    g.C = o.data;                                                              \
    g.symmetric = (o.flags & 1) != 0;                                          \
    return fn(g);                                                              \
  }
          ZB_GAUSSIAN_DIMS(ZB_CASE)
#undef ZB_CASE
        }
        break;
      case ZEUS_OBJ_POISSON_NLL:
        if (o.dim == 4) {
          zeus::PoissonNLL p;
          p.centres = o.data;
          p.counts = o.idata;
          p.bins = o.nll_bins;
          p.nbins = o.ndata;
          return fn(p);
        }
        break;
    }
    set_error("objective kind %d with dim %d is not built", o.kind, o.dim);
    return ZEUS_E_UNSUPPORTED;
  }

  inline bool
  builtin_supported(int kind, int dim)
  {
    switch (kind) {
#define ZB_CASE(D)                                                             \
  case D:                                                                      \
    return true;
      case ZEUS_OBJ_ROSENBROCK:
        switch (dim) { ZB_ROSENBROCK_DIMS(ZB_CASE) }
        return false;
      case ZEUS_OBJ_RASTRIGIN:
        switch (dim) { ZB_RASTRIGIN_DIMS(ZB_CASE) }
        return false;
      case ZEUS_OBJ_ACKLEY:
        switch (dim) { ZB_ACKLEY_DIMS(ZB_CASE) }
        return false;
      case ZEUS_OBJ_GAUSSIAN:
        switch (dim) { ZB_GAUSSIAN_DIMS(ZB_CASE) }
        return false;
#undef ZB_CASE
      case ZEUS_OBJ_POISSON_NLL:
        return dim == 4;
    }
    return false;
  }

} // namespace zb
