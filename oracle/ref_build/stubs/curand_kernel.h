// Stand-in for <curand_kernel.h> in the host build of the reference.
// The reference only needs the state type names and curand_uniform_double();
// the oracle always injects start points (pso_array != nullptr), so no random
// number is ever drawn.  Drawing one aborts, loudly.
#pragma once
#include <cstdlib>

struct curandStateXORWOW {
  unsigned int unused;
};
typedef curandStateXORWOW curandStateXORWOW_t;
typedef curandStateXORWOW curandState;
typedef curandStateXORWOW curandState_t;
struct curandStatePhilox4_32_10 {
  unsigned int unused;
};
typedef curandStatePhilox4_32_10 curandStatePhilox4_32_10_t;
struct curandStateSobol32 {
  unsigned int unused;
};
typedef curandStateSobol32 curandStateSobol32_t;
typedef unsigned int curandDirectionVectors32_t[32];

template <class S>
inline double
curand_uniform_double(S*)
{
  ::abort();
  return 0.0;
}

enum curandDirectionVectorSet { CURAND_DIRECTION_VECTORS_32_JOEKUO6 = 101 };
inline int
curandGetDirectionVectors32(curandDirectionVectors32_t**, curandDirectionVectorSet)
{
  ::abort();
  return 0;
}
