// Sobol' direction numbers: the host construction and the per-device copy
// (the point formula and its use are in zb_sobol.cuh).
#include <mutex>
#include <vector>

#include "zb_internal.h"
#include "zb_sobol.cuh"

namespace zb {

  namespace {

    // a * b mod p over GF(2), deg p = s <= 31
    uint32_t
    gf2_mulmod(uint32_t a, uint32_t b, uint32_t p, int s)
    {
      uint64_t r = 0;
      for (int i = 0; i < 32; ++i)
        if ((b >> i) & 1u)
          r ^= (uint64_t)a << i;
      for (int i = 62; i >= s; --i)
        if ((r >> i) & 1u)
          r ^= (uint64_t)p << (i - s);
      return (uint32_t)r;
    }

    uint32_t
    gf2_powmod_x(uint64_t e, uint32_t p, int s)
    {
      uint32_t r = 1u, b = gf2_mulmod(2u, 1u, p, s); // x mod p
      while (e) {
        if (e & 1u)
          r = gf2_mulmod(r, b, p, s);
        b = gf2_mulmod(b, b, p, s);
        e >>= 1;
      }
      return r;
    }

    // p (bit s set, bit 0 set) is primitive iff x has order 2^s - 1 mod p
    bool
    primitive(uint32_t p, int s)
    {
      const uint64_t ord = (1ull << s) - 1;
      if (gf2_powmod_x(ord, p, s) != 1u)
        return false;
      uint64_t m = ord;
      for (uint64_t q = 2; q * q <= m; ++q)
        if (m % q == 0) {
          if (gf2_powmod_x(ord / q, p, s) == 1u)
            return false;
          while (m % q == 0)
            m /= q;
        }
      if (m > 1 && gf2_powmod_x(ord / m, p, s) == 1u)
        return false;
      return true;
    }

    uint64_t
    splitmix64(uint64_t* state)
    {
      uint64_t z = (*state += 0x9E3779B97F4A7C15ull);
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      return z ^ (z >> 31);
    }

    constexpr uint64_t kSobolInitSeed = 0x5A17B01Dull;

    static __device__ uint32_t g_sobol_dirs[kSobolMaxDim * kSobolBits];

  } // namespace

  void
  sobol_table(int ndim, uint32_t* dirs)
  {
    for (int k = 0; k < kSobolBits && ndim > 0; ++k)
      dirs[k] = 1u << (31 - k); // dimension 0: van der Corput
    int d = 1;
    for (int s = 1; d < ndim && s < 31; ++s)
      for (uint32_t p = (1u << s) | 1u; d < ndim && p < (2u << s); p += 2u) {
        if (!primitive(p, s))
          continue;
        uint32_t* v = dirs + (size_t)d * kSobolBits;
        uint64_t st = kSobolInitSeed + 0x100000001B3ull * (uint64_t)d;
        for (int k = 1; k <= s && k <= kSobolBits; ++k) {
          const uint32_t m = (uint32_t)(splitmix64(&st) >> 32) & ((1u << k) - 1u);
          v[k - 1] = (m | 1u) << (32 - k);
        }
        // v_k = v_{k-s} ^ (v_{k-s} >> s) ^ sum_{i<s} a_i v_{k-i},
        // a_i the coefficient of x^{s-i}
        for (int k = s + 1; k <= kSobolBits; ++k) {
          uint32_t x = v[k - s - 1] ^ (v[k - s - 1] >> s);
          for (int i = 1; i < s; ++i)
            if ((p >> (s - i)) & 1u)
              x ^= v[k - i - 1];
          v[k - 1] = x;
        }
        ++d;
      }
  }

  int
  sobol_table_device(const uint32_t** out)
  {
    static std::mutex mu;
    static const uint32_t* addr[64] = {};
    static std::vector<uint32_t> host;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
      return cuda_fail(e, "Sobol table: cudaGetDevice");
    if (dev < 0 || dev >= 64) {
      set_error("Sobol table: device index %d out of range", dev);
      return ZEUS_E_INVALID;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev]) {
      if (host.empty()) {
        host.assign((size_t)kSobolMaxDim * kSobolBits, 0u);
        sobol_table(kSobolMaxDim, host.data());
      }
      e = cudaMemcpyToSymbol(g_sobol_dirs, host.data(),
                             sizeof(uint32_t) * host.size());
      if (e != cudaSuccess)
        return cuda_fail(e, "Sobol table: copy to device");
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_sobol_dirs);
      if (e != cudaSuccess || !p)
        return cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                         "Sobol table: cudaGetSymbolAddress");
      addr[dev] = static_cast<const uint32_t*>(p);
    }
    *out = addr[dev];
    return ZEUS_OK;
  }

} // namespace zb

using namespace zb;

extern "C" {

int
zeus_sobol_directions(int32_t ndim, uint32_t* out)
{
  if (ndim <= 0 || ndim > kSobolMaxDim || !out) {
    set_error("zeus_sobol_directions: 1 <= ndim <= %d and an output array "
              "are required",
              kSobolMaxDim);
    return ZEUS_E_INVALID;
  }
  sobol_table(ndim, out);
  return ZEUS_OK;
}

int
zeus_sobol_device_table(const uint32_t** d_table)
{
  if (!d_table) {
    set_error("zeus_sobol_device_table: output pointer is NULL");
    return ZEUS_E_INVALID;
  }
  return sobol_table_device(d_table);
}

} // extern "C"
