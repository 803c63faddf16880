// Goldilocks field arithmetic for sm_100a.  p = 2^64 - 2^32 + 1.
//
// Values live in [0, 2^64) and are not necessarily canonical, like the reference's
// field<2> (crates/boojum-cuda/native/goldilocks.cuh:90-185).  Reductions use
// 2^64 = 2^32 - 1 (EPS) and 2^96 = -1 (mod p).  No tensor cores, no floating point:
// 32x32->64 integer multiply-adds (IMAD.WIDE) and carry chains.
#pragma once
#include <cstdint>

namespace glc {

static constexpr uint64_t P = 0xFFFFFFFF00000001ull;
static constexpr uint64_t EPS = 0xFFFFFFFFull;  // 2^64 mod p

__host__ __device__ __forceinline__ uint64_t canon(uint64_t a) { return a >= P ? a - P : a; }

// a + b mod p, inputs and output in [0, 2^64).
__device__ __forceinline__ uint64_t add(uint64_t a, uint64_t b) {
  uint64_t s = a + b;
  if (s < a) {       // wrapped: s + 2^64 = s + EPS
    s += EPS;
    if (s < EPS) s += EPS;  // wrapped again (only when s >= p); cannot wrap a third time
  }
  return s;
}

// a - b mod p.
__device__ __forceinline__ uint64_t sub(uint64_t a, uint64_t b) {
  uint64_t d = a - b;
  if (a < b) {       // borrowed: d - 2^64 = d - EPS
    uint64_t e = d - EPS;
    if (d < EPS) e -= EPS;  // borrowed again
    d = e;
  }
  return d;
}

// Reduce the 128-bit value hi:lo to [0, 2^64).
__device__ __forceinline__ uint64_t reduce128(uint64_t lo, uint64_t hi) {
  const uint64_t hh = hi >> 32;
  const uint64_t hl = hi & 0xFFFFFFFFull;
  uint64_t t0 = lo - hh;                 // lo - hh*2^96 == lo + hh*(-1)
  if (lo < hh) t0 -= EPS;                // borrow: -2^64 = -EPS; t0 >= 2^64 - 2^32 so no new borrow
  const uint64_t t1 = hl * EPS;          // hl * 2^64 == hl * EPS, < 2^64
  uint64_t r = t0 + t1;
  if (r < t1) r += EPS;                  // carry; r <= 2^64 - 2^33 before, so no new carry
  return r;
}

// 64x64 -> 128 product from four 32x32->64 multiply-adds.
__device__ __forceinline__ void mul_wide(uint64_t a, uint64_t b, uint64_t &lo, uint64_t &hi) {
  const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
  const uint32_t b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
  const uint64_t p00 = (uint64_t)a0 * b0;
  const uint64_t t = (uint64_t)a1 * b0 + (p00 >> 32);             // < 2^64
  const uint64_t u = (uint64_t)a0 * b1 + (t & 0xFFFFFFFFull);     // < 2^64
  hi = (uint64_t)a1 * b1 + (t >> 32) + (u >> 32);                  // <= 2^64 - 1
  lo = (u << 32) | (p00 & 0xFFFFFFFFull);
}

__device__ __forceinline__ uint64_t mul(uint64_t a, uint64_t b) {
  uint64_t lo, hi;
  mul_wide(a, b, lo, hi);
  return reduce128(lo, hi);
}

__device__ __forceinline__ uint64_t sqr(uint64_t a) { return mul(a, a); }

__device__ __forceinline__ uint64_t pow(uint64_t a, uint64_t e) {
  uint64_t r = 1;
  while (e) {
    if (e & 1) r = mul(r, a);
    a = mul(a, a);
    e >>= 1;
  }
  return r;
}

// ---- host-side exact arithmetic (table construction) ----
inline uint64_t h_mul(uint64_t a, uint64_t b) {
  const unsigned __int128 x = (unsigned __int128)a * b;
  const uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
  const uint64_t hh = hi >> 32, hl = hi & 0xFFFFFFFFull;
  uint64_t t0 = lo - hh;
  if (lo < hh) t0 -= EPS;
  const uint64_t t1 = hl * EPS;
  uint64_t r = t0 + t1;
  if (r < t1) r += EPS;
  return canon(r);
}

inline uint64_t h_pow(uint64_t a, uint64_t e) {
  uint64_t r = 1;
  a = canon(a);
  while (e) {
    if (e & 1) r = h_mul(r, a);
    a = h_mul(a, a);
    e >>= 1;
  }
  return r;
}

inline uint64_t h_inv(uint64_t a) { return h_pow(a, P - 2); }

static constexpr uint64_t GENERATOR = 7;  // multiplicative generator (boojum-cuda src/context.rs:232)

// w_{2^k} = 7^((p-1)/2^k)
inline uint64_t h_root_of_unity(uint32_t log_n) { return h_pow(GENERATOR, (P - 1) >> log_n); }

}  // namespace glc
