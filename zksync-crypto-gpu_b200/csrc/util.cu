// Device utilities: seeded synthetic field elements and the modular-multiply throughput probe.
#include "glc_field.cuh"
#include "glc_internal.h"

namespace glc {

__device__ __forceinline__ uint32_t rotl32(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }

#define GLC_QR(a, b, c, d)                                                                                   \
  a += b; d ^= a; d = rotl32(d, 16);                                                                       \
  c += d; b ^= c; b = rotl32(b, 12);                                                                       \
  a += b; d ^= a; d = rotl32(d, 8);                                                                        \
  c += d; b ^= c; b = rotl32(b, 7);

// ChaCha20 block function (RFC 8439 section 2.3): key, 32-bit counter, 64-bit nonce in words 13-14.
__device__ void chacha20_block(const uint32_t key[8], uint32_t counter, uint64_t nonce, uint32_t out[16]) {
  uint32_t s[16] = {0x61707865u, 0x3320646Eu, 0x79622D32u, 0x6B206574u, key[0], key[1], key[2], key[3],
                    key[4],      key[5],      key[6],      key[7],      counter, (uint32_t)nonce,
                    (uint32_t)(nonce >> 32), 0u};
  uint32_t x[16];
#pragma unroll
  for (int i = 0; i < 16; i++) x[i] = s[i];
#pragma unroll
  for (int r = 0; r < 10; r++) {
    GLC_QR(x[0], x[4], x[8], x[12]);
    GLC_QR(x[1], x[5], x[9], x[13]);
    GLC_QR(x[2], x[6], x[10], x[14]);
    GLC_QR(x[3], x[7], x[11], x[15]);
    GLC_QR(x[0], x[5], x[10], x[15]);
    GLC_QR(x[1], x[6], x[11], x[12]);
    GLC_QR(x[2], x[7], x[8], x[13]);
    GLC_QR(x[3], x[4], x[9], x[14]);
  }
#pragma unroll
  for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}

struct Key {
  uint32_t k[8];
};

// element i = word i of the keystream (nonce 0); a word >= p is replaced by the first word < p of
// block i of the nonce-1 keystream (same definition as the Python generator).
__global__ void fill_random_kernel(uint64_t *dst, uint64_t count, uint64_t offset, Key key) {
  const uint64_t blk = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;  // one ChaCha block = 8 elements
  const uint64_t first = offset / 8 + blk;
  uint32_t out[16];
  chacha20_block(key.k, (uint32_t)first, 0, out);
#pragma unroll
  for (int w = 0; w < 8; w++) {
    const uint64_t idx = first * 8 + w;
    if (idx < offset || idx >= offset + count) continue;
    uint64_t v = ((uint64_t)out[2 * w + 1] << 32) | out[2 * w];
    if (v >= P) {
      uint32_t alt[16];
      chacha20_block(key.k, (uint32_t)idx, 1, alt);
      uint64_t pick = (((uint64_t)alt[1] << 32) | alt[0]) % P;
      for (int q = 7; q >= 0; q--) {
        const uint64_t a = ((uint64_t)alt[2 * q + 1] << 32) | alt[2 * q];
        if (a < P) pick = a;
      }
      v = pick;
    }
    dst[idx - offset] = v;
  }
}

// Independent multiply chains on every SM: the achievable modular-multiply rate of this device.
__global__ void __launch_bounds__(256) modmul_probe_kernel(uint64_t *out, uint64_t seed, uint32_t iters) {
  uint64_t x[8], y[8];
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    x[k] = seed * (t + 1) + k * 0x9E3779B97F4A7C15ull;
    y[k] = (seed ^ 0xABCDEFull) * (k + 3) + t;
  }
  for (uint32_t i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = mul(x[k], y[k]);
  }
  uint64_t acc = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) acc ^= x[k];
  out[t] = acc;
}

}  // namespace glc

using namespace glc;

extern "C" glc_status glc_fill_random(uint64_t *dst, uint64_t count, uint64_t offset, const uint8_t *key32,
                                      void *stream) {
  if (!dst || !key32) return fail("fill_random: null pointer");
  if (count == 0) return 0;
  if ((offset + count + 7) / 8 > 0xffffffffull) return fail("fill_random: stream position beyond 2^35 elements");
  Key key;
  for (int i = 0; i < 8; i++)
    key.k[i] = (uint32_t)key32[4 * i] | ((uint32_t)key32[4 * i + 1] << 8) | ((uint32_t)key32[4 * i + 2] << 16) |
               ((uint32_t)key32[4 * i + 3] << 24);
  const uint64_t blocks = (offset + count + 7) / 8 - offset / 8;
  const uint32_t threads = 256;
  fill_random_kernel<<<(uint32_t)((blocks + threads - 1) / threads), threads, 0, (cudaStream_t)stream>>>(dst, count,
                                                                                                      offset, key);
  return last_launch_error();
}

extern "C" glc_status glc_modmul_probe(uint64_t *scratch, uint32_t blocks, uint32_t iters, void *stream) {
  if (!scratch || blocks == 0) return fail("modmul_probe: bad arguments");
  modmul_probe_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(scratch, 12345, iters);
  return last_launch_error();
}
