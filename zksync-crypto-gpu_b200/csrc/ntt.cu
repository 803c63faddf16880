// Batched Goldilocks NTT / coset LDE and bit reversal for sm_100a.
//
// Replaces boojum-cuda's ntt:: and ops_complex::bit_reverse (crates/boojum-cuda/src/ntt.rs,
// native/ntt*.cu*, native/ops_complex.cu:88-156) with a B200 design of its own:
//
//  * An NTT of size N = 2^L runs as one pass (L <= 12) or two passes (L <= 24).  A pass covers
//    k consecutive radix-2 stages.  Writing a position as i = hi*2^(L-s0) + mid*M + lo
//    (M = 2^(L-s0-k)), the pass transforms the 2^k values of every (hi, lo) group.  One CTA
//    owns a tile of W consecutive lo values of one hi (W*8 bytes contiguous per row: coalesced
//    128-bit loads), stages it in shared memory and runs the k stages as radix-8 register
//    rounds with XOR-swizzled shared-memory exchanges.  The CTA walks several columns with the
//    same twiddles, which it builds once in shared memory.
//  * n2b (natural -> bit-reversed) runs the stages in increasing order with DIT butterflies,
//    b2n (bit-reversed -> natural) is its transpose: decreasing order, DIF butterflies.  Both
//    use the twiddle T[b] = w^bitrev(b) of block b at each stage; T is one flat table.
//  * Coset scaling (forward LDE: x s^j on load) and N^-1 s^-j (inverse: on store) are fused
//    into the first / last pass, so an LDE costs no extra HBM pass.
//  * Optionally (tuning), batches larger than an L2-sized chunk of columns run pass 1 and pass 2
//    chunk by chunk, so the second pass reads the first pass's output from the 126 MB L2.  The
//    NTT is integer-bound, and small chunks cost more in per-CTA twiddle tables than they save
//    in HBM traffic, so the default is one chunk.
#include <algorithm>

#include "glc_field.cuh"
#include "glc_internal.h"

namespace glc {

static constexpr uint32_t MAX_TILE_LOG = 13;  // 8192 elements = 64 KiB of shared memory
static constexpr uint32_t PASS_THREADS = 512;
// Radix-16 rounds hold 16 values per thread: capped at 256 threads with 3 CTAs per SM they get
// 85 registers (no spills) instead of the 64 a 512-thread CTA pair allows (measured 1-1.5%
// faster on B200).
__host__ __device__ constexpr uint32_t pass_threads(uint32_t rb) { return rb >= 4 ? 256 : PASS_THREADS; }
__host__ __device__ constexpr uint32_t pass_min_blocks(uint32_t rb) { return rb >= 4 ? 3 : 2; }
static constexpr uint32_t SINGLE_PASS_MAX_LOG = 12;
static constexpr int NTT_SMEM_MAX = 140 * 1024;  // tile 64 KiB + twiddles 32 KiB + scaling tables 32 KiB  // one column per tile, tile + twiddles <= 64 KiB

struct PassArgs {
  const uint64_t *in;
  uint64_t *out;
  uint64_t in_stride, out_stride;
  uint32_t num_cols, cols_per_cta;
  uint32_t log_n, s0, k, log_w;
  uint32_t dif;  // 0: n2b stages (DIT, increasing), 1: b2n stages (DIF, decreasing)
  const uint64_t *tw;
  uint32_t scale;     // 0: none, 1: x s^j on load, 2: x N^-1 s^-j on store
  uint32_t fold;      // 1: forward n2b coset NTT with s folded into the block twiddles
  uint32_t last;      // last pass: canonical output
  uint32_t vec2;      // 16-byte loads and stores: aligned matrices, even strides, no per-element
                      // coset factor on load, no coset factor on store
  uint32_t j_bitrev;  // exponent j = bitrev_L(position) instead of position
  uint32_t log_ext, coset;
  uint64_t n_inv;
  const uint64_t *g_lo, *g_hi;  // powers of g (scale 1) or g^-1 (scale 2)
  const uint64_t *w_lo, *w_hi;  // powers of w_{2^30}
};

__device__ __forceinline__ uint32_t swz(uint32_t e) { return e ^ ((e >> 4) & 15u); }

// s^j (scale 1) or s^-j (scale 2) for the coset shift s = g * w_{2^(L+e)}^c; 1 without extension
__device__ __forceinline__ uint64_t coset_power(const PassArgs &a, uint32_t j) {
  uint64_t f = 1;
  if (a.log_ext) {
    f = mul(a.g_lo[j & 4095], a.g_hi[j >> 12]);
    if (a.coset) {
      // s^j carries w_{2^(L+e)}^(c*j) = w_{2^30}^((c*j) << (30-L-e)); c*j < 2^(L+e) <= 2^30
      uint32_t y = (a.coset * j) << (OMEGA_LOG_ORDER - a.log_n - a.log_ext);
      if (a.scale == 2) y = ((1u << OMEGA_LOG_ORDER) - y) & ((1u << OMEGA_LOG_ORDER) - 1);
      f = mul(f, mul(a.w_lo[y & 32767], a.w_hi[y >> 15]));
    }
  }
  return f;
}

__device__ __forceinline__ uint32_t brev_low(uint32_t x, uint32_t bits) { return bits ? __brev(x) >> (32 - bits) : 0; }

template <uint32_t R, bool DIF>
__device__ __forceinline__ void radix_round(uint64_t *tile, const uint64_t *tws, uint32_t k, uint32_t log_w, uint32_t t) {
  const uint32_t log_e = k + log_w;
  const uint32_t p = k - t - R + log_w;  // lowest active bit of the tile index
  const uint32_t jobs = 1u << (log_e - R);
  for (uint32_t q = threadIdx.x; q < jobs; q += blockDim.x) {
    const uint32_t base = ((q >> p) << (p + R)) | (q & ((1u << p) - 1));
    const uint32_t mid_base = base >> log_w;
    uint64_t v[1 << R];
#pragma unroll
    for (uint32_t j = 0; j < (1u << R); j++) v[j] = tile[swz(base | (j << p))];
#pragma unroll
    for (uint32_t uu = 0; uu < R; uu++) {
      const uint32_t u = DIF ? R - 1 - uu : uu;
      const uint32_t level = t + u;
      const uint32_t bit = R - 1 - u;
      const uint32_t mb = mid_base >> (k - level);
#pragma unroll
      for (uint32_t j = 0; j < (1u << R); j++) {
        if (j & (1u << bit)) continue;
        const uint32_t m = mb | (j >> (R - u));
        const uint64_t w = tws[(1u << level) - 1 + m];
        const uint64_t x = v[j], y = v[j | (1u << bit)];
        if (!DIF) {
          const uint64_t yw = mul(y, w);
          v[j] = add(x, yw);
          v[j | (1u << bit)] = sub(x, yw);
        } else {
          v[j] = add(x, y);
          v[j | (1u << bit)] = mul(sub(x, y), w);
        }
      }
    }
#pragma unroll
    for (uint32_t j = 0; j < (1u << R); j++) tile[swz(base | (j << p))] = v[j];
  }
}

template <bool DIF, uint32_t RB>
__device__ __forceinline__ void round_dispatch(uint64_t *tile, const uint64_t *tws, uint32_t k, uint32_t log_w, uint32_t t,
                                               uint32_t r) {
  if (RB >= 4 && r == 4)
    radix_round<(RB >= 4 ? 4 : 1), DIF>(tile, tws, k, log_w, t);
  else if (RB >= 3 && r == 3)
    radix_round<(RB >= 3 ? 3 : 1), DIF>(tile, tws, k, log_w, t);
  else if (r == 2)
    radix_round<2, DIF>(tile, tws, k, log_w, t);
  else
    radix_round<1, DIF>(tile, tws, k, log_w, t);
}

template <uint32_t RB>
__global__ void __launch_bounds__(pass_threads(RB), pass_min_blocks(RB)) ntt_pass_kernel(const PassArgs a) {
  extern __shared__ uint64_t smem[];
  const uint32_t k = a.k, log_w = a.log_w;
  const uint32_t E = 1u << (k + log_w);
  uint64_t *tile = smem;
  uint64_t *tws = smem + E;
  const uint32_t log_m = a.log_n - a.s0 - k;
  const uint32_t log_tph = log_m - log_w;
  const uint32_t hi = blockIdx.x >> log_tph;
  const uint32_t lo0 = (blockIdx.x & ((1u << log_tph) - 1)) << log_w;
  const uint64_t base_i = ((uint64_t)hi << (a.log_n - a.s0)) + lo0;
  // tws[2^t - 1 + m] = T[hi * 2^t + m]: block twiddles of stage s0 + t for this hi.
  // Folded coset NTT: DFT(x_j s^j) splits at every stage into two half-size problems whose
  // cosets differ by the stage's twiddle, so each block twiddle of stage u gains the factor
  // s^(2^(L-1-u)) and the x s^j scaling disappears from the data path.
  __shared__ uint64_t sig[MAX_TILE_LOG];
  if (a.fold) {
    if (threadIdx.x < k) sig[threadIdx.x] = coset_power(a, 1u << (a.log_n - 1 - a.s0 - threadIdx.x));
    __syncthreads();
  }
  for (uint32_t idx = threadIdx.x; idx + 1 < (1u << k); idx += blockDim.x) {
    const uint32_t t = 31 - __clz(idx + 1);
    const uint32_t m = idx + 1 - (1u << t);
    const uint64_t w = a.tw[((uint64_t)hi << t) + m];
    tws[idx] = a.fold ? mul(w, sig[t]) : w;
  }
  // Coset / size scaling as two per-CTA tables: the exponent j of element (mid, w) splits as
  //   natural j = mid * M + (lo0 + w)                      (strided pass, hi = 0)
  //   bit-reversed j = bitrev_k(mid) << (L - k) + bitrev_{L-k}(hi)  (contiguous pass, W = 1)
  // so the factor is P[mid] * Q[w] (P carries N^-1 on the inverse side): 2 multiplies per element.
  uint64_t *Pt = tws + (1u << k);
  uint64_t *Qt = Pt + (1u << k);
  if (a.scale == 1 || (a.scale == 2 && a.log_ext)) {
    for (uint32_t m = threadIdx.x; m < (1u << k); m += blockDim.x) {
      const uint32_t jm = a.j_bitrev ? brev_low(m, k) << (a.log_n - k) : m << log_m;
      const uint64_t pm = coset_power(a, jm);
      Pt[m] = a.scale == 2 ? mul(pm, a.n_inv) : pm;
    }
    const uint32_t nq = a.j_bitrev ? 1u : (1u << log_w);
    for (uint32_t w = threadIdx.x; w < nq; w += blockDim.x)
      Qt[w] = coset_power(a, a.j_bitrev ? brev_low(hi, a.log_n - k) : lo0 + w);
  }
  const uint32_t col0 = blockIdx.y * a.cols_per_cta;
  const uint32_t col1 = min(col0 + a.cols_per_cta, a.num_cols);
  const uint32_t wmask = (1u << log_w) - 1;
  const uint32_t nrounds = (k + RB - 1) / RB;
  for (uint32_t col = col0; col < col1; col++) {
    const uint64_t *src = a.in + (uint64_t)col * a.in_stride;
    uint64_t *dst = a.out + (uint64_t)col * a.out_stride;
    __syncthreads();
    if (a.vec2) {
      // two consecutive elements per thread, one 16-byte load: tile indexes e and e + 1 are
      // adjacent in memory (same row of a W >= 2 tile, or a contiguous W = 1 tile)
      for (uint32_t e = 2 * threadIdx.x; e < E; e += 2 * blockDim.x) {
        const uint64_t i = base_i + ((uint64_t)(e >> log_w) << log_m) + (e & wmask);
        const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(src + i);
        tile[swz(e)] = v.x;
        tile[swz(e + 1)] = v.y;
      }
    } else {
      for (uint32_t e = threadIdx.x; e < E; e += blockDim.x) {
        const uint64_t i = base_i + ((uint64_t)(e >> log_w) << log_m) + (e & wmask);
        uint64_t v = src[i];
        if (a.scale == 1) v = mul(v, mul(Pt[e >> log_w], Qt[a.j_bitrev ? 0u : (e & wmask)]));
        tile[swz(e)] = v;
      }
    }
    __syncthreads();
    if (!a.dif) {
      for (uint32_t q = 0; q < nrounds; q++) {
        const uint32_t t = q * RB;
        round_dispatch<false, RB>(tile, tws, k, log_w, t, min(RB, k - t));
        __syncthreads();
      }
    } else {
      for (int q = (int)nrounds - 1; q >= 0; q--) {
        const uint32_t t = q * RB;
        round_dispatch<true, RB>(tile, tws, k, log_w, t, min(RB, k - t));
        __syncthreads();
      }
    }
    if (a.vec2) {
      for (uint32_t e = 2 * threadIdx.x; e < E; e += 2 * blockDim.x) {
        const uint64_t i = base_i + ((uint64_t)(e >> log_w) << log_m) + (e & wmask);
        uint64_t v0 = tile[swz(e)], v1 = tile[swz(e + 1)];
        if (a.scale == 2) {
          v0 = mul(v0, a.n_inv);
          v1 = mul(v1, a.n_inv);
        }
        if (a.last) {
          v0 = canon(v0);
          v1 = canon(v1);
        }
        *reinterpret_cast<ulonglong2 *>(dst + i) = make_ulonglong2(v0, v1);
      }
    } else {
      for (uint32_t e = threadIdx.x; e < E; e += blockDim.x) {
        const uint64_t i = base_i + ((uint64_t)(e >> log_w) << log_m) + (e & wmask);
        uint64_t v = tile[swz(e)];
        if (a.scale == 2)
          v = a.log_ext ? mul(v, mul(Pt[e >> log_w], Qt[a.j_bitrev ? 0u : (e & wmask)])) : mul(v, a.n_inv);
        dst[i] = a.last ? canon(v) : v;  // a following pass accepts any value below 2^64
      }
    }
  }
}

// ---- bit reversal (ops_complex.cu:88-156 semantics) ----

__global__ void bitrev_naive_kernel(const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride,
                                    uint32_t log_rows) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (1u << log_rows)) return;
  const uint32_t r = log_rows ? __brev(i) >> (32 - log_rows) : 0;
  if (i > r) return;
  const uint64_t col = blockIdx.y;
  const uint64_t vi = src[col * src_stride + i], vr = src[col * src_stride + r];
  dst[col * dst_stride + i] = vr;
  dst[col * dst_stride + r] = vi;
}

// log_rows = 2h + odd, h >= 5.  Position i = a*2^(h+odd) + m*2^h + b.  Tile (A, B, m) holds
// a = x*2^(h-5) + A, b = B*32 + y (x, y < 32); its image is tile (rev(B), rev(A), m) with
// (x, y) -> (rev5(y), rev5(x)).  One CTA moves a tile and its image, so in place is safe.
__global__ void __launch_bounds__(256) bitrev_tiled_kernel(const uint64_t *src, uint64_t src_stride, uint64_t *dst,
                                                           uint64_t dst_stride, uint32_t log_rows) {
  __shared__ uint64_t t0[32][33];
  __shared__ uint64_t t1[32][33];
  const uint32_t h = log_rows >> 1;
  const uint32_t odd = log_rows & 1;
  const uint32_t hb = h - 5;
  const uint32_t A = blockIdx.x >> hb, B = blockIdx.x & ((1u << hb) - 1);
  const uint32_t As = hb ? __brev(B) >> (32 - hb) : 0, Bs = hb ? __brev(A) >> (32 - hb) : 0;
  if (A > As || (A == As && B > Bs)) return;  // the image tile's CTA moves this pair
  const uint32_t m = blockIdx.z;
  const uint64_t col = blockIdx.y;
  const uint64_t *s = src + col * src_stride;
  uint64_t *d = dst + col * dst_stride;
  const bool self = (A == As && B == Bs);
  auto pos = [&](uint32_t TA, uint32_t TB, uint32_t x, uint32_t y) -> uint64_t {
    const uint64_t a = ((uint64_t)x << hb) + TA, b = ((uint64_t)TB << 5) + y;
    return (a << (h + odd)) + ((uint64_t)m << h) + b;
  };
  const uint32_t tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 8 rows per sweep
  for (uint32_t x = ty; x < 32; x += 8) {
    t0[x][tx] = s[pos(A, B, x, tx)];
    if (!self) t1[x][tx] = s[pos(As, Bs, x, tx)];
  }
  __syncthreads();
  // element (x, y) of tile (A, B) goes to (rev5(y), rev5(x)) of tile (As, Bs); store row-wise
  for (uint32_t xr = ty; xr < 32; xr += 8) {
    const uint32_t y = __brev(xr) >> 27, x = __brev(tx) >> 27;
    d[pos(As, Bs, xr, tx)] = t0[x][y];
    if (!self) d[pos(A, B, xr, tx)] = t1[x][y];
  }
}

int ntt_init_device() {
  cudaError_t e = cudaFuncSetAttribute(ntt_pass_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, NTT_SMEM_MAX);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(ntt_pass_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, NTT_SMEM_MAX);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(ntt_pass_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, NTT_SMEM_MAX);
  return (int)e;
}

int bitrev_launch(const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride, uint32_t log_rows,
                  uint32_t cols, cudaStream_t stream) {
  if (cols == 0) return 0;
  if (cols > 65535) {
    for (uint32_t c = 0; c < cols; c += 65535) {
      const int e = bitrev_launch(src + c * src_stride, src_stride, dst + c * dst_stride, dst_stride, log_rows,
                                  std::min<uint32_t>(65535, cols - c), stream);
      if (e) return e;
    }
    return 0;
  }
  if (log_rows < 10) {
    const uint32_t n = 1u << log_rows;
    const uint32_t threads = std::min<uint32_t>(n, 256);
    bitrev_naive_kernel<<<dim3((n + threads - 1) / threads, cols), threads, 0, stream>>>(src, src_stride, dst, dst_stride,
                                                                                          log_rows);
  } else {
    const uint32_t h = log_rows >> 1;
    const uint32_t tiles = 1u << (2 * (h - 5));
    bitrev_tiled_kernel<<<dim3(tiles, cols, 1u << (log_rows & 1)), 256, 0, stream>>>(src, src_stride, dst, dst_stride,
                                                                                   log_rows);
  }
  return last_launch_error();
}

// ---- NTT planner ----

NttTuning g_ntt_tuning[MAX_DEVICES][MAX_LOG_N + 1];

NttTuning &ntt_tuning(uint32_t log_n) {
  int dev = 0;
  cudaGetDevice(&dev);
  return g_ntt_tuning[(dev >= 0 && dev < MAX_DEVICES) ? dev : 0][std::min(log_n, MAX_LOG_N)];
}

struct Pass {
  uint32_t s0, k, log_w;
};

static uint32_t make_plan(uint32_t log_n, bool b2n, const NttTuning &tu, Pass *passes) {
  uint32_t ks[2];
  uint32_t np;
  if (log_n <= SINGLE_PASS_MAX_LOG) {
    np = 1;
    ks[0] = log_n;
  } else {
    np = 2;
    // strided pass (stages 0 .. k0-1) then contiguous pass (stages k0 .. L-1), each <= 12 stages
    uint32_t k0 = tu.k1 ? tu.k1 : log_n / 2;
    k0 = std::max(log_n - SINGLE_PASS_MAX_LOG, std::min(k0, SINGLE_PASS_MAX_LOG));
    ks[0] = k0;
    ks[1] = log_n - k0;
  }
  Pass p[2];
  for (uint32_t q = 0; q < np; q++) {
    const uint32_t s0 = q == 0 ? 0 : ks[0];
    const uint32_t k = ks[q];
    const uint32_t log_m = log_n - s0 - k;
    uint32_t log_w = std::min<uint32_t>(MAX_TILE_LOG - k, tu.max_log_w);
    log_w = std::min(log_w, log_m);
    p[q] = {s0, k, log_w};
  }
  // n2b runs stage groups in increasing order, b2n (the transposed network) in decreasing order
  for (uint32_t q = 0; q < np; q++) passes[q] = b2n ? p[np - 1 - q] : p[q];
  return np;
}

int ntt_launch(const uint64_t *in, uint64_t *out, uint32_t log_n, uint32_t num_ntts, uint64_t in_stride,
               uint64_t out_stride, bool bitrev_inputs, bool inverse, uint32_t log_ext, uint32_t coset_idx,
               cudaStream_t stream, uint32_t l2_chunk_cols) {
  const DeviceTables *t = current_tables();
  if (!t) return fail("NTT: glc_context_create has not been called on this device");
  if (num_ntts == 0) return 0;
  const NttTuning &tu = ntt_tuning(log_n);
  Pass passes[2];
  const uint32_t np = make_plan(log_n, bitrev_inputs, tu, passes);
  const uint64_t n = 1ull << log_n;
  if (l2_chunk_cols == 0) {
    // keep one chunk of columns resident in L2 across the passes
    // (chunking trades HBM traffic for CTAs that each cover fewer columns and rebuild their
    // twiddles more often; on B200 the NTT is integer-bound, so one chunk usually wins)
    const uint64_t budget = (uint64_t)tu.l2_chunk_mb << 20;
    l2_chunk_cols = tu.l2_chunk_mb ? (uint32_t)std::max<uint64_t>(1, budget / (n * 8)) : num_ntts;
  }
  if (np == 1) l2_chunk_cols = num_ntts;
  for (uint32_t c0 = 0; c0 < num_ntts; c0 += l2_chunk_cols) {
    const uint32_t cols = std::min(l2_chunk_cols, num_ntts - c0);
    for (uint32_t q = 0; q < np; q++) {
      const Pass &ps = passes[q];
      PassArgs a{};
      a.in = (q == 0 ? in + (uint64_t)c0 * in_stride : out + (uint64_t)c0 * out_stride);
      a.in_stride = q == 0 ? in_stride : out_stride;
      a.out = out + (uint64_t)c0 * out_stride;
      a.out_stride = out_stride;
      a.num_cols = cols;
      a.log_n = log_n;
      a.s0 = ps.s0;
      a.k = ps.k;
      a.log_w = ps.log_w;
      a.dif = bitrev_inputs ? 1 : 0;
      a.tw = inverse ? t->tw_inv : t->tw_fwd;
      a.log_ext = log_ext;
      a.coset = coset_idx;
      a.n_inv = t->inv_sizes[log_n];
      a.w_lo = t->w_lo;
      a.w_hi = t->w_hi;
      const bool first = q == 0, last = q + 1 == np;
      a.last = last ? 1 : 0;
      if (!inverse && log_ext > 0 && !bitrev_inputs) {
        a.fold = 1;  // every pass: the coset factor rides on the block twiddles
        a.g_lo = t->g_lo;
        a.g_hi = t->g_hi;
      } else if (!inverse && first && log_ext > 0) {
        a.scale = 1;
        a.j_bitrev = bitrev_inputs ? 1 : 0;  // b2n input position i holds coefficient bitrev(i)
        a.g_lo = t->g_lo;
        a.g_hi = t->g_hi;
      } else if (inverse && last) {
        a.scale = 2;
        a.j_bitrev = bitrev_inputs ? 0 : 1;  // n2b output position i holds coefficient bitrev(i)
        a.g_lo = t->gi_lo;
        a.g_hi = t->gi_hi;
      }
      const bool aligned = ((reinterpret_cast<uintptr_t>(a.in) | reinterpret_cast<uintptr_t>(a.out)) & 15) == 0 &&
                           (a.in_stride & 1) == 0 && (a.out_stride & 1) == 0;
      // pairs of tile indexes (e, e + 1) must be adjacent in memory: rows of W >= 2 elements, or
      // W = 1 with a contiguous tile (M = 1)
      const bool pairs_adjacent = ps.log_w >= 1 || log_n - ps.s0 - ps.k == 0;
      a.vec2 = (aligned && pairs_adjacent && a.scale != 1 && !(a.scale == 2 && log_ext)) ? 1 : 0;
      const uint32_t tile_log = ps.k + ps.log_w;
      const uint64_t tiles_per_col = n >> tile_log;
      // enough CTAs to fill 148 SMs a few times over; the rest of the columns loop inside a CTA
      const uint64_t want = 148ull * 8;
      uint32_t cpc = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(tu.max_cols_per_cta, (tiles_per_col * cols) / want));
      a.cols_per_cta = cpc;
      const uint32_t gy = (cols + cpc - 1) / cpc;
      // tile + block twiddles (+ the P/Q scaling tables on a scaled pass)
      // (the inverse NTT's last pass without a coset multiplies by N^-1 only: no tables, and the
      // 2^k-entry table it does not need would cost a third CTA per SM on 2^12-element tiles)
      const bool tables = a.scale == 1 || (a.scale == 2 && a.log_ext);
      const size_t smem = ((size_t(1) << tile_log) + (size_t(1) << ps.k) +
                           (tables ? (size_t(1) << ps.k) + (size_t(1) << ps.log_w) : 0)) *
                          sizeof(uint64_t);
      const uint32_t threads =
          (uint32_t)std::min<uint64_t>(pass_threads(tu.radix_bits), std::max<uint64_t>(32, (1ull << tile_log) >> tu.radix_bits));
      if (gy > 65535) count_launches((gy - 1) / 65535);
      for (uint32_t y0 = 0; y0 < gy; y0 += 65535) {
        PassArgs b = a;
        const uint32_t ycount = std::min<uint32_t>(65535, gy - y0);
        b.in += (uint64_t)y0 * cpc * b.in_stride;
        b.out += (uint64_t)y0 * cpc * b.out_stride;
        b.num_cols = std::min<uint32_t>(cols - y0 * cpc, ycount * cpc);
        const dim3 grid((uint32_t)tiles_per_col, ycount);
        if (tu.radix_bits == 2)
          ntt_pass_kernel<2><<<grid, threads, smem, stream>>>(b);
        else if (tu.radix_bits == 4)
          ntt_pass_kernel<4><<<grid, threads, smem, stream>>>(b);
        else
          ntt_pass_kernel<3><<<grid, threads, smem, stream>>>(b);
      }
      const int e = last_launch_error();
      if (e) return e;
    }
  }
  return 0;
}

static int ntt_check(uint32_t log_n, uint32_t num_ntts, uint64_t in_stride, uint64_t out_stride, uint32_t log_ext,
                     uint32_t coset_idx) {
  (void)num_ntts;
  // ntt.rs:192-200
  if (log_n < 1) return fail("NTT: log_n must be >= 1");
  if (log_n + log_ext > OMEGA_LOG_ORDER) return fail("NTT: log_n + log_extension_degree must be <= 30");
  if (log_n > MAX_LOG_N) return fail("NTT: log_n must be <= 24");
  const uint64_t n = 1ull << log_n;
  if (n > in_stride || n > out_stride) return fail("NTT: n must be <= the strides between arrays");
  if (coset_idx > 0) {
    if (log_ext == 0) return fail("NTT: coset_index > 0 requires log_extension_degree > 0");
    if (coset_idx >= (1u << log_ext)) return fail("NTT: coset_index must be < 2^log_extension_degree");
  }
  return 0;
}

}  // namespace glc

using namespace glc;

extern "C" glc_status glc_batch_ntt_out_of_place(const uint64_t *inputs_matrix, size_t inputs_len,
                                                 uint64_t *outputs_matrix, size_t outputs_len, uint32_t log_n,
                                                 uint32_t num_ntts, uint32_t inputs_offset, uint32_t outputs_offset,
                                                 uint32_t stride_between_input_arrays,
                                                 uint32_t stride_between_output_arrays, bool bitrev_inputs,
                                                 bool inverse, uint32_t log_extension_degree, uint32_t coset_index,
                                                 void *stream) {
  // ntt.rs:308-320
  if (log_n >= 32) return fail("NTT: log_n out of range");
  const uint64_t n = 1ull << log_n;
  if ((uint64_t)inputs_offset + n > stride_between_input_arrays)
    return fail("NTT: inputs_offset + n must be <= stride_between_input_arrays");
  if ((uint64_t)outputs_offset + n > stride_between_output_arrays)
    return fail("NTT: outputs_offset + n must be <= stride_between_output_arrays");
  if (inputs_len < (uint64_t)num_ntts * stride_between_input_arrays)
    return fail("NTT: inputs_matrix shorter than num_ntts * stride_between_input_arrays");
  if (outputs_len < (uint64_t)num_ntts * stride_between_output_arrays)
    return fail("NTT: outputs_matrix shorter than num_ntts * stride_between_output_arrays");
  if (inputs_matrix == outputs_matrix) return fail("NTT: out-of-place call with identical matrices");
  if (inputs_matrix + inputs_offset == outputs_matrix + outputs_offset)
    return fail("NTT: out-of-place call with identical offset pointers");
  int e = ntt_check(log_n, num_ntts, stride_between_input_arrays, stride_between_output_arrays, log_extension_degree,
                    coset_index);
  if (e) return e;
  return ntt_launch(inputs_matrix + inputs_offset, outputs_matrix + outputs_offset, log_n, num_ntts,
                    stride_between_input_arrays, stride_between_output_arrays, bitrev_inputs, inverse,
                    log_extension_degree, coset_index, (cudaStream_t)stream, 0);
}

extern "C" glc_status glc_batch_ntt_in_place(uint64_t *inputs_matrix, size_t inputs_len, uint32_t log_n,
                                             uint32_t num_ntts, uint32_t inputs_offset,
                                             uint32_t stride_between_input_arrays, bool bitrev_inputs, bool inverse,
                                             uint32_t log_extension_degree, uint32_t coset_index, void *stream) {
  // ntt.rs:350-353
  if (log_n >= 32) return fail("NTT: log_n out of range");
  const uint64_t n = 1ull << log_n;
  if ((uint64_t)inputs_offset + n > stride_between_input_arrays)
    return fail("NTT: inputs_offset + n must be <= stride_between_input_arrays");
  if (inputs_len < (uint64_t)num_ntts * stride_between_input_arrays)
    return fail("NTT: inputs_matrix shorter than num_ntts * stride_between_input_arrays");
  int e = ntt_check(log_n, num_ntts, stride_between_input_arrays, stride_between_input_arrays, log_extension_degree,
                    coset_index);
  if (e) return e;
  uint64_t *p = inputs_matrix + inputs_offset;
  return ntt_launch(p, p, log_n, num_ntts, stride_between_input_arrays, stride_between_input_arrays, bitrev_inputs,
                    inverse, log_extension_degree, coset_index, (cudaStream_t)stream, 0);
}

static int bitrev_check(uint32_t rows, uint64_t src_stride, uint64_t dst_stride) {
  // ops_complex.rs:280-283
  if (rows == 0 || (rows & (rows - 1))) return fail("bit_reverse: rows must be a power of two");
  if (src_stride < rows || dst_stride < rows) return fail("bit_reverse: stride must be >= rows");
  return 0;
}

extern "C" glc_status glc_bit_reverse(const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride,
                                      uint32_t rows, uint32_t cols, void *stream) {
  int e = bitrev_check(rows, src_stride, dst_stride);
  if (e) return e;
  return bitrev_launch(src, src_stride, dst, dst_stride, 31 - __builtin_clz(rows), cols, (cudaStream_t)stream);
}

extern "C" glc_status glc_bit_reverse_in_place(uint64_t *values, uint64_t stride, uint32_t rows, uint32_t cols,
                                               void *stream) {
  int e = bitrev_check(rows, stride, stride);
  if (e) return e;
  return bitrev_launch(values, stride, values, stride, 31 - __builtin_clz(rows), cols, (cudaStream_t)stream);
}
