// NTT tile machinery shared by the per-pass kernels (ntt.cu) and the fused batch kernel: the pass
// arguments, the radix rounds on a shared-memory tile, one CTA's tile of a pass, and the host-side
// plan of the passes.  Header-only (inline and templates), so each translation unit that launches
// these kernels has its own copy; it holds no device state of its own.
#pragma once
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
static constexpr int NTT_SMEM_MAX = 140 * 1024;  // tile 68 KiB + twiddles 34 KiB + scaling tables 32 KiB (padded)

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

// Shared-memory slot of tile element e: one padding slot after every 16 elements.  Every radix
// round's accesses are free of bank conflicts in this layout (a warp's 32 8-byte accesses cover 16
// distinct bank pairs twice), and the map is additive on the index sets a round touches: for a
// round base b whose bits p .. p+R-1 are zero, pad(b | j << p) = pad(b) + pad(j << p), and
// pad(j << p) = j * pad(1 << p) when p >= 4.  A thread's 2^R slots are thus one base slot plus
// per-round offsets (multiples of one stride when p >= 4).
__host__ __device__ constexpr uint32_t pad(uint32_t e) { return e + (e >> 4); }
// Block twiddle idx (heap order: level l holds idx 2^l - 1 .. 2^(l+1) - 2) sits in slot
// pad(idx + 1) - 1: each level padded like the tile, so a thread's twiddles of one level are one
// base slot plus its small index.

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

template <uint32_t R, bool DIF, bool LIN>
__device__ __forceinline__ void radix_round(uint64_t *tile, const uint64_t *tws, uint32_t k, uint32_t log_w, uint32_t t) {
  const uint32_t log_e = k + log_w;
  const uint32_t p = k - t - R + log_w;  // lowest active bit of the tile index
  const uint32_t jobs = 1u << (log_e - R);
  const uint32_t S = pad(1u << p);       // slot stride of the round's elements when LIN (p >= 4)
  for (uint32_t q = threadIdx.x; q < jobs; q += blockDim.x) {
    const uint32_t base = ((q >> p) << (p + R)) | (q & ((1u << p) - 1));
    const uint32_t mid_base = base >> log_w;
    uint64_t *tb = tile + pad(base);
    uint64_t v[1 << R];
#pragma unroll
    for (uint32_t j = 0; j < (1u << R); j++) v[j] = tb[LIN ? j * S : pad(j << p)];
#pragma unroll
    for (uint32_t uu = 0; uu < R; uu++) {
      const uint32_t u = DIF ? R - 1 - uu : uu;
      const uint32_t level = t + u;
      const uint32_t bit = R - 1 - u;
      // twiddle m = mb + jj (jj < 2^u, mb with zero low u bits): slot pad(2^level + mb) - 1 + jj
      const uint64_t *tl = tws + pad((1u << level) + (mid_base >> (k - level))) - 1;
#pragma unroll
      for (uint32_t j = 0; j < (1u << R); j++) {
        if (j & (1u << bit)) continue;
        const uint64_t w = tl[j >> (R - u)];
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
    for (uint32_t j = 0; j < (1u << R); j++) tb[LIN ? j * S : pad(j << p)] = v[j];
  }
}

template <uint32_t R, bool DIF>
__device__ __forceinline__ void radix_round_p(uint64_t *tile, const uint64_t *tws, uint32_t k, uint32_t log_w, uint32_t t) {
  if (k + log_w >= t + R + 4)  // p >= 4: slots of the round's elements are multiples of one stride
    radix_round<R, DIF, true>(tile, tws, k, log_w, t);
  else
    radix_round<R, DIF, false>(tile, tws, k, log_w, t);
}

template <bool DIF, uint32_t RB>
__device__ __forceinline__ void round_dispatch(uint64_t *tile, const uint64_t *tws, uint32_t k, uint32_t log_w, uint32_t t,
                                               uint32_t r) {
  if (RB >= 4 && r == 4)
    radix_round_p<(RB >= 4 ? 4 : 1), DIF>(tile, tws, k, log_w, t);
  else if (RB >= 3 && r == 3)
    radix_round_p<(RB >= 3 ? 3 : 1), DIF>(tile, tws, k, log_w, t);
  else if (r == 2)
    radix_round<2, DIF, false>(tile, tws, k, log_w, t);
  else
    radix_round<1, DIF, false>(tile, tws, k, log_w, t);
}

// One CTA's share of a pass: tile bx of column group by (what the ntt_pass_kernel CTA with block
// coordinates (bx, by) computes).  Every thread of the CTA calls it; any block size works (the
// loops stride by blockDim.x).  smem holds the tile, the block twiddles and the scaling tables.
template <uint32_t RB>
__device__ __forceinline__ void ntt_pass_tile(const PassArgs &a, uint32_t bx, uint32_t by, uint64_t *smem) {
  const uint32_t k = a.k, log_w = a.log_w;
  const uint32_t E = 1u << (k + log_w);
  uint64_t *tile = smem;
  uint64_t *tws = smem + pad(E);
  const uint32_t log_m = a.log_n - a.s0 - k;
  const uint32_t log_tph = log_m - log_w;
  const uint32_t hi = bx >> log_tph;
  const uint32_t lo0 = (bx & ((1u << log_tph) - 1)) << log_w;
  const uint64_t base_i = ((uint64_t)hi << (a.log_n - a.s0)) + lo0;
  // block twiddle 2^t - 1 + m = T[hi * 2^t + m]: twiddles of stage s0 + t for this hi.
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
    tws[pad(idx + 1) - 1] = a.fold ? mul(w, sig[t]) : w;
  }
  // Coset / size scaling as two per-CTA tables: the exponent j of element (mid, w) splits as
  //   natural j = mid * M + (lo0 + w)                      (strided pass, hi = 0)
  //   bit-reversed j = bitrev_k(mid) << (L - k) + bitrev_{L-k}(hi)  (contiguous pass, W = 1)
  // so the factor is P[mid] * Q[w] (P carries N^-1 on the inverse side): 2 multiplies per element.
  uint64_t *Pt = tws + pad(1u << k);
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
  const uint32_t col0 = by * a.cols_per_cta;
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
        tile[pad(e)] = v.x;
        tile[pad(e + 1)] = v.y;
      }
    } else {
      for (uint32_t e = threadIdx.x; e < E; e += blockDim.x) {
        const uint64_t i = base_i + ((uint64_t)(e >> log_w) << log_m) + (e & wmask);
        uint64_t v = src[i];
        if (a.scale == 1) v = mul(v, mul(Pt[e >> log_w], Qt[a.j_bitrev ? 0u : (e & wmask)]));
        tile[pad(e)] = v;
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
        uint64_t v0 = tile[pad(e)], v1 = tile[pad(e + 1)];
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
        uint64_t v = tile[pad(e)];
        if (a.scale == 2)
          v = a.log_ext ? mul(v, mul(Pt[e >> log_w], Qt[a.j_bitrev ? 0u : (e & wmask)])) : mul(v, a.n_inv);
        dst[i] = a.last ? canon(v) : v;  // a following pass accepts any value below 2^64
      }
    }
  }
}


// ---- host side: the plan of an NTT and the arguments of each pass ----

struct Pass {
  uint32_t s0, k, log_w;
};

// Stage groups of an NTT of 2^log_n: one pass (log_n <= 12) or a strided pass then a contiguous
// one, each at most 12 stages; n2b runs them in increasing order, b2n in decreasing order.
static inline uint32_t make_plan(uint32_t log_n, bool b2n, const NttTuning &tu, Pass *passes) {
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
  for (uint32_t q = 0; q < np; q++) passes[q] = b2n ? p[np - 1 - q] : p[q];
  return np;
}

// Launch shape of one pass: tiles per column (grid x), column groups (grid y), dynamic shared
// memory and threads per CTA.
struct PassShape {
  uint64_t tiles_per_col;
  uint32_t groups;
  size_t smem;
  uint32_t threads;
};

// Arguments of pass q (of np) of a batch of `cols` NTTs, and its launch shape.
static inline PassShape make_pass(PassArgs &a, const DeviceTables *t, const NttTuning &tu, const Pass &ps,
                                  uint32_t q, uint32_t np, const uint64_t *in, uint64_t *out, uint64_t in_stride,
                                  uint64_t out_stride, uint32_t cols, uint32_t log_n, bool bitrev_inputs,
                                  bool inverse, uint32_t log_ext, uint32_t coset_idx, uint32_t max_cols_per_cta) {
  a = PassArgs{};
  a.in = q == 0 ? in : out;
  a.in_stride = q == 0 ? in_stride : out_stride;
  a.out = out;
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
  PassShape sh;
  sh.tiles_per_col = (1ull << log_n) >> tile_log;
  // enough CTAs to fill 148 SMs a few times over; the rest of the columns loop inside a CTA
  const uint64_t want = 148ull * 8;
  const uint32_t cpc =
      (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(max_cols_per_cta, (sh.tiles_per_col * cols) / want));
  a.cols_per_cta = cpc;
  sh.groups = (cols + cpc - 1) / cpc;
  // tile + block twiddles (+ the P/Q scaling tables on a scaled pass; the inverse NTT's last
  // pass without a coset multiplies by N^-1 only: no tables, and the 2^k-entry table it does not
  // need would cost a third CTA per SM on 2^12-element tiles)
  const bool tables = a.scale == 1 || (a.scale == 2 && a.log_ext);
  sh.smem = ((size_t)pad(1u << tile_log) + pad(1u << ps.k) +
             (tables ? (size_t(1) << ps.k) + (size_t(1) << ps.log_w) : 0)) * sizeof(uint64_t);
  sh.threads = (uint32_t)std::min<uint64_t>(pass_threads(tu.radix_bits),
                                            std::max<uint64_t>(32, (1ull << tile_log) >> tu.radix_bits));
  return sh;
}

}  // namespace glc
