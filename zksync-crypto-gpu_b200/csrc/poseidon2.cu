// Poseidon2 over Goldilocks (width 12, rate 8, capacity 4, x^7, 4+22+4 rounds) for sm_100a:
// leaf hashing, node hashing, Merkle trees and query gathers.
//
// Replaces boojum-cuda's GLHasher kernels (crates/boojum-cuda/native/poseidon2/gl/*,
// native/poseidon2/queries.cuh) and GpuTreeHasher (crates/boojum-cuda/src/poseidon2.rs).
// Design:
//  * one thread per permutation with the 12-element state in registers; the linear layers are
//    evaluated lazily on 128-bit accumulators (shift-add only) and reduced once per round, and
//    the next round's constants are added before that reduction, so a round constant costs no
//    modular addition;
//  * round constants live in __constant__ memory (uniform across a warp: one broadcast read);
//  * Merkle node layers run as fused subtrees: one CTA hashes 2*T children down through
//    log2(2T) layers in shared memory, so a tree of 2^20 leaves needs 3 launches, not 20.
#include <algorithm>

#include "glc_field.cuh"
#include "glc_internal.h"

namespace glc {

static constexpr uint32_t ROUNDS = 30;
static constexpr uint32_t WIDTH = 12;

static constexpr uint64_t k_placeholder_rc[ROUNDS][WIDTH] = {
#include "p2_round_constants_placeholder.inc"
};

__constant__ uint64_t c_rc[ROUNDS][WIDTH] = {
#include "p2_round_constants_placeholder.inc"
};

// The constants as the external layer adds them: 2^52 + each 32-bit half, as doubles (see
// external_layer).  Rows 0..29: round r's constants; row 30: round 4's constant on element 0
// only (the layer before the partial rounds); row 31: none (the last layer).
static constexpr uint32_t RC_ROW_PARTIAL_ENTRY = 30, RC_ROW_NONE = 31;
struct ExternalConstants {
  double rcd[32][WIDTH][2];
};
static constexpr double TWO52 = 4503599627370496.0;
constexpr ExternalConstants make_external_constants(const uint64_t (&rc)[ROUNDS][WIDTH]) {
  ExternalConstants t{};
  for (uint32_t r = 0; r < 32; r++)
    for (uint32_t i = 0; i < WIDTH; i++) {
      const uint64_t v = r < ROUNDS ? rc[r][i] : (r == RC_ROW_PARTIAL_ENTRY && i == 0 ? rc[4][0] : 0);
      t.rcd[r][i][0] = TWO52 + (double)(uint32_t)v;
      t.rcd[r][i][1] = TWO52 + (double)(uint32_t)(v >> 32);
    }
  return t;
}
__constant__ ExternalConstants c_ext = make_external_constants(k_placeholder_rc);

static bool g_rc_installed[MAX_DEVICES];

__device__ __forceinline__ uint64_t sbox(uint64_t x) {
  const uint64_t x2 = sqr(x);
  const uint64_t x3 = mul(x2, x);
  const uint64_t x4 = sqr(x2);
  return mul(x3, x4);
}

// ---- M_E = circ(2 M4, M4, M4) (poseidon2_gl_st.cuh:35-55) on the FP64 pipe ----
// Evaluated as out_t = M4 (x_t + x_0 + x_1 + x_2) separately on the low and the high 32-bit
// halves of the state.  Every intermediate is an integer below 2^40, so double-precision adds
// and multiply-adds by 2 and 4 are exact: the layer runs on the otherwise idle FP64 pipe while
// the integer pipes carry the S-box products.  The results come back through the exponent
// trick: for an integer 0 <= x < 2^52, the bits of x + 2^52 are 0x433 << 52 | x, and the
// addend 2^52 + (half of the next round's constant) adds that constant for free.  fold() then
// combines the two halves into one 64-bit value.  Measured on B200: 2.4% faster per
// permutation than the same layer in 64-bit integer adds.

// M4 of eprint 2023/323 Appendix B (poseidon2_gl.cuh:11-25)
__device__ __forceinline__ void m4(double &x0, double &x1, double &x2, double &x3) {
  const double t0 = x0 + x1, t1 = x2 + x3;
  const double t2 = fma(x1, 2.0, t1), t3 = fma(x3, 2.0, t0);
  const double t4 = fma(t1, 4.0, t3), t5 = fma(t0, 4.0, t2);
  x0 = t3 + t5;
  x1 = t5;
  x2 = t2 + t4;
  x3 = t4;
}

// s <- M_E s + the constants of row `row` of c_ext
__device__ __forceinline__ void external_layer(uint64_t s[WIDTH], uint32_t row) {
  double xl[WIDTH], xh[WIDTH];
#pragma unroll
  for (int i = 0; i < WIDTH; i++) {
    xl[i] = (double)lo32(s[i]);
    xh[i] = (double)hi32(s[i]);
  }
  double L[WIDTH], H[WIDTH];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const double sl = xl[j] + xl[4 + j] + xl[8 + j];
    const double sh = xh[j] + xh[4 + j] + xh[8 + j];
#pragma unroll
    for (int t = 0; t < 3; t++) {
      L[4 * t + j] = sl + xl[4 * t + j];
      H[4 * t + j] = sh + xh[4 * t + j];
    }
  }
#pragma unroll
  for (int t = 0; t < 3; t++) {
    m4(L[4 * t], L[4 * t + 1], L[4 * t + 2], L[4 * t + 3]);
    m4(H[4 * t], H[4 * t + 1], H[4 * t + 2], H[4 * t + 3]);
  }
  const double(*rcd)[2] = c_ext.rcd[row];
#pragma unroll
  for (int i = 0; i < WIDTH; i++) {
    const uint64_t A = (uint64_t)__double_as_longlong(L[i] + rcd[i][0]) & 0x000FFFFFFFFFFFFFull;
    const uint64_t B = (uint64_t)__double_as_longlong(H[i] + rcd[i][1]) & 0x000FFFFFFFFFFFFFull;
    s[i] = fold(A, B);
  }
}

// ---- M_I = J + diag(2^LOG_MU_MINUS_ONE) (poseidon2_gl_st.cuh:57-65) ----
// 96-bit lazy sums with carry chains (ALU pipe: the S-box products already load the IMAD pipe),
// one 96 -> 64 fold per element.
struct w96 {
  uint32_t l0, l1, h;
};
__device__ __forceinline__ w96 w_from(uint64_t x) { return {lo32(x), hi32(x), 0u}; }
__device__ __forceinline__ w96 w_add(w96 a, w96 b) {
  w96 r;
  asm("add.cc.u32 %0, %3, %6;\n\taddc.cc.u32 %1, %4, %7;\n\taddc.u32 %2, %5, %8;"
      : "=r"(r.l0), "=r"(r.l1), "=r"(r.h)
      : "r"(a.l0), "r"(a.l1), "r"(a.h), "r"(b.l0), "r"(b.l1), "r"(b.h));
  return r;
}
__device__ __forceinline__ w96 w_add64(uint64_t a, uint64_t b) {
  w96 r;
  asm("add.cc.u32 %0, %3, %5;\n\taddc.cc.u32 %1, %4, %6;\n\taddc.u32 %2, 0, 0;"
      : "=r"(r.l0), "=r"(r.l1), "=r"(r.h)
      : "r"(lo32(a)), "r"(hi32(a)), "r"(lo32(b)), "r"(hi32(b)));
  return r;
}
__device__ __forceinline__ w96 w_shl64(uint64_t x, int k) {  // x * 2^k, k < 32
  w96 r;
  const uint32_t x0 = lo32(x), x1 = hi32(x);
  r.h = k ? x1 >> (32 - k) : 0u;
  r.l1 = __funnelshift_l(x0, x1, k);
  r.l0 = x0 << k;
  return r;
}
// 96 -> 64: h * 2^64 + l == l + h * EPS; one carry correction (h < 2^31)
__device__ __forceinline__ uint64_t w_red(w96 a) {
  uint32_t v0, v1;
  asm("{\n\t.reg .u32 u0, u1, c;\n\t"
      "sub.cc.u32 u0, 0, %4;\n\tsubc.u32 u1, %4, 0;\n\t"
      "add.cc.u32 %0, %2, u0;\n\taddc.cc.u32 %1, %3, u1;\n\taddc.u32 c, 0, 0;\n\t"
      "neg.s32 c, c;\n\tadd.cc.u32 %0, %0, c;\n\taddc.u32 %1, %1, 0;\n\t}"
      : "=r"(v0), "=r"(v1)
      : "r"(a.l0), "r"(a.l1), "r"(a.h));
  return pack(v0, v1);
}

__device__ __forceinline__ w96 w_shl(w96 a, int k) {  // a * 2^k, k < 32, no overflow of 96 bits
  w96 r;
  r.h = __funnelshift_l(a.l1, a.h, k);
  r.l1 = __funnelshift_l(a.l0, a.l1, k);
  r.l0 = a.l0 << k;
  return r;
}
// Partial 96 -> 65-bit reduction (h < 2^31): h * 2^64 + l == l + h * EPS = (h * EPS + l0) + l1 * 2^32,
// kept as a 96-bit value < 2^65 (one mad.wide, one carry add).
__device__ __forceinline__ w96 w_partial(w96 a) {
  const uint64_t t = madw(a.h, 0xFFFFFFFFu, (uint64_t)a.l0);
  w96 r;
  r.l0 = lo32(t);
  asm("add.cc.u32 %0, %2, %3;\n\taddc.u32 %1, 0, 0;" : "=r"(r.l1), "=r"(r.h) : "r"(hi32(t)), "r"(a.l1));
  return r;
}

// The 22 partial rounds with s1..s11 kept partially reduced in 96 bits: only s0 enters the
// S-box, so only s0 is fully reduced each round.  Rounds alternate: REDUCE = false skips the
// partial reduction of s1..s11, REDUCE = true applies it.  Bounds, starting from values
// < 2^65: a round without reduction sums 12 values (< 2^69) and adds 2^14 * s_i (< 2^79), so
// every s_i < 2^80; the next round sums to < 2^84 and shifts to < 2^94, so s_i < 2^95 and the
// top word stays below 2^31, which w_partial and w_red need; w_partial then brings s_i back
// below 2^65.
template <bool REDUCE>
__device__ __forceinline__ void internal_lazy(uint64_t &s0, w96 t[WIDTH], uint64_t rc0) {
  constexpr int LOG_MU_MINUS_ONE[WIDTH] = {4, 14, 11, 8, 0, 5, 2, 9, 13, 6, 3, 12};
  // t[1..11] do not depend on this round's S-box output: sum them as a tree (depth 4) that runs
  // beside the S-box, so only one add stands between the S-box and the new state
  const w96 a = w_add(t[1], t[2]), b = w_add(t[3], t[4]), c = w_add(t[5], t[6]), d = w_add(t[7], t[8]);
  const w96 e = w_add(w_add(t[9], t[10]), t[11]);
  const w96 sum = w_add(w_add(w_add(a, b), w_add(c, d)), w_add(e, w_from(s0)));
  s0 = w_red(w_add(w_add(sum, w_shl64(s0, LOG_MU_MINUS_ONE[0])), w_from(rc0)));
#pragma unroll
  for (int i = 1; i < WIDTH; i++) {
    const w96 v = w_add(sum, w_shl(t[i], LOG_MU_MINUS_ONE[i]));
    t[i] = REDUCE ? w_partial(v) : v;
  }
}

template <int MODE>
__device__ __forceinline__ void internal_layer(uint64_t s[WIDTH], const uint64_t *rc) {
  constexpr int LOG_MU_MINUS_ONE[WIDTH] = {4, 14, 11, 8, 0, 5, 2, 9, 13, 6, 3, 12};
  w96 sum = w_add64(s[0], s[1]);
#pragma unroll
  for (int i = 2; i < WIDTH; i++) sum = w_add(sum, w_from(s[i]));
#pragma unroll
  for (int i = 0; i < WIDTH; i++) {
    w96 v = w_add(sum, w_shl64(s[i], LOG_MU_MINUS_ONE[i]));
    if (MODE == 1 || (MODE == 2 && i == 0)) v = w_add(v, w_from(rc[i]));
    s[i] = w_red(v);
  }
}

// The 22 partial rounds plus the last one's internal layer, which adds round 26's constants.
template <bool ROLLED, bool LAZY>
__device__ __forceinline__ void partial_rounds(uint64_t s[WIDTH]) {
  if (!LAZY) {
    if (ROLLED) {
#pragma unroll 1
      for (int r = 4; r < 25; r++) {
        s[0] = sbox(s[0]);
        internal_layer<2>(s, c_rc[r + 1]);
      }
    } else {
#pragma unroll
      for (int r = 4; r < 25; r++) {
        s[0] = sbox(s[0]);
        internal_layer<2>(s, c_rc[r + 1]);
      }
    }
  } else {
    w96 t[WIDTH];
#pragma unroll
    for (int i = 1; i < WIDTH; i++) t[i] = w_from(s[i]);
    uint64_t s0 = s[0];
    // rounds 4..23 in pairs (without, then with the partial reduction), then round 24
    if (ROLLED) {
#pragma unroll 1
      for (int r = 4; r < 24; r += 2) {
        s0 = sbox(s0);
        internal_lazy<false>(s0, t, c_rc[r + 1][0]);
        s0 = sbox(s0);
        internal_lazy<true>(s0, t, c_rc[r + 2][0]);
      }
    } else {
#pragma unroll
      for (int r = 4; r < 24; r += 2) {
        s0 = sbox(s0);
        internal_lazy<false>(s0, t, c_rc[r + 1][0]);
        s0 = sbox(s0);
        internal_lazy<true>(s0, t, c_rc[r + 2][0]);
      }
    }
    s0 = sbox(s0);
    internal_lazy<true>(s0, t, c_rc[25][0]);
    s[0] = s0;
#pragma unroll
    for (int i = 1; i < WIDTH; i++) s[i] = w_red(t[i]);
  }
  s[0] = sbox(s[0]);
  internal_layer<1>(s, c_rc[26]);
}

// Poseidon2 permutation (poseidon2_gl_st.cu:9-23): M_E, 4 full rounds, 22 partial, 4 full.
// Round r's constants are added by the linear layer that precedes it.  ROLL = 0 unrolls every
// round; ROLL = 1 keeps the 22 partial rounds in a loop; ROLL = 2 also runs the 8 full rounds
// through one loop body (about a quarter of the code: the unrolled permutation is larger than
// the instruction cache, and warps at different rounds evict each other's code).  LAZY keeps
// s1..s11 partially reduced between partial rounds.  The autotuner picks per device.
template <int ROLL, bool LAZY>
__device__ __forceinline__ void permutation(uint64_t s[WIDTH]) {
  external_layer(s, 0);
  if (ROLL == 2) {
#pragma unroll 1
    for (int q = 0; q < 8; q++) {
#pragma unroll
      for (int i = 0; i < WIDTH; i++) s[i] = sbox(s[i]);
      // full round r = q (q < 4) or q + 22; the layer after it adds round r + 1's constants:
      // all of them, only element 0's before the partial rounds (q == 3), none after the last
      const int r = q < 4 ? q : q + 22;
      external_layer(s, q == 7 ? RC_ROW_NONE : (q == 3 ? RC_ROW_PARTIAL_ENTRY : (uint32_t)(r + 1)));
      if (q == 3) partial_rounds<true, LAZY>(s);
    }
  } else {
#pragma unroll
    for (int r = 0; r < 4; r++) {
#pragma unroll
      for (int i = 0; i < WIDTH; i++) s[i] = sbox(s[i]);
      external_layer(s, r < 3 ? (uint32_t)(r + 1) : RC_ROW_PARTIAL_ENTRY);
    }
    partial_rounds<ROLL == 1, LAZY>(s);
#pragma unroll
    for (int r = 26; r < 30; r++) {
#pragma unroll
      for (int i = 0; i < WIDTH; i++) s[i] = sbox(s[i]);
      external_layer(s, r < 29 ? (uint32_t)(r + 1) : RC_ROW_NONE);
    }
  }
#pragma unroll
  for (int i = 0; i < WIDTH; i++) s[i] = canon(s[i]);
}

// Leaf hashes (poseidon2_gl_st.cu:25-59): leaf i absorbs values[(i<<r) + row + col*rows*count]
// column by column, rows within a column, 8 per permutation into state[0..8) (overwrite),
// zero-padding the last chunk.  Capacity state[8..12) starts at 0 or is loaded from results.
// Register cap: MINB = 2 allows 128 registers (two 256-thread CTAs per SM), MINB = 3 allows 85
// (three 256-thread CTAs), MINB = 5 allows 102 with at most 128 threads per CTA (five CTAs).
__host__ __device__ constexpr int leaf_max_threads(int minb) { return minb == 5 ? 128 : 256; }
// The leaf hash of leaf gid (one thread's work in p2_leaves_kernel and in the fused batch kernel).
template <int ROLL, bool LAZY>
__device__ __forceinline__ void leaf_hash(const uint64_t *values, uint64_t *results, uint32_t log_rows, uint64_t cols,
                                          uint64_t count, bool load_intermediate, bool store_intermediate,
                                          uint64_t gid) {
  uint64_t s[WIDTH];
#pragma unroll
  for (int i = 0; i < WIDTH; i++) s[i] = 0;
  if (load_intermediate) {
#pragma unroll
    for (int k = 0; k < 4; k++) s[8 + k] = results[gid + k * count];
  }
  const uint64_t rows = 1ull << log_rows;
  const uint64_t total = rows * cols;
  const uint64_t *v = values + (gid << log_rows);
  const uint64_t col_stride = rows * count;
  // value o of this leaf: row o % rows of column o / rows.  The next chunk's 8 values are loaded
  // before the current permutation runs, so the DRAM latency of 8 column streams hides behind
  // ~14K instructions of hashing.  One permutation call site keeps the code small.
  uint64_t nxt[8];
#pragma unroll
  for (int i = 0; i < 8; i++)
    nxt[i] = (uint64_t)i < total ? __ldcs(v + ((uint64_t)i & (rows - 1)) + ((uint64_t)i >> log_rows) * col_stride) : 0;
  for (uint64_t off = 0; off < total; off += 8) {
#pragma unroll
    for (int i = 0; i < 8; i++) s[i] = nxt[i];
    if (off + 8 < total) {
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const uint64_t o = off + 8 + i;
        nxt[i] = o < total ? __ldcs(v + (o & (rows - 1)) + (o >> log_rows) * col_stride) : 0;
      }
    }
    permutation<ROLL, LAZY>(s);
  }
#pragma unroll
  for (int k = 0; k < 4; k++) results[gid + k * count] = canon(store_intermediate ? s[8 + k] : s[k]);
}

template <int ROLL, bool LAZY, int MINB>
__global__ void __launch_bounds__(leaf_max_threads(MINB), MINB) p2_leaves_kernel(const uint64_t *values, uint64_t *results, uint32_t log_rows,
                                                        uint64_t cols, uint64_t count, bool load_intermediate,
                                                        bool store_intermediate) {
  const uint64_t gid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= count) return;
  leaf_hash<ROLL, LAZY>(values, results, log_rows, cols, count, load_intermediate, store_intermediate, gid);
}

// Node hashes (poseidon2_gl_st.cu:61-82): node i = P2(L0..L3, R0..R3, 0,0,0,0)[0..4] with
// L, R = digests 2i and 2i+1 of the [4][2*count] input layer.
template <int ROLL, bool LAZY>
__device__ __forceinline__ void hash_node(const uint64_t l[4], const uint64_t r[4], uint64_t out[4]) {
  uint64_t s[WIDTH];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    s[k] = l[k];
    s[4 + k] = r[k];
    s[8 + k] = 0;
  }
  permutation<ROLL, LAZY>(s);
#pragma unroll
  for (int k = 0; k < 4; k++) out[k] = s[k];
}

// Children 2i and 2i+1 of row k of a [4][2*count] layer: one 16-byte load when the layer is
// 16-byte aligned (always, for layers inside a tree buffer), else two 8-byte loads.
__device__ __forceinline__ void load_children(const uint64_t *layer, uint64_t count, uint64_t i, uint64_t l[4],
                                              uint64_t r[4], bool aligned) {
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (aligned) {
      const ulonglong2 lr = __ldcs(reinterpret_cast<const ulonglong2 *>(layer + k * 2 * count) + i);
      l[k] = lr.x;
      r[k] = lr.y;
    } else {
      l[k] = __ldcs(layer + k * 2 * count + 2 * i);
      r[k] = __ldcs(layer + k * 2 * count + 2 * i + 1);
    }
  }
}

template <int ROLL, bool LAZY>
__global__ void __launch_bounds__(256) p2_nodes_kernel(const uint64_t *values, uint64_t *results, uint64_t count,
                                                       bool aligned) {
  const uint64_t gid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= count) return;
  uint64_t l[4], r[4], o[4];
  load_children(values, count, gid, l, r, aligned);
  hash_node<ROLL, LAZY>(l, r, o);
#pragma unroll
  for (int k = 0; k < 4; k++) results[k * count + gid] = o[k];
}

// Fused node layers: the CTA owns 2*T consecutive children of layer `in` ([4][2*count]) and
// produces up to `layers` parent layers, the j-th written to out_j ([4][count >> j] at
// out + offset of layer j).  out points at the first parent layer; each following layer starts
// right after the previous one (reference tree layout, poseidon2.rs:276-314).
template <uint32_t T, int ROLL, bool LAZY>
__global__ void __launch_bounds__(T) p2_subtree_kernel(const uint64_t *in, uint64_t *out, uint64_t count,
                                                       uint32_t layers, bool aligned) {
  __shared__ uint64_t sh[4][T];
  const uint32_t tid = threadIdx.x;
  uint64_t layer_count = count;          // nodes in the layer being produced
  uint64_t node = (uint64_t)blockIdx.x * T + tid;  // this thread's node in that layer
  uint64_t *dst = out;
  uint32_t active = T;
  // first layer: children straight from global memory
  {
    uint64_t l[4], r[4], o[4];
    const bool live = node < layer_count;
    if (live) {
      load_children(in, layer_count, node, l, r, aligned);
      hash_node<ROLL, LAZY>(l, r, o);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        dst[k * layer_count + node] = o[k];
        sh[k][tid] = o[k];
      }
    }
  }
  for (uint32_t j = 1; j < layers && active > 1; j++) {
    __syncthreads();
    dst += 4 * layer_count;
    layer_count >>= 1;
    active >>= 1;
    node = (uint64_t)blockIdx.x * active + tid;
    uint64_t o[4];
    const bool live = tid < active && node < layer_count;
    if (live) {
      uint64_t l[4], r[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        l[k] = sh[k][2 * tid];
        r[k] = sh[k][2 * tid + 1];
      }
      hash_node<ROLL, LAZY>(l, r, o);
#pragma unroll
      for (int k = 0; k < 4; k++) dst[k * layer_count + node] = o[k];
    }
    __syncthreads();
    if (live) {
#pragma unroll
      for (int k = 0; k < 4; k++) sh[k][tid] = o[k];
    }
  }
}

// gather_rows (queries.cuh:9-19)
__global__ void p2_gather_rows_kernel(const uint32_t *indexes, uint32_t indexes_count, uint32_t log_rows_per_index,
                                      const uint64_t *values, uint64_t values_stride, uint64_t *results,
                                      uint64_t results_stride, uint64_t cols) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t rows_out = (uint64_t)indexes_count << log_rows_per_index;
  if (t >= rows_out) return;
  const uint64_t idx = t >> log_rows_per_index, x = t & ((1ull << log_rows_per_index) - 1);
  const uint64_t src_row = ((uint64_t)indexes[idx] << log_rows_per_index) + x;
  for (uint64_t c = blockIdx.y; c < cols; c += gridDim.y)
    results[c * results_stride + t] = values[c * values_stride + src_row];
}

// gather_merkle_paths (queries.cuh:21-37)
__global__ void p2_gather_paths_kernel(const uint32_t *indexes, uint32_t indexes_count, const uint64_t *values,
                                       uint32_t log_leaves, uint64_t *results, uint32_t layers) {
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= indexes_count) return;
  const uint32_t col = blockIdx.y, layer = blockIdx.z;
  if (layer >= layers) return;
  const uint64_t layer_off = (4ull << (log_leaves + 1)) - (4ull << (log_leaves + 1 - layer));
  const uint64_t col_off = (uint64_t)col << (log_leaves - layer);
  const uint64_t hash_idx = (uint64_t)(indexes[idx] >> layer) ^ 1u;
  results[(uint64_t)layer * indexes_count * 4 + (uint64_t)indexes_count * col + idx] = values[layer_off + col_off + hash_idx];
}

// ---- launchers ----

P2Tuning g_p2_tuning[MAX_DEVICES];

P2Tuning &p2_tuning() {
  int dev = 0;
  cudaGetDevice(&dev);
  return g_p2_tuning[(dev >= 0 && dev < MAX_DEVICES) ? dev : 0];
}

template <int ROLL, bool LAZY>
static void leaves_go(uint32_t minb, uint32_t blocks, uint32_t threads, cudaStream_t stream, const uint64_t *values,
                      uint64_t *results, uint32_t log_rows, uint64_t cols, uint64_t count, bool li, bool si) {
  if (minb == 5 && threads <= 128)
    p2_leaves_kernel<ROLL, LAZY, 5><<<blocks, threads, 0, stream>>>(values, results, log_rows, cols, count, li, si);
  else if (minb >= 3)
    p2_leaves_kernel<ROLL, LAZY, 3><<<blocks, threads, 0, stream>>>(values, results, log_rows, cols, count, li, si);
  else
    p2_leaves_kernel<ROLL, LAZY, 2><<<blocks, threads, 0, stream>>>(values, results, log_rows, cols, count, li, si);
}

// Calls F<ROLL, LAZY>() for the tuned variant.
#define GLC_P2_VARIANT(tu, F)             \
  do {                                    \
    if ((tu).rolled >= 2 && (tu).lazy)    \
      F(2, true);                         \
    else if ((tu).rolled >= 2)            \
      F(2, false);                        \
    else if ((tu).rolled && (tu).lazy)    \
      F(1, true);                         \
    else if ((tu).rolled)                 \
      F(1, false);                        \
    else if ((tu).lazy)                   \
      F(0, true);                         \
    else                                  \
      F(0, false);                        \
  } while (0)

int p2_leaves_launch(const uint64_t *values, uint64_t *results, uint32_t log_rows, uint64_t cols, uint64_t count,
                     bool load_intermediate, bool store_intermediate, cudaStream_t stream) {
  if (count == 0) return 0;
  const P2Tuning &tu = p2_tuning();
  const uint32_t threads = tu.leaf_threads;
  const uint64_t blocks = (count + threads - 1) / threads;
  if (blocks > 0x7fffffffull) return fail("poseidon2: too many leaves");
#define GLC_LEAVES(R, L) leaves_go<R, L>(tu.min_blocks, (uint32_t)blocks, threads, stream, values, results, log_rows, \
                                         cols, count, load_intermediate, store_intermediate)
  GLC_P2_VARIANT(tu, GLC_LEAVES);
#undef GLC_LEAVES
  return last_launch_error();
}

int p2_nodes_launch(const uint64_t *values, uint64_t *results, uint64_t count, cudaStream_t stream) {
  if (count == 0) return 0;
  const P2Tuning &tu = p2_tuning();
  const uint32_t threads = tu.leaf_threads;
  const uint64_t blocks = (count + threads - 1) / threads;
  if (blocks > 0x7fffffffull) return fail("poseidon2: too many nodes");
  const bool aligned = (reinterpret_cast<uintptr_t>(values) & 15) == 0;
#define GLC_NODES(R, L) p2_nodes_kernel<R, L><<<(uint32_t)blocks, threads, 0, stream>>>(values, results, count, aligned)
  GLC_P2_VARIANT(tu, GLC_NODES);
#undef GLC_NODES
  return last_launch_error();
}

int p2_tree_nodes_launch(uint64_t *layer0, uint64_t leaves, uint32_t layers, cudaStream_t stream) {
  constexpr uint32_t T = 128;
  const uint64_t *in = layer0;
  uint64_t *out = layer0 + 4 * leaves;
  uint64_t count = leaves >> 1;  // nodes of the first layer to produce
  uint32_t remaining = layers;
  // Wide layers: one launch per layer keeps every thread busy.  Once a layer no longer fills
  // the GPU a few times over, fused subtree launches cover up to 8 layers each, so the narrow
  // top of the tree costs a handful of launches instead of one per layer.
  const uint64_t wide = 148ull * 128;
  while (remaining > 0 && count >= wide) {
    const int e = p2_nodes_launch(in, out, count, stream);
    if (e) return e;
    in = out;
    out += 4 * count;
    count >>= 1;
    remaining--;
  }
  while (remaining > 0) {
    // one launch covers up to log2(T)+1 layers (T threads -> 1 node)
    uint32_t l = 1;
    while (l < remaining && (T >> l) >= 1 && l < 8) l++;
    const uint64_t blocks = (count + T - 1) / T;
    if (blocks > 0x7fffffffull) return fail("poseidon2: too many nodes");
    const bool aligned = (reinterpret_cast<uintptr_t>(in) & 15) == 0;
    const P2Tuning &tu = p2_tuning();
#define GLC_SUB(R, L) p2_subtree_kernel<T, R, L><<<(uint32_t)blocks, T, 0, stream>>>(in, out, count, l, aligned)
    GLC_P2_VARIANT(tu, GLC_SUB);
#undef GLC_SUB
    const int e = last_launch_error();
    if (e) return e;
    // advance past the l layers just written
    for (uint32_t j = 0; j < l; j++) {
      in = out;
      out += 4 * count;
      count >>= 1;
    }
    remaining -= l;
  }
  return 0;
}

int p2_install_round_constants(const uint64_t *rc) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  e = cudaMemcpyToSymbol(c_rc, rc, sizeof(uint64_t) * ROUNDS * WIDTH);
  if (e == cudaSuccess) {
    uint64_t t[ROUNDS][WIDTH];
    for (uint32_t r = 0; r < ROUNDS; r++)
      for (uint32_t i = 0; i < WIDTH; i++) t[r][i] = rc[r * WIDTH + i];
    static ExternalConstants ext;  // large; built on the host, copied once
    ext = make_external_constants(t);
    e = cudaMemcpyToSymbol(c_ext, &ext, sizeof(ext));
  }
  if (e == cudaSuccess && dev >= 0 && dev < MAX_DEVICES) g_rc_installed[dev] = true;
  return (int)e;
}

bool p2_constants_installed() {
  int dev = 0;
  cudaGetDevice(&dev);
  return dev >= 0 && dev < MAX_DEVICES && g_rc_installed[dev];
}

}  // namespace glc

using namespace glc;

extern "C" glc_status glc_poseidon2_set_round_constants(const uint64_t *round_constants) {
  if (!round_constants) return fail("poseidon2: null round constants");
  return p2_install_round_constants(round_constants);
}

extern "C" glc_status glc_poseidon2_round_constants_installed(uint32_t *out) {
  if (!out) return fail("poseidon2: null output");
  *out = p2_constants_installed() ? 1u : 0u;
  return 0;
}

extern "C" glc_status glc_poseidon2_compute_leaf_hashes(const uint64_t *values, size_t values_len, uint64_t *results,
                                                        size_t results_len, uint32_t log_rows_per_hash,
                                                        bool load_intermediate, bool store_intermediate,
                                                        void *stream) {
  // poseidon2.rs:188-209
  if (results_len % 4) return fail("compute_leaf_hashes: results_len must be a multiple of 4");
  const uint64_t count = results_len / 4;
  if (log_rows_per_hash >= 32) return fail("compute_leaf_hashes: log_rows_per_hash too large");
  const uint64_t per = count << log_rows_per_hash;
  if (per == 0 || values_len % per) return fail("compute_leaf_hashes: values_len must be a multiple of count << log_rows_per_hash");
  const uint64_t rows = 1ull << log_rows_per_hash;
  const uint64_t cols = values_len / per;
  if (store_intermediate && (rows * cols) % 8)
    return fail("compute_leaf_hashes: a checkpointed column slab must fill whole rate-8 chunks");
  if (cols > 0xffffffffull || count > 0xffffffffull) return fail("compute_leaf_hashes: sizes exceed u32");
  return p2_leaves_launch(values, results, log_rows_per_hash, cols, count, load_intermediate, store_intermediate,
                          (cudaStream_t)stream);
}

extern "C" glc_status glc_poseidon2_compute_node_hashes(const uint64_t *values, size_t values_len, uint64_t *results,
                                                        size_t results_len, void *stream) {
  // poseidon2.rs:233-242
  if (values_len % 8) return fail("compute_node_hashes: values_len must be a multiple of 8");
  if (results_len % 4) return fail("compute_node_hashes: results_len must be a multiple of 4");
  if (values_len != results_len * 2) return fail("compute_node_hashes: values_len must be 2 * results_len");
  if (results_len / 4 > 0xffffffffull) return fail("compute_node_hashes: too many nodes");
  return p2_nodes_launch(values, results, results_len / 4, (cudaStream_t)stream);
}

extern "C" glc_status glc_poseidon2_build_merkle_tree_leaves(const uint64_t *values, size_t values_len,
                                                             uint64_t *results, size_t results_len,
                                                             uint32_t log_rows_per_hash, bool load_intermediate,
                                                             bool store_intermediate, void *stream) {
  // poseidon2.rs:261-265
  if (results_len % 4) return fail("build_merkle_tree_leaves: results_len must be a multiple of 4");
  const uint64_t leaves = results_len / 4;
  if (leaves == 0 || values_len % leaves) return fail("build_merkle_tree_leaves: values_len must be a multiple of leaves");
  return glc_poseidon2_compute_leaf_hashes(values, values_len, results, results_len, log_rows_per_hash,
                                           load_intermediate, store_intermediate, stream);
}

static int nodes_checked(const uint64_t *values, size_t values_len, uint64_t *results, size_t results_len,
                         uint32_t layers_count, cudaStream_t stream) {
  // poseidon2.rs:282-292, applied to every layer; then one fused launch sequence
  if (layers_count == 0) return 0;
  size_t len = values_len;
  for (uint32_t l = 0; l < layers_count; l++) {
    if (len % 8) return fail("build_merkle_tree_nodes: layer length must be a multiple of 8");
    const size_t v = len / 8;
    if (v & (v - 1)) return fail("build_merkle_tree_nodes: layer length must be 8 << layer");
    len /= 2;
  }
  if (values_len != results_len) return fail("build_merkle_tree_nodes: values_len must equal results_len");
  const uint64_t leaves = values_len / 4;
  if (values + values_len == results) return p2_tree_nodes_launch(const_cast<uint64_t *>(values), leaves, layers_count, stream);
  // layers of a tree whose leaves live elsewhere: first layer from `values`, then in place
  int e = p2_nodes_launch(values, results, leaves / 2, stream);
  if (e || layers_count == 1) return e;
  return p2_tree_nodes_launch(results, leaves / 2, layers_count - 1, stream);
}

extern "C" glc_status glc_poseidon2_build_merkle_tree_nodes(const uint64_t *values, size_t values_len,
                                                            uint64_t *results, size_t results_len,
                                                            uint32_t layers_count, void *stream) {
  return nodes_checked(values, values_len, results, results_len, layers_count, (cudaStream_t)stream);
}

extern "C" glc_status glc_poseidon2_build_merkle_tree(const uint64_t *values, size_t values_len, uint64_t *results,
                                                      size_t results_len, uint32_t log_rows_per_hash,
                                                      uint32_t layers_count, void *stream) {
  // poseidon2.rs:304-313
  if (layers_count == 0) return fail("build_merkle_tree: layers_count must be > 0");
  if (results_len % 8) return fail("build_merkle_tree: results_len must be a multiple of 8");
  const uint64_t leaves = results_len / 8;
  if (layers_count - 1 >= 64 || (1ull << (layers_count - 1)) > leaves)
    return fail("build_merkle_tree: 2^(layers_count-1) must be <= leaves");
  if (leaves == 0 || values_len % leaves) return fail("build_merkle_tree: values_len must be a multiple of leaves");
  const size_t half = results_len / 2;
  int e = glc_poseidon2_build_merkle_tree_leaves(values, values_len, results, half, log_rows_per_hash, false, false,
                                                 stream);
  if (e) return e;
  return nodes_checked(results, half, results + half, half, layers_count - 1, (cudaStream_t)stream);
}

extern "C" glc_status glc_poseidon2_gather_rows(const uint32_t *indexes, size_t indexes_len,
                                                uint32_t log_rows_per_index, const uint64_t *values,
                                                uint64_t values_rows, uint64_t values_cols, uint64_t values_stride,
                                                uint64_t *results, uint64_t results_rows, uint64_t results_cols,
                                                uint64_t results_stride, void *stream) {
  // poseidon2.rs:323-333
  if (log_rows_per_index >= 32) return fail("gather_rows: log_rows_per_index must be < 32");
  if (results_cols != values_cols) return fail("gather_rows: result cols must equal values cols");
  if (results_rows != ((uint64_t)indexes_len << log_rows_per_index))
    return fail("gather_rows: result rows must be indexes_len << log_rows_per_index");
  if (indexes_len > 0xffffffffull) return fail("gather_rows: too many indexes");
  if (values_stride < values_rows || results_stride < results_rows) return fail("gather_rows: stride < rows");
  if (results_rows == 0 || values_cols == 0) return 0;
  const uint32_t threads = 128;
  const uint64_t blocks = (results_rows + threads - 1) / threads;
  const uint32_t gy = (uint32_t)std::min<uint64_t>(values_cols, 65535);
  p2_gather_rows_kernel<<<dim3((uint32_t)blocks, gy), threads, 0, (cudaStream_t)stream>>>(
      indexes, (uint32_t)indexes_len, log_rows_per_index, values, values_stride, results, results_stride, values_cols);
  return last_launch_error();
}

extern "C" glc_status glc_poseidon2_gather_merkle_paths(const uint32_t *indexes, size_t indexes_len,
                                                        const uint64_t *values, size_t values_len, uint64_t *results,
                                                        size_t results_len, uint32_t layers_count, void *stream) {
  // poseidon2.rs:357-370
  if (indexes_len > 0xffffffffull) return fail("gather_merkle_paths: too many indexes");
  if (values_len % 4) return fail("gather_merkle_paths: values_len must be a multiple of 4");
  const uint64_t vc = values_len / 4;
  if (vc == 0 || (vc & (vc - 1))) return fail("gather_merkle_paths: values_len / 4 must be a power of two");
  const uint32_t log_vc = 63 - __builtin_clzll(vc);
  if (log_vc == 0) return fail("gather_merkle_paths: tree too small");
  const uint32_t log_leaves = log_vc - 1;
  if (layers_count > log_leaves) return fail("gather_merkle_paths: layers_count must be <= log2(leaves)");
  if ((uint64_t)indexes_len * layers_count * 4 != results_len)
    return fail("gather_merkle_paths: results_len must be indexes_len * layers_count * 4");
  if (indexes_len == 0 || layers_count == 0) return 0;
  const uint32_t threads = 32;
  const uint32_t blocks = (uint32_t)((indexes_len + threads - 1) / threads);
  p2_gather_paths_kernel<<<dim3(blocks, 4, layers_count), threads, 0, (cudaStream_t)stream>>>(
      indexes, (uint32_t)indexes_len, values, log_leaves, results, layers_count);
  return last_launch_error();
}

// The fused batch of small commitments (one cooperative launch), which uses this file's round
// constants and hash functions.
#include "fused.cuh"
