/*
 * glc_oracle.c -- CPU oracle for the Goldilocks LDE + Poseidon2 Merkle commitment path.
 *
 * TEST INFRASTRUCTURE ONLY (see glc_oracle.h).  Plain, exact u128 arithmetic; clarity over
 * speed, with a pthread parallel-for so that the benchmark can time it as a CPU baseline on
 * all host cores.  Each function cites the reference code whose behaviour it restates.
 */
#include "glc_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------------------------
 * Field.  p = 2^64 - 2^32 + 1.  (crates/boojum-cuda/native/goldilocks.cuh:90-185: the
 * reference keeps values in [0, 2^64) and compares canonically; the oracle canonicalises.)
 * ---------------------------------------------------------------------------------------- */
/* Branch-free helpers (the carries are data-dependent, so branches would mispredict half the
 * time).  fr_* results are in [0, 2^64), congruent mod p but not necessarily canonical. */
static inline uint64_t fr_canon(uint64_t a) { return a >= OR_P ? a - OR_P : a; }

/* a + b: a carry out of 64 bits is worth EPS = 2^32 - 1; adding it can carry once more only
 * when the wrapped sum is >= p, and then the second EPS cannot carry (the wrapped sum is at most
 * 2^64 - 2). */
static inline uint64_t fr_add(uint64_t a, uint64_t b) {
  uint64_t s, s2;
  const uint64_t c1 = __builtin_add_overflow(a, b, &s);
  const uint64_t c2 = __builtin_add_overflow(s, 0xFFFFFFFFull & (0 - c1), &s2);
  return s2 + (0xFFFFFFFFull & (0 - c2));
}

/* 128-bit product reduced with 2^64 = 2^32 - 1 and 2^96 = -1 (mod p): with hi = hh:hl,
 * x = lo - hh + hl * (2^32 - 1).  A borrow in lo - hh leaves at least 2^64 - 2^32 + 1, so
 * subtracting EPS for it cannot borrow again; a carry in the final sum leaves less than
 * (2^32 - 1)^2, so adding EPS for it cannot carry again. */
static inline uint64_t fr_mul(uint64_t a, uint64_t b) {
  const u128 x = (u128)a * b;
  const uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
  const uint64_t hh = hi >> 32, hl = hi & 0xFFFFFFFFull;
  uint64_t t0, t2;
  const uint64_t br = __builtin_sub_overflow(lo, hh, &t0);
  t0 -= 0xFFFFFFFFull & (0 - br);
  const uint64_t t1 = hl * 0xFFFFFFFFull;
  const uint64_t cr = __builtin_add_overflow(t0, t1, &t2);
  return t2 + (0xFFFFFFFFull & (0 - cr));
}

uint64_t or_canon(uint64_t a) { return fr_canon(a); }

uint64_t or_add(uint64_t a, uint64_t b) { return fr_canon(fr_add(a, b)); }

uint64_t or_sub(uint64_t a, uint64_t b) {
  a = fr_canon(a);
  b = fr_canon(b);
  const uint64_t d = a - b;
  return a >= b ? d : d + OR_P;
}

uint64_t or_mul(uint64_t a, uint64_t b) { return fr_canon(fr_mul(a, b)); }

uint64_t or_pow(uint64_t a, uint64_t e) {
  uint64_t r = 1, x = or_canon(a);
  while (e) {
    if (e & 1) r = or_mul(r, x);
    x = or_mul(x, x);
    e >>= 1;
  }
  return r;
}

/* Fermat inverse (the reference uses binary GCD, goldilocks.cuh:280-304; same value). */
uint64_t or_inv(uint64_t a) { return or_pow(a, OR_P - 2); }

/* Multiplicative generator 7 (crates/boojum-cuda/src/context.rs:232). */
#define OR_GENERATOR 7ull

uint64_t or_root_of_unity(uint32_t log_n) { return or_pow(OR_GENERATOR, (OR_P - 1) >> log_n); }

static uint32_t or_bitrev(uint32_t x, uint32_t bits) {
  if (bits == 0) return 0;
  uint32_t r = 0;
  for (uint32_t i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

/* ------------------------------------------------------------------------------------------
 * Parallel-for over [0, n) with at most `threads` pthreads.
 * ---------------------------------------------------------------------------------------- */
typedef void (*or_range_fn)(void *ctx, size_t begin, size_t end);

typedef struct {
  or_range_fn fn;
  void *ctx;
  size_t begin, end;
} or_job;

static void *or_job_main(void *arg) {
  or_job *j = (or_job *)arg;
  j->fn(j->ctx, j->begin, j->end);
  return NULL;
}

static void or_parallel_for(size_t n, int threads, or_range_fn fn, void *ctx) {
  if (threads <= 1 || n <= 1) {
    fn(ctx, 0, n);
    return;
  }
  if ((size_t)threads > n) threads = (int)n;
  pthread_t *tids = (pthread_t *)malloc(sizeof(pthread_t) * threads);
  or_job *jobs = (or_job *)malloc(sizeof(or_job) * threads);
  size_t chunk = (n + threads - 1) / threads;
  int started = 0;
  for (int t = 0; t < threads; t++) {
    size_t b = t * chunk, e = b + chunk < n ? b + chunk : n;
    if (b >= e) break;
    jobs[t] = (or_job){fn, ctx, b, e};
    if (pthread_create(&tids[t], NULL, or_job_main, &jobs[t]) != 0) {
      fn(ctx, b, e); /* could not start a thread: run this range inline */
      jobs[t].fn = NULL;
    }
    started = t + 1;
  }
  for (int t = 0; t < started; t++)
    if (jobs[t].fn) pthread_join(tids[t], NULL);
  free(tids);
  free(jobs);
}

/* ------------------------------------------------------------------------------------------
 * NTT.  Definitions from the reference's test oracle (crates/boojum-cuda/src/ntt.rs:527-583,
 * boojum fft_natural_to_bitreversed / ifft_natural_to_natural):
 *   s = 1 if log_extension_degree == 0, else g * w_{N*2^e}^coset_idx  (ntt.rs:527-537)
 *   forward: X[i] = sum_j a_j (s w_N^i)^j              (evaluations of the coefficients a)
 *   inverse: a_j = N^-1 s^-j sum_i X[i] w_N^-ij        (coefficients of the evaluations X)
 *   n2b (bitrev_inputs = 0): natural-order input, bit-reversed output.
 *   b2n (bitrev_inputs = 1): bit-reversed input, natural-order output.
 * ---------------------------------------------------------------------------------------- */
static uint64_t or_coset_shift(uint32_t log_n, uint32_t log_ext, uint32_t coset_idx) {
  if (log_ext == 0) return 1;
  uint64_t w = or_root_of_unity(log_n + log_ext);
  return or_mul(OR_GENERATOR, or_pow(w, coset_idx));
}

static int or_ntt_check(uint32_t log_n, uint64_t in_stride, uint64_t out_stride, uint32_t log_ext, uint32_t coset_idx) {
  /* ntt.rs:192-200 */
  if (log_n < 1 || log_n + log_ext > 30) return -1;
  uint64_t n = 1ull << log_n;
  if (n > in_stride || n > out_stride) return -1;
  if (coset_idx > 0 && (log_ext == 0 || coset_idx >= (1u << log_ext))) return -1;
  return 0;
}

/* In-place natural-order DFT with root w (iterative radix-2: bit-reverse, then DIT). */
static void or_dft_natural(uint64_t *x, uint32_t log_n, uint64_t w, uint64_t *tw /* n/2 scratch */) {
  uint32_t n = 1u << log_n;
  for (uint32_t i = 0; i < n; i++) {
    uint32_t r = or_bitrev(i, log_n);
    if (r > i) {
      uint64_t t = x[i];
      x[i] = x[r];
      x[r] = t;
    }
  }
  tw[0] = 1;
  for (uint32_t i = 1; i < n / 2; i++) tw[i] = or_mul(tw[i - 1], w);
  for (uint32_t len = 2; len <= n; len <<= 1) {
    uint32_t half = len >> 1, step = n / len;
    for (uint32_t b = 0; b < n; b += len)
      for (uint32_t j = 0; j < half; j++) {
        uint64_t u = x[b + j], v = or_mul(x[b + j + half], tw[j * step]);
        x[b + j] = or_add(u, v);
        x[b + j + half] = or_sub(u, v);
      }
  }
}

typedef struct {
  const uint64_t *in;
  uint64_t *out;
  uint32_t log_n;
  uint64_t in_stride, out_stride;
  int bitrev_inputs, inverse;
  uint64_t s;
} or_ntt_ctx;

static void or_ntt_range(void *vctx, size_t begin, size_t end) {
  const or_ntt_ctx *c = (const or_ntt_ctx *)vctx;
  uint32_t n = 1u << c->log_n;
  uint64_t *x = (uint64_t *)malloc(sizeof(uint64_t) * n);
  uint64_t *tw = (uint64_t *)malloc(sizeof(uint64_t) * (n / 2 + 1));
  uint64_t w = or_root_of_unity(c->log_n);
  uint64_t n_inv = or_inv(n);
  uint64_t s_inv = or_inv(c->s);
  for (size_t k = begin; k < end; k++) {
    const uint64_t *src = c->in + k * c->in_stride;
    uint64_t *dst = c->out + k * c->out_stride;
    for (uint32_t j = 0; j < n; j++) x[j] = or_canon(src[c->bitrev_inputs ? or_bitrev(j, c->log_n) : j]);
    if (!c->inverse) {
      uint64_t sp = 1;
      for (uint32_t j = 0; j < n; j++, sp = or_mul(sp, c->s)) x[j] = or_mul(x[j], sp);
      or_dft_natural(x, c->log_n, w, tw);
    } else {
      or_dft_natural(x, c->log_n, or_inv(w), tw);
      uint64_t sp = n_inv;
      for (uint32_t j = 0; j < n; j++, sp = or_mul(sp, s_inv)) x[j] = or_mul(x[j], sp);
    }
    /* n2b writes bit-reversed, b2n writes natural; in place is safe since x is a copy */
    for (uint32_t i = 0; i < n; i++) dst[i] = x[c->bitrev_inputs ? i : or_bitrev(i, c->log_n)];
  }
  free(x);
  free(tw);
}

int or_batch_ntt(const uint64_t *in, uint64_t *out, uint32_t log_n, uint32_t num_ntts, uint64_t in_stride,
                 uint64_t out_stride, int bitrev_inputs, int inverse, uint32_t log_ext, uint32_t coset_idx,
                 int threads) {
  if (or_ntt_check(log_n, in_stride, out_stride, log_ext, coset_idx)) return -1;
  or_ntt_ctx c = {in, out, log_n, in_stride, out_stride, bitrev_inputs, inverse,
                  or_coset_shift(log_n, log_ext, coset_idx)};
  or_parallel_for(num_ntts, threads, or_ntt_range, &c);
  return 0;
}

int or_batch_ntt_naive(const uint64_t *in, uint64_t *out, uint32_t log_n, uint32_t num_ntts, uint64_t in_stride,
                       uint64_t out_stride, int bitrev_inputs, int inverse, uint32_t log_ext, uint32_t coset_idx) {
  if (or_ntt_check(log_n, in_stride, out_stride, log_ext, coset_idx)) return -1;
  uint32_t n = 1u << log_n;
  uint64_t s = or_coset_shift(log_n, log_ext, coset_idx);
  uint64_t w = or_root_of_unity(log_n);
  uint64_t *x = (uint64_t *)malloc(sizeof(uint64_t) * n);
  uint64_t *y = (uint64_t *)malloc(sizeof(uint64_t) * n);
  for (uint32_t k = 0; k < num_ntts; k++) {
    for (uint32_t j = 0; j < n; j++) x[j] = in[k * in_stride + (bitrev_inputs ? or_bitrev(j, log_n) : j)];
    for (uint32_t i = 0; i < n; i++) {
      uint64_t acc = 0;
      if (!inverse) {
        /* X[i] = sum_j x_j (s w^i)^j */
        uint64_t pt = or_mul(s, or_pow(w, i)), pj = 1;
        for (uint32_t j = 0; j < n; j++, pj = or_mul(pj, pt)) acc = or_add(acc, or_mul(x[j], pj));
      } else {
        /* a_i = N^-1 s^-i sum_j X[j] w^-ij */
        uint64_t pt = or_inv(or_pow(w, i)), pj = 1;
        for (uint32_t j = 0; j < n; j++, pj = or_mul(pj, pt)) acc = or_add(acc, or_mul(x[j], pj));
        acc = or_mul(acc, or_mul(or_inv(n), or_inv(or_pow(s, i))));
      }
      y[i] = acc;
    }
    for (uint32_t i = 0; i < n; i++) out[k * out_stride + i] = y[bitrev_inputs ? i : or_bitrev(i, log_n)];
  }
  free(x);
  free(y);
  return 0;
}

/* ops_complex.cu:88-156: per-column permutation x[i] <-> x[bitrev(i)]; src == dst allowed. */
void or_bit_reverse(const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride, uint32_t log_rows,
                    uint32_t cols) {
  uint32_t n = 1u << log_rows;
  uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * n);
  for (uint32_t c = 0; c < cols; c++) {
    for (uint32_t i = 0; i < n; i++) tmp[i] = src[c * src_stride + or_bitrev(i, log_rows)];
    memcpy(dst + c * dst_stride, tmp, sizeof(uint64_t) * n);
  }
  free(tmp);
}

/* GoldilocksExt2 layout conversions (goldilocks_extension.cu:8-34: element (row, col) read
 * through one accessor and written through the other). */
void or_ef_vectorized_to_tuples(const uint64_t *v, uint64_t v_stride, uint64_t *t, uint64_t t_stride, uint32_t rows,
                                uint32_t cols) {
  for (uint64_t k = 0; k < cols; k++)
    for (uint64_t r = 0; r < rows; r++) {
      t[2 * (k * t_stride + r)] = v[2 * k * v_stride + r];
      t[2 * (k * t_stride + r) + 1] = v[(2 * k + 1) * v_stride + r];
    }
}

void or_ef_tuples_to_vectorized(const uint64_t *t, uint64_t t_stride, uint64_t *v, uint64_t v_stride, uint32_t rows,
                                uint32_t cols) {
  for (uint64_t k = 0; k < cols; k++)
    for (uint64_t r = 0; r < rows; r++) {
      v[2 * k * v_stride + r] = t[2 * (k * t_stride + r)];
      v[(2 * k + 1) * v_stride + r] = t[2 * (k * t_stride + r) + 1];
    }
}

/* ---- witness-to-trace fill (ops_complex.cu:158-164; shivini trace.rs:108-193, cs/witness.rs:6-31) ---- */
void or_select(const uint32_t *indexes, uint64_t count, const uint64_t *src, uint64_t src_len, uint64_t *dst) {
  for (uint64_t i = 0; i < count; i++) {
    const uint32_t ix = indexes[i];
    dst[i] = (ix & 0x80000000u) || ix >= src_len ? 0 : src[ix];
  }
}

void or_trace_fill(const uint32_t *variable_indexes, const uint32_t *witness_indexes, const uint64_t *values,
                   uint64_t values_len, const uint32_t *multiplicities, uint64_t multiplicities_len, uint64_t *trace,
                   uint32_t nv, uint32_t nw, uint32_t nm, uint64_t n) {
  or_select(variable_indexes, (uint64_t)nv * n, values, values_len, trace);
  or_select(witness_indexes, (uint64_t)nw * n, values, values_len, trace + (uint64_t)nv * n);
  if (nm) {
    uint64_t *m = trace + (uint64_t)(nv + nw) * n;
    for (uint64_t i = 0; i < n; i++) m[i] = i < multiplicities_len ? (uint64_t)multiplicities[i] : 0;
  }
}

/* ------------------------------------------------------------------------------------------
 * Poseidon2 over Goldilocks, width 12, rate 8, capacity 4, x^7, 4+4 full and 22 partial
 * rounds (crates/boojum-cuda/native/poseidon2/gl/poseidon2_gl_st.cu:9-23,
 * poseidon2_gl_st.cuh:11-65, poseidon2_gl.cuh:11-25, poseidon2_gl_constants.cuh.template:6-20).
 * ---------------------------------------------------------------------------------------- */
static uint64_t g_rc[30][12];
/* M_I diagonal: 1 + 2^LOG_MU_MINUS_ONE[i] (poseidon2_gl_constants.cuh.template:17). */
static const uint32_t OR_LOG_MU_MINUS_ONE[12] = {4, 14, 11, 8, 0, 5, 2, 9, 13, 6, 3, 12};

void or_p2_set_round_constants(const uint64_t rc[30 * 12]) { memcpy(g_rc, rc, sizeof(g_rc)); }

/* m4 from eprint 2023/323 Appendix B (poseidon2_gl.cuh:11-25). */
static void or_m4(uint64_t *x) {
  uint64_t t0 = fr_add(x[0], x[1]);
  uint64_t t1 = fr_add(x[2], x[3]);
  uint64_t t2 = fr_add(fr_add(x[1], x[1]), t1);
  uint64_t t3 = fr_add(fr_add(x[3], x[3]), t0);
  uint64_t t4 = fr_add(fr_mul(t1, 4), t3);
  uint64_t t5 = fr_add(fr_mul(t0, 4), t2);
  uint64_t t6 = fr_add(t3, t5);
  uint64_t t7 = fr_add(t2, t4);
  x[0] = t6;
  x[1] = t5;
  x[2] = t7;
  x[3] = t4;
}

/* M_E = circ(2 M4, M4, M4) (poseidon2_gl_st.cuh:35-55). */
static void or_external(uint64_t *s) {
  for (int t = 0; t < 12; t += 4) or_m4(s + t);
  for (int j = 0; j < 4; j++) {
    uint64_t acc = fr_add(fr_add(s[j], s[4 + j]), s[8 + j]);
    for (int t = 0; t < 12; t += 4) s[t + j] = fr_add(s[t + j], acc);
  }
}

/* M_I = J + diag(2^LOG_MU_MINUS_ONE) (poseidon2_gl_st.cuh:57-65). */
static void or_internal(uint64_t *s) {
  uint64_t sum = 0;
  for (int i = 0; i < 12; i++) sum = fr_add(sum, s[i]);
  for (int i = 0; i < 12; i++) s[i] = fr_add(sum, fr_mul(s[i], 1ull << OR_LOG_MU_MINUS_ONE[i]));
}

static uint64_t or_sbox(uint64_t x) {
  uint64_t x2 = fr_mul(x, x), x3 = fr_mul(x2, x), x4 = fr_mul(x2, x2);
  return fr_mul(x3, x4);
}

/* Values stay in [0, 2^64) between the rounds and are canonicalised at the end. */
void or_p2_permutation(uint64_t s[12]) {
  or_external(s);
  for (int r = 0; r < 30; r++) {
    if (r < 4 || r >= 26) {
      for (int i = 0; i < 12; i++) s[i] = or_sbox(fr_add(s[i], g_rc[r][i]));
      or_external(s);
    } else {
      s[0] = or_sbox(fr_add(s[0], g_rc[r][0]));
      or_internal(s);
    }
  }
  for (int i = 0; i < 12; i++) s[i] = fr_canon(s[i]);
}

typedef struct {
  const uint64_t *values;
  uint64_t *results;
  uint32_t rows, cols;
  size_t count;
  int load_intermediate, store_intermediate;
} or_leaves_ctx;

/* poseidon2_gl_st.cu:25-59: overwrite-mode sponge over cols x rows values of one leaf,
 * column-major then row-minor, 8 per permutation, missing tail absorbed as zeros. */
static void or_leaves_range(void *vctx, size_t begin, size_t end) {
  const or_leaves_ctx *c = (const or_leaves_ctx *)vctx;
  const uint64_t total = (uint64_t)c->rows * c->cols;
  for (size_t gid = begin; gid < end; gid++) {
    uint64_t st[12] = {0};
    if (c->load_intermediate)
      for (int k = 0; k < 4; k++) st[8 + k] = c->results[gid + k * c->count];
    for (uint64_t off = 0; off < total;) {
      for (int i = 0; i < 8; i++, off++) {
        uint64_t row = off % c->rows, col = off / c->rows;
        st[i] = col < c->cols ? c->values[gid * c->rows + row + col * c->rows * c->count] : 0;
      }
      or_p2_permutation(st);
    }
    for (int k = 0; k < 4; k++)
      c->results[gid + k * c->count] = or_canon(st[(c->store_intermediate ? 8 : 0) + k]);
  }
}

int or_p2_leaves(const uint64_t *values, size_t values_len, uint64_t *results, size_t results_len,
                 uint32_t log_rows_per_hash, int load_intermediate, int store_intermediate, int threads) {
  /* poseidon2.rs:188-209 */
  if (results_len % 4) return -1;
  size_t count = results_len / 4;
  if (count == 0) return 0;
  size_t rows = (size_t)1 << log_rows_per_hash;
  if (values_len % (count * rows)) return -1;
  size_t cols = values_len / (count * rows);
  if (store_intermediate && (rows * cols) % 8) return -1;
  or_leaves_ctx c = {values, results, (uint32_t)rows, (uint32_t)cols, count, load_intermediate, store_intermediate};
  or_parallel_for(count, threads, or_leaves_range, &c);
  return 0;
}

typedef struct {
  const uint64_t *values;
  uint64_t *results;
  size_t count;
} or_nodes_ctx;

/* poseidon2_gl_st.cu:61-82: node i = P2([L0..L3, R0..R3, 0,0,0,0])[0..4], L/R = children 2i, 2i+1. */
static void or_nodes_range(void *vctx, size_t begin, size_t end) {
  const or_nodes_ctx *c = (const or_nodes_ctx *)vctx;
  for (size_t gid = begin; gid < end; gid++) {
    uint64_t st[12] = {0};
    for (int k = 0; k < 4; k++) {
      st[k] = c->values[k * 2 * c->count + 2 * gid];
      st[4 + k] = c->values[k * 2 * c->count + 2 * gid + 1];
    }
    or_p2_permutation(st);
    for (int k = 0; k < 4; k++) c->results[k * c->count + gid] = or_canon(st[k]);
  }
}

int or_p2_nodes(const uint64_t *values, size_t values_len, uint64_t *results, size_t results_len, int threads) {
  /* poseidon2.rs:233-242 */
  if (values_len % 8 || results_len % 4 || values_len != 2 * results_len) return -1;
  or_nodes_ctx c = {values, results, results_len / 4};
  or_parallel_for(c.count, threads, or_nodes_range, &c);
  return 0;
}

int or_p2_build_merkle_tree(const uint64_t *values, size_t values_len, uint64_t *results, size_t results_len,
                            uint32_t log_rows_per_hash, uint32_t layers_count, int threads) {
  /* poseidon2.rs:297-314 and build_merkle_tree_nodes poseidon2.rs:276-295 */
  if (layers_count == 0 || results_len % 8) return -1;
  size_t leaves = results_len / 8;
  if (leaves == 0 || layers_count - 1 >= 64 || ((size_t)1 << (layers_count - 1)) > leaves || values_len % leaves)
    return -1;
  size_t half = results_len / 2;
  if (or_p2_leaves(values, values_len, results, half, log_rows_per_hash, 0, 0, threads)) return -1;
  const uint64_t *layer = results;
  uint64_t *rest = results + half;
  size_t len = half; /* values_len of the current node step == results_len of the step */
  for (uint32_t l = 1; l < layers_count; l++) {
    if (len % 8) return -1;
    size_t v = len / 8;
    if (v & (v - 1)) return -1; /* values_len must be RATE << layer */
    if (or_p2_nodes(layer, len, rest, len / 2, threads)) return -1;
    layer = rest;
    rest += len / 2;
    len /= 2;
  }
  return 0;
}

void or_p2_gather_rows(const uint32_t *indexes, uint32_t indexes_count, uint32_t log_rows_per_index,
                       const uint64_t *values, uint64_t values_stride, uint32_t cols, uint64_t *results,
                       uint64_t result_stride) {
  uint32_t rpi = 1u << log_rows_per_index;
  for (uint32_t idx = 0; idx < indexes_count; idx++)
    for (uint32_t x = 0; x < rpi; x++) {
      uint64_t src_row = (uint64_t)indexes[idx] * rpi + x, dst_row = (uint64_t)idx * rpi + x;
      for (uint32_t c = 0; c < cols; c++) results[dst_row + c * result_stride] = values[src_row + c * values_stride];
    }
}

int or_p2_gather_merkle_paths(const uint32_t *indexes, uint32_t indexes_count, const uint64_t *values,
                              size_t values_len, uint32_t layers_count, uint64_t *results, size_t results_len) {
  /* poseidon2.rs:350-380, queries.cuh:21-37 */
  if (values_len % 4) return -1;
  size_t vc = values_len / 4;
  if (vc == 0 || (vc & (vc - 1))) return -1;
  uint32_t log_vc = 0;
  while (((size_t)1 << log_vc) < vc) log_vc++;
  if (log_vc == 0) return -1;
  uint32_t log_leaves = log_vc - 1;
  if (layers_count > log_leaves) return -1;
  if ((size_t)indexes_count * layers_count * 4 != results_len) return -1;
  for (uint32_t layer = 0; layer < layers_count; layer++)
    for (uint32_t col = 0; col < 4; col++)
      for (uint32_t idx = 0; idx < indexes_count; idx++) {
        size_t layer_off = ((size_t)4 << (log_leaves + 1)) - ((size_t)4 << (log_leaves + 1 - layer));
        size_t col_off = (size_t)col << (log_leaves - layer);
        size_t hash_idx = (size_t)(indexes[idx] >> layer) ^ 1u;
        results[(size_t)layer * indexes_count * 4 + (size_t)indexes_count * col + idx] =
            values[layer_off + col_off + hash_idx];
      }
  return 0;
}

static int64_t or_climb(const uint64_t d[4], const uint64_t *path, uint32_t level, uint32_t depth,
                        const uint64_t *cap, uint32_t cap_len, uint64_t index) {
  if (level == depth) {
    for (uint32_t k = 0; k < cap_len; k++)
      if (d[0] == or_canon(cap[4 * k]) && d[1] == or_canon(cap[4 * k + 1]) && d[2] == or_canon(cap[4 * k + 2]) &&
          d[3] == or_canon(cap[4 * k + 3]))
        return (int64_t)(index | ((uint64_t)k << depth));
    return -1;
  }
  for (int side = 0; side < 2; side++) {
    uint64_t st[12] = {0};
    const uint64_t *sib = path + 4 * level;
    for (int j = 0; j < 4; j++) {
      st[j + (side ? 4 : 0)] = d[j];
      st[j + (side ? 0 : 4)] = sib[j];
    }
    or_p2_permutation(st);
    uint64_t nd[4] = {or_canon(st[0]), or_canon(st[1]), or_canon(st[2]), or_canon(st[3])};
    int64_t r = or_climb(nd, path, level + 1, depth, cap, cap_len, index | ((uint64_t)side << level));
    if (r >= 0) return r;
  }
  return -1;
}

int64_t or_p2_find_opening(const uint64_t *leaf, uint32_t leaf_len, const uint64_t *path, uint32_t depth,
                           const uint64_t *cap, uint32_t cap_len) {
  uint64_t d[4];
  if (or_p2_leaves(leaf, leaf_len, d, 4, 0, 0, 0, 1)) return -1;
  if (depth > 40) return -1;
  return or_climb(d, path, 0, depth, cap, cap_len, 0);
}

/* ------------------------------------------------------------------------------------------
 * Commitment job: shivini's trace commitment restated.
 *   evaluations -> monomials: inverse n2b NTT then bit reverse (storage.rs:155-192)
 *   coset c of 2^log_lde: forward n2b NTT with coset index bitrev(c) (primitives/ntt.rs:25,
 *     storage.rs:245-330), subtree per coset with cap 2^(log_cap-log_lde) (cache.rs:353-377,
 *     mod.rs:37-44), caps concatenated in coset order (cache.rs:379-418).
 * ---------------------------------------------------------------------------------------- */
int or_commit(const uint64_t *evals, uint32_t log_n, uint32_t cols, uint32_t log_lde, uint32_t log_cap,
              uint64_t *monomials_out, uint64_t *lde_out, uint64_t *trees_out, uint64_t *cap_out, int threads) {
  if (log_cap < log_lde || log_n + log_lde > 30 || log_n < 1) return -1;
  uint32_t log_ccap = log_cap - log_lde;
  if (log_n < log_ccap) return -1;
  size_t n = (size_t)1 << log_n, f = (size_t)1 << log_lde, cap = (size_t)1 << log_cap, ccap = (size_t)1 << log_ccap;
  size_t col_elems = n * cols;
  uint64_t *mono = monomials_out ? monomials_out : (uint64_t *)malloc(sizeof(uint64_t) * col_elems);
  if (or_batch_ntt(evals, mono, log_n, cols, n, n, 0, 1, 0, 0, threads)) return -1;
  or_bit_reverse(mono, n, mono, n, log_n, cols);
  for (size_t c = 0; c < f; c++) {
    uint64_t *lde = lde_out + c * col_elems;
    uint64_t *tree = trees_out + c * 8 * n;
    if (or_batch_ntt(mono, lde, log_n, cols, n, n, 0, 0, log_lde, or_bitrev((uint32_t)c, log_lde), threads)) return -1;
    if (or_p2_build_merkle_tree(lde, col_elems, tree, 8 * n, 0, log_n - log_ccap + 1, threads)) return -1;
    const uint64_t *sub_cap = tree + 8 * n - 8 * ccap;
    for (size_t m = 0; m < ccap; m++)
      for (int j = 0; j < 4; j++) cap_out[j * cap + c * ccap + m] = sub_cap[j * ccap + m];
  }
  if (!monomials_out) free(mono);
  return 0;
}
