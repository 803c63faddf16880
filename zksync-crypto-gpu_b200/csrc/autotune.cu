// Autotuner: per device, times candidate launch configurations of the NTT (radix bits per
// register round, stages in the strided pass, tile width, columns per CTA, L2 chunk size) for
// each size, and of the Poseidon2 leaf kernel (threads per CTA, unrolled / partly / fully rolled
// rounds), installs the fastest, and saves / loads the table as text.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "glc_internal.h"

namespace glc {

static float time_ms(cudaStream_t s, int reps, const std::function<int()> &fn, int *err) {
  cudaEvent_t a = nullptr, b = nullptr;
  float ms = 0;
  *err = (int)cudaEventCreate(&a);
  if (!*err) *err = (int)cudaEventCreate(&b);
  if (!*err) *err = fn();  // warm-up
  if (!*err) *err = (int)cudaEventRecord(a, s);
  for (int i = 0; i < reps && !*err; i++) *err = fn();
  if (!*err) *err = (int)cudaEventRecord(b, s);
  if (!*err) *err = (int)cudaEventSynchronize(b);
  if (!*err) *err = (int)cudaEventElapsedTime(&ms, a, b);
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  return reps ? ms / reps : ms;
}

}  // namespace glc

using namespace glc;

extern "C" glc_status glc_tuning_get_ntt(uint32_t log_n, glc_ntt_tuning *out) {
  if (!out || log_n < 1 || log_n > MAX_LOG_N) return fail("tuning: bad arguments");
  const NttTuning &t = ntt_tuning(log_n);
  *out = {t.radix_bits, t.k1, t.max_log_w, t.max_cols_per_cta, t.l2_chunk_mb};
  return 0;
}

extern "C" glc_status glc_tuning_set_ntt(uint32_t log_n, const glc_ntt_tuning *in) {
  if (!in || log_n < 1 || log_n > MAX_LOG_N) return fail("tuning: bad arguments");
  if (in->radix_bits < 2 || in->radix_bits > 4) return fail("tuning: radix_bits must be 2, 3 or 4");
  if (in->max_log_w > 5 || in->max_cols_per_cta == 0 || in->max_cols_per_cta > 64)
    return fail("tuning: values out of range");
  if (in->k1 && (in->k1 > 12 || log_n - in->k1 > 12 || in->k1 >= log_n)) return fail("tuning: k1 out of range");
  NttTuning &t = ntt_tuning(log_n);
  t.radix_bits = in->radix_bits;
  t.k1 = in->k1;
  t.max_log_w = in->max_log_w;
  t.max_cols_per_cta = in->max_cols_per_cta;
  t.l2_chunk_mb = in->l2_chunk_mb;
  return 0;
}

extern "C" glc_status glc_tuning_get_p2(glc_p2_tuning *out) {
  if (!out) return fail("tuning: bad arguments");
  const P2Tuning &t = p2_tuning();
  *out = {t.leaf_threads, t.rolled, t.lazy ? 1u : 0u, t.min_blocks};
  return 0;
}

extern "C" glc_status glc_tuning_set_p2(const glc_p2_tuning *in) {
  if (!in || (in->leaf_threads != 64 && in->leaf_threads != 128 && in->leaf_threads != 256))
    return fail("tuning: leaf_threads must be 64, 128 or 256");
  if (in->min_blocks != 2 && in->min_blocks != 3 && in->min_blocks != 5)
    return fail("tuning: min_blocks must be 2, 3 or 5");
  if (in->min_blocks == 5 && in->leaf_threads > 128) return fail("tuning: min_blocks 5 needs leaf_threads <= 128");
  if (in->rolled > 2) return fail("tuning: rolled must be 0, 1 or 2");
  P2Tuning &t = p2_tuning();
  t.leaf_threads = in->leaf_threads;
  t.rolled = in->rolled;
  t.lazy = in->lazy != 0;
  t.min_blocks = in->min_blocks;
  return 0;
}

extern "C" glc_status glc_autotune(uint32_t log_n_min, uint32_t log_n_max, uint32_t cols, uint32_t reps) {
  if (log_n_min < 1 || log_n_max > MAX_LOG_N || log_n_min > log_n_max || cols > 65536)
    return fail("autotune: bad size range");
  if (!current_tables()) return fail("autotune: glc_context_create has not been called on this device");
  if (reps == 0) reps = 3;
  // cols == 0: a commitment-sized batch per size, 128 columns up to 2^28 elements (2 GiB)
  auto cols_for = [&](uint32_t log_n) -> uint32_t {
    return cols ? cols : (uint32_t)std::min<uint64_t>(128, std::max<uint64_t>(8, (1ull << 28) >> log_n));
  };
  // scratch: the largest NTT batch, and the leaf probe's 128 x 2^19 values (larger than L2, many
  // column streams, like a real commitment) + 4 x 2^17 digests
  constexpr uint64_t LEAF_ROWS = 1ull << 19, LEAF_COLS = 128;
  uint64_t elems = (LEAF_COLS + 4) * LEAF_ROWS;
  for (uint32_t l = log_n_min; l <= log_n_max; l++) elems = std::max<uint64_t>(elems, (uint64_t)cols_for(l) << l);
  uint64_t *buf = nullptr;
  cudaError_t ce = cudaMalloc(&buf, elems * sizeof(uint64_t));
  if (ce != cudaSuccess) return (int)ce;
  cudaStream_t s = nullptr;
  ce = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(buf, 0x5a, elems * sizeof(uint64_t), s);
  if (ce != cudaSuccess) {
    if (s) cudaStreamDestroy(s);
    cudaFree(buf);
    return (int)ce;
  }
  int err = 0;
  for (uint32_t log_n = log_n_min; log_n <= log_n_max && !err; log_n++) {
    const NttTuning saved = ntt_tuning(log_n);
    NttTuning best = saved;
    float best_ms = 1e30f;
    const uint32_t nc = cols_for(log_n);
    // strided-pass stages within 3 of an even split (0 = the default split)
    std::vector<uint32_t> k1s = {0};
    if (log_n > 12)
      for (uint32_t k = std::max(log_n - 12, 1u); k <= std::min(12u, log_n - 1); k++)
        if (k + 3 >= log_n / 2 && k <= log_n / 2 + 3) k1s.push_back(k);
    for (uint32_t rb : {2u, 3u, 4u})
      for (uint32_t k1 : k1s)
        for (uint32_t lw : {2u, 3u, 4u, 5u})
          for (uint32_t cpc : {1u, 4u, 8u})
            for (uint32_t mb : {0u, 48u}) {
            if (err || (mb && log_n <= 12)) continue;  // stop after an error; one pass: nothing to chunk
            NttTuning c = saved;
            c.radix_bits = rb;
            c.k1 = k1;
            c.max_log_w = lw;
            c.max_cols_per_cta = cpc;
            c.l2_chunk_mb = mb;
            ntt_tuning(log_n) = c;
            // time a forward coset LDE (the commitment's dominant NTT), in place
            const float ms = time_ms(s, (int)reps, [&] {
              return ntt_launch(buf, buf, log_n, nc, 1ull << log_n, 1ull << log_n, false, false, 1, 1, s, 0);
            }, &err);
            if (err) break;
            if (ms < best_ms) {
              best_ms = ms;
              best = c;
            }
          }
    ntt_tuning(log_n) = err ? saved : best;
  }
  if (!err) {
    // Poseidon2 leaves: LEAF_ROWS rows x LEAF_COLS columns (buf[0, LEAF_COLS * count)), digests after them
    const uint64_t count = LEAF_ROWS;
    const P2Tuning saved = p2_tuning();
    P2Tuning best = saved;
    float best_ms = 1e30f;
    for (uint32_t th : {128u, 256u})
      for (uint32_t rolled : {0u, 1u, 2u})
        for (bool lazy : {false, true})
          for (uint32_t minb : {2u, 3u, 5u}) {
        if (err || (minb == 5 && th > 128)) continue;
        P2Tuning c;
        c.leaf_threads = th;
        c.rolled = rolled;
        c.lazy = lazy;
        c.min_blocks = minb;
        p2_tuning() = c;
        const float ms = time_ms(s, (int)reps, [&] {
          return p2_leaves_launch(buf, buf + LEAF_COLS * count, 0, LEAF_COLS, count, false, false, s);
        }, &err);
        if (err) break;
        if (ms < best_ms) {
          best_ms = ms;
          best = c;
        }
      }
    p2_tuning() = err ? saved : best;
  }
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  cudaFree(buf);
  return err;
}

extern "C" glc_status glc_tuning_save(const char *path) {
  if (!path) return fail("tuning: null path");
  FILE *f = fopen(path, "w");
  if (!f) return fail(std::string("tuning: cannot write ") + path);
  const P2Tuning &p = p2_tuning();
  fprintf(f, "p2 %u %u %u %u\n", p.leaf_threads, p.rolled, p.lazy ? 1u : 0u, p.min_blocks);
  for (uint32_t l = 1; l <= MAX_LOG_N; l++) {
    const NttTuning &t = ntt_tuning(l);
    fprintf(f, "ntt %u %u %u %u %u %u\n", l, t.radix_bits, t.k1, t.max_log_w, t.max_cols_per_cta, t.l2_chunk_mb);
  }
  fclose(f);
  return 0;
}

extern "C" glc_status glc_tuning_load(const char *path) {
  if (!path) return fail("tuning: null path");
  FILE *f = fopen(path, "r");
  if (!f) return fail(std::string("tuning: cannot read ") + path);
  char kind[8];
  int e = 0;
  while (!e && fscanf(f, "%7s", kind) == 1) {
    if (!strcmp(kind, "p2")) {
      glc_p2_tuning p;
      if (fscanf(f, "%u %u %u %u", &p.leaf_threads, &p.rolled, &p.lazy, &p.min_blocks) != 4)
        e = fail("tuning: malformed p2 line");
      else e = glc_tuning_set_p2(&p);
    } else if (!strcmp(kind, "ntt")) {
      uint32_t l;
      glc_ntt_tuning t;
      if (fscanf(f, "%u %u %u %u %u %u", &l, &t.radix_bits, &t.k1, &t.max_log_w, &t.max_cols_per_cta, &t.l2_chunk_mb) != 6)
        e = fail("tuning: malformed ntt line");
      else
        e = glc_tuning_set_ntt(l, &t);
    } else {
      e = fail("tuning: unknown line kind");
    }
  }
  fclose(f);
  return e;
}
