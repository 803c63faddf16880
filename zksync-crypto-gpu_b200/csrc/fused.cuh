// Fused batch of small commitments: ONE persistent launch runs every stage of every job.
//
// The per-call form issues about 28 kernels per commitment (NTT passes, bit reversal, one leaf
// launch and node layers per coset, the cap gather); for jobs of 2^12..2^16 rows each of those
// kernels runs for microseconds and cannot fill 148 SMs, so a batch of such jobs is bound by
// launch latency and by the tails of small grids; jobs up to 2^22 rows (two NTT passes on
// 2^12-element tiles whose rows stay at least 4 elements = 32 bytes wide) run in the same launch (the reference's per-stage and per-layer
// launches, crates/boojum-cuda/src/ntt.rs:201-241 and src/poseidon2.rs:276-295, are the same
// shape).  Here a persistent grid (as many CTAs as fit on the device at once, launched
// cooperatively so that all of them are resident) takes work items from one global counter, in
// a topological order:
//   inverse NTT pass 1, pass 2 -> bit reversal -> forward coset NTT pass 1, pass 2 (the coset
//   that transforms the monomials in place last, after the others have read them) -> leaf
//   hashes -> node layer 1, 2, ... -> cap gather,
// every stage listing the items of all jobs, heaviest first.  An item is an NTT tile of 2^12
// elements (or a whole column of a smaller NTT) in up to 4 columns (8 from 2^17 rows), 4096
// rows of a bit reversal, 256 leaves, 256 nodes or 256 cap entries: large enough that the
// per-item costs (the claim of the item number, the search for its entry, the dependency check
// and the release of its count, a few microseconds together) stay a few percent of its work.  Before it runs, an item waits
// until the items it reads from are done: each stage of each job (per coset where it applies)
// counts its finished items, and the item waits for its producer's count to reach the producer's
// item total.  Items wait only for items that come earlier in the order, which some resident CTA
// fetched already, so the grid always makes progress; different jobs' stages overlap freely.
// Every wait is bounded (about 1 s): on expiry the item counts a timeout in a device counter
// (glc_commit_batch_fused_timeouts), raises the launch's abort flag, which ends every other
// wait, and runs anyway, so a bug shows as wrong results and a non-zero count, never as a hang.
// The items reuse the tile and hash code of the per-call kernels (ntt_pass_tile, leaf_hash,
// hash_node), so the results are the same bits.
//
// Included at the end of poseidon2.cu: it needs that file's __constant__ round constants.
#pragma once
#include <cooperative_groups.h>

#include <mutex>
#include <vector>

#include "ntt_tile.cuh"

namespace glc {

namespace cg = cooperative_groups;

static constexpr uint32_t FUSED_THREADS = 256;
static constexpr uint32_t FUSED_MAX_LOG_N = 22;  // two passes of at most 12 stages on 2^12-element tiles with rows of >= 4 elements
// columns per NTT item (fewer when a job has fewer): each item rebuilds its tile's block
// twiddles, so more columns amortise them; jobs from 2^17 rows have items to spare.  Measured on
// the uneven batch: 2 / 4 columns: small jobs 20.7 / 20.4 ms; 8 columns from 2^17 rows: the
// 300 jobs 4851 -> 4726 ms.
static constexpr uint32_t FUSED_NTT_COLS = 4, FUSED_NTT_COLS_LARGE = 8, FUSED_LARGE_LOG_N = 17;
// rows of one column per bit-reversal item
static constexpr uint32_t FUSED_BITREV_ROWS = 4096;

enum FusedKind : uint32_t { FK_NTT = 0, FK_BITREV = 1, FK_LEAVES = 2, FK_NODES = 3, FK_CAPS = 4 };

static constexpr uint32_t NO_COUNTER = 0xFFFFFFFFu;

// One job's share of one stage: `units` items, numbered globally from `first`.
struct FusedEntry {
  uint64_t first;          // global number of this entry's first item
  uint64_t units;
  uint32_t kind;
  uint32_t log_rows;       // bit reversal: log2 of the rows
  uint32_t dep;            // counter this entry's items wait on (NO_COUNTER: none) ...
  uint32_t dep_target;     // ... until it reaches this value
  uint32_t done1, done2;   // counters each finished item increments (NO_COUNTER: none)
  uint64_t tiles_per_col;  // NTT: tiles per column (units = tiles_per_col x column groups)
  PassArgs ntt;            // NTT: the pass
  const uint64_t *src;     // leaves: values; nodes: child layer; caps: trees
  uint64_t *dst;           // bit reversal: the matrix (in place); leaves: digests; nodes: parent layer; caps: cap
  uint64_t stride;         // bit reversal: column stride; caps: length of one subtree buffer
  uint64_t count;          // leaves: leaves; nodes: parent nodes; caps: cap entries x 4
  uint64_t cols;           // leaves: columns; caps: cosets
  uint64_t aux;            // nodes: child layer 16-byte aligned; caps: offset of a subtree's cap
  uint32_t ccap;           // caps: cap entries per coset
};

// Waits that expired (device-wide, since the library was loaded).
static __device__ unsigned long long g_fused_timeouts;

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_add(uint32_t *p, uint32_t v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Trace timestamps: the GPU's global nanosecond timer (one clock for every SM).
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ uint32_t sm_id() {
  uint32_t v;
  asm("mov.u32 %0, %%smid;" : "=r"(v));
  return v;
}

static constexpr uint32_t FUSED_WAIT_LIMIT = 1u << 22;  // x 200 ns sleeps: about 1 s

__global__ void __launch_bounds__(FUSED_THREADS, 3)
    fused_commit_kernel(const FusedEntry *entries, uint32_t n_entries, uint64_t total_units, uint32_t *counters,
                        uint32_t *abort_flag, unsigned long long *next_unit, unsigned long long *trace,
                        uint64_t trace_items, const volatile uint32_t *cancel, uint32_t *status) {
  extern __shared__ uint64_t smem[];
  __shared__ uint64_t s_unit;
  __shared__ uint32_t s_entry, s_skip;
  const uint32_t tid = threadIdx.x;
  // launch-wide words after the abort flag: CTAs that have left, and whether a cancel skipped items
  uint32_t *exited = abort_flag + 1, *cancelled = abort_flag + 2;
  // Thread 0 claims the CTA's next item while the current one runs, so the claim's round trip
  // to L2 is off the critical path.  Progress still holds: a CTA's claims increase, so the CTA
  // that holds the lowest unfinished item is running it (its claimed-next item is above it),
  // and that item's producers, all lower, are finished.
  unsigned long long claimed = 0;
  if (tid == 0) claimed = atomicAdd(next_unit, 1ull);
  while (true) {
    __syncthreads();  // the previous item's last reads of s_unit, s_entry and shared memory are done
    if (tid == 0) {
      s_unit = claimed;
      if (claimed < total_units) {
        if (cancel && *cancel) {
          // cancelled: claim nothing more, skip this item, and end every wait of the launch
          atomicExch(cancelled, 1u);
          atomicExch(abort_flag, 1u);
          s_unit = total_units;
        } else {
          claimed = atomicAdd(next_unit, 1ull);
        }
      }
    }
    __syncthreads();
    const uint64_t u = s_unit;
    if (u >= total_units) break;
    const unsigned long long t_claim = (trace && tid == 0) ? global_ns() : 0ull;
    // the entry holding item u, the last one whose first item is <= u: a 32-way search by warp 0
    // (three rounds of dependent loads for up to 32K entries)
    if (tid < 32) {
      uint32_t lo = 0, span = n_entries;  // entries[lo].first <= u; the answer is below lo + span
      while (span > 1) {
        const uint32_t step = (span + 31) / 32;
        const uint32_t idx = lo + tid * step;
        const bool ok = idx < lo + span && entries[idx].first <= u;
        const uint32_t last = 31 - __clz(__ballot_sync(0xFFFFFFFFu, ok));  // lane 0 is always ok
        const uint32_t nlo = lo + last * step;
        span = min(step, lo + span - nlo);
        lo = nlo;
      }
      if (tid == 0) s_entry = lo;
    }
    __syncthreads();
    const FusedEntry &E = entries[s_entry];
    if (tid == 0) {
      if (E.dep != NO_COUNTER) {
        // after one expired wait (a bug, not a slow producer) no item waits any more: the launch
        // then ends within one wait limit whatever else is wrong
        uint32_t it = 0;
        while (ld_acquire(counters + E.dep) < E.dep_target && !ld_acquire(abort_flag)) {
          if (++it > FUSED_WAIT_LIMIT) {
            atomicAdd(&g_fused_timeouts, 1ull);
            atomicExch(abort_flag, 1u);
            break;
          }
          if (cancel && (it & 63) == 0 && *cancel) {
            atomicExch(cancelled, 1u);
            atomicExch(abort_flag, 1u);
          }
          __nanosleep(200);
        }
      }
      // a cancelled launch skips the items it has not started (their inputs may be incomplete)
      s_skip = cancel && ld_acquire(cancelled) ? 1u : 0u;
    }
    __syncthreads();  // the acquire above orders the producers' writes before this CTA's reads
    if (s_skip) break;
    const unsigned long long t_start = (trace && tid == 0) ? global_ns() : 0ull;
    const uint64_t local = u - E.first;
    const uint32_t kind = E.kind;
    if (kind == FK_NTT) {
      const PassArgs a = E.ntt;
      const uint64_t tpc = E.tiles_per_col;
      ntt_pass_tile<4>(a, (uint32_t)(local % tpc), (uint32_t)(local / tpc), smem);
    } else if (kind == FK_BITREV) {
      const uint32_t L = E.log_rows;
      const uint64_t n = 1ull << L, chunks = (n + FUSED_BITREV_ROWS - 1) / FUSED_BITREV_ROWS;
      const uint64_t col = local / chunks, i0 = (local % chunks) * FUSED_BITREV_ROWS;
      uint64_t *x = E.dst + col * E.stride;
      for (uint64_t i = i0 + tid; i < min(i0 + FUSED_BITREV_ROWS, n); i += FUSED_THREADS) {
        const uint64_t r = brev_low((uint32_t)i, L);
        if (i < r) {
          const uint64_t vi = x[i], vr = x[r];
          x[i] = vr;
          x[r] = vi;
        }
      }
    } else if (kind == FK_LEAVES) {
      const uint64_t gid = local * FUSED_THREADS + tid;
      if (gid < E.count) leaf_hash<2, true>(E.src, E.dst, 0, E.cols, E.count, false, false, gid);
    } else if (kind == FK_NODES) {
      const uint64_t i = local * FUSED_THREADS + tid, count = E.count;
      if (i < count) {
        uint64_t l[4], r[4], o[4];
        load_children(E.src, count, i, l, r, E.aux != 0);
        hash_node<2, true>(l, r, o);
#pragma unroll
        for (int k = 0; k < 4; k++) E.dst[k * count + i] = o[k];
      }
    } else {  // FK_CAPS: cap[j*ccap*f + c*ccap + m] = tree_c[cap_off + j*ccap + m]
      const uint64_t t = local * FUSED_THREADS + tid;
      if (t < E.count) {
        const uint64_t ccap = E.ccap, f = E.cols;
        const uint64_t m = t % ccap, c = (t / ccap) % f, j = t / (ccap * f);
        E.dst[j * ccap * f + c * ccap + m] = E.src[c * E.stride + E.aux + j * ccap + m];
      }
    }
    __syncthreads();  // every thread's writes of this item precede the release below
    if (tid == 0) {
      if (trace && u < trace_items) {
        unsigned long long *r = trace + 4 * u;
        r[0] = t_claim;
        r[1] = t_start;
        r[2] = global_ns();
        r[3] = ((unsigned long long)sm_id() << 40) | ((unsigned long long)blockIdx.x << 8) | E.kind;
      }
      if (E.done1 != NO_COUNTER) red_release_add(counters + E.done1, 1u);
      if (E.done2 != NO_COUNTER) red_release_add(counters + E.done2, 1u);
    }
  }
  // the last CTA to leave reports how the launch ended: 1 = every item ran, 2 = cancelled
  if (status && tid == 0) {
    __threadfence();
    if (atomicAdd(exited, 1u) == gridDim.x - 1) {
      *reinterpret_cast<volatile uint32_t *>(status) = ld_acquire(cancelled) ? 2u : 1u;
      __threadfence_system();
    }
  }
}

// Host side: the work list of a batch (stages in order, items numbered globally, each entry
// with its dependency counter) and the launch of the persistent grid.
struct FusedPlan {
  std::vector<FusedEntry> entries;
  std::vector<uint32_t> target;       // per counter: the items that count into it
  std::vector<size_t> stage_begin;    // index in `entries` of each stage's first entry
  size_t smem = 0;

  uint32_t counter() {
    target.push_back(0);
    return (uint32_t)target.size() - 1;
  }
  void begin_stage() { stage_begin.push_back(entries.size()); }
  void add(FusedEntry e, uint32_t dep, uint32_t done1, uint32_t done2 = NO_COUNTER) {
    e.dep = dep;
    e.done1 = done1;
    e.done2 = done2;
    if (done1 != NO_COUNTER) target[done1] += (uint32_t)e.units;
    if (done2 != NO_COUNTER) target[done2] += (uint32_t)e.units;
    if (e.units) entries.push_back(e);
  }
  // Heaviest items of each stage first (the last items to start bound a stage's tail), then the
  // global numbering and the wait targets.  Sorts indexes, then moves each entry once.
  uint64_t finish() {
    std::vector<FusedEntry> out;
    out.reserve(entries.size());
    std::vector<uint32_t> order;
    uint64_t first = 0;
    for (size_t s = 0; s < stage_begin.size(); s++) {
      const size_t b = stage_begin[s], e = s + 1 < stage_begin.size() ? stage_begin[s + 1] : entries.size();
      order.resize(e - b);
      for (size_t i = b; i < e; i++) order[i - b] = (uint32_t)i;
      std::stable_sort(order.begin(), order.end(),
                       [&](uint32_t x, uint32_t y) { return cost(entries[x]) > cost(entries[y]); });
      for (uint32_t i : order) {
        FusedEntry &x = entries[i];
        x.first = first;
        first += x.units;
        x.dep_target = x.dep == NO_COUNTER ? 0 : target[x.dep];
        out.push_back(x);
      }
    }
    entries.swap(out);
    return first;
  }
  static uint64_t cost(const FusedEntry &e) {
    if (e.kind == FK_NTT) return (1ull << (e.ntt.k + e.ntt.log_w)) * e.ntt.k * e.ntt.cols_per_cta;
    if (e.kind == FK_LEAVES) return 4096 * ((e.cols + 7) / 8);
    return 1;
  }
};

static uint32_t fused_brev(uint32_t x, uint32_t bits) {
  uint32_t r = 0;
  for (uint32_t i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

// Passes of an NTT in the fused batch: tiles of 2^12 elements wherever the size allows, so the
// items are few and large (each item rebuilds its tile's block twiddles and pays a claim, a
// search and a dependency check): one pass up to 2^12 rows, else a strided pass of log_n - 12
// stages over tiles of 2^(24 - log_n) columns and a contiguous pass of 12 stages.
static uint32_t fused_ntt_plan(uint32_t log_n, Pass *p) {
  if (log_n <= SINGLE_PASS_MAX_LOG) {
    p[0] = {0, log_n, 0};
    return 1;
  }
  const uint32_t k0 = log_n - SINGLE_PASS_MAX_LOG;
  p[0] = {0, k0, SINGLE_PASS_MAX_LOG - k0};
  p[1] = {k0, SINGLE_PASS_MAX_LOG, 0};
  return 2;
}

static FusedEntry ntt_entry(const DeviceTables *t, uint32_t log_n, uint32_t q, uint32_t np, const Pass &ps,
                            const uint64_t *in, uint64_t *out, uint64_t in_stride, uint64_t out_stride, uint32_t cols,
                            bool inverse, uint32_t log_ext, uint32_t coset, size_t &smem) {
  FusedEntry e{};
  e.kind = FK_NTT;
  NttTuning tu{};  // the fused items use radix-16 rounds; make_pass reads nothing else from it here
  tu.radix_bits = 4;
  const PassShape sh = make_pass(e.ntt, t, tu, ps, q, np, in, out, in_stride, out_stride, cols, log_n, false, inverse,
                                 log_ext, coset, 1);
  // the batch fills the device together: the item width does not shrink for small batches
  e.ntt.cols_per_cta = std::min(log_n >= FUSED_LARGE_LOG_N ? FUSED_NTT_COLS_LARGE : FUSED_NTT_COLS, cols);
  e.tiles_per_col = sh.tiles_per_col;
  e.units = sh.tiles_per_col * ((cols + e.ntt.cols_per_cta - 1) / e.ntt.cols_per_cta);
  smem = std::max(smem, sh.smem);
  return e;
}

static uint64_t fused_plan(const DeviceTables *t, const glc_commit_job *jobs, uint32_t n_jobs, FusedPlan &P) {
  auto units = [](uint64_t n) { return (n + FUSED_THREADS - 1) / FUSED_THREADS; };
  struct J {
    const glc_commit_job *j;
    uint64_t n, f, coset_elems;
    uint64_t *mono;
    Pass inv[2], fwd[2];
    uint32_t np, layers;  // NTT passes; tree layers including the leaves
    bool in_place_last;   // the last coset transforms the monomials in place
    uint32_t c_inv[2], c_brev, c_readers, c_trees;
    std::vector<uint32_t> c_fwd0, c_fwd1, c_layer;  // per coset (c_layer: the latest layer built)
  };
  std::vector<J> js(n_jobs);
  uint32_t max_layers = 0;
  for (uint32_t i = 0; i < n_jobs; i++) {
    J &x = js[i];
    x.j = &jobs[i];
    x.n = 1ull << jobs[i].log_n;
    x.f = 1ull << jobs[i].log_lde;
    x.coset_elems = x.n * jobs[i].cols;
    x.in_place_last = !jobs[i].monomials;
    x.mono = jobs[i].monomials ? jobs[i].monomials : jobs[i].lde + (x.f - 1) * x.coset_elems;
    // tiles of at most 2^12 elements: at most 68 KB of shared memory, three CTAs per SM
    x.np = fused_ntt_plan(jobs[i].log_n, x.inv);
    fused_ntt_plan(jobs[i].log_n, x.fwd);
    x.layers = jobs[i].log_n - (jobs[i].log_cap - jobs[i].log_lde) + 1;
    max_layers = std::max(max_layers, x.layers);
    x.c_inv[0] = P.counter();
    x.c_inv[1] = P.counter();
    x.c_brev = P.counter();
    x.c_readers = P.counter();
    x.c_trees = P.counter();
    x.c_fwd0.resize(x.f);
    x.c_fwd1.resize(x.f);
    x.c_layer.resize(x.f);
    for (uint64_t c = 0; c < x.f; c++) {
      x.c_fwd0[c] = P.counter();
      x.c_fwd1[c] = P.counter();
    }
  }
  // inverse NTT (evaluations -> bit-reversed coefficients x N^-1), pass by pass
  for (uint32_t q = 0; q < 2; q++) {
    P.begin_stage();
    for (J &x : js)
      if (q < x.np)
        P.add(ntt_entry(t, x.j->log_n, q, x.np, x.inv[q], x.j->evals, x.mono, x.j->evals_stride, x.n, x.j->cols, true, 0,
                        0, P.smem),
              q ? x.c_inv[0] : NO_COUNTER, x.c_inv[q]);
  }
  // bit reversal: natural-order monomials
  P.begin_stage();
  for (J &x : js) {
    FusedEntry e{};
    e.kind = FK_BITREV;
    e.log_rows = x.j->log_n;
    e.dst = x.mono;
    e.stride = x.n;
    e.units = (uint64_t)x.j->cols * ((x.n + FUSED_BITREV_ROWS - 1) / FUSED_BITREV_ROWS);
    P.add(e, x.c_inv[x.np - 1], x.c_brev);
  }
  // forward coset NTTs; without a monomials buffer the last coset transforms the monomials in
  // place, so its first pass waits until the other cosets' first passes have read them
  for (int last = 0; last < 2; last++)
    for (uint32_t q = 0; q < 2; q++) {
      P.begin_stage();
      for (J &x : js) {
        if (q >= x.np) continue;
        for (uint64_t c = 0; c < x.f; c++) {
          const bool ipl = x.in_place_last && c == x.f - 1;
          if (ipl != (last == 1)) continue;
          const FusedEntry e = ntt_entry(t, x.j->log_n, q, x.np, x.fwd[q], x.mono, x.j->lde + c * x.coset_elems, x.n,
                                         x.n, x.j->cols, false, x.j->log_lde, fused_brev((uint32_t)c, x.j->log_lde),
                                         P.smem);
          const uint32_t done = q ? x.c_fwd1[c] : x.c_fwd0[c];
          if (q == 1)
            P.add(e, x.c_fwd0[c], done);
          else if (!ipl)
            P.add(e, x.c_brev, done, x.in_place_last ? x.c_readers : NO_COUNTER);
          else
            P.add(e, x.f > 1 ? x.c_readers : x.c_brev, done);
        }
      }
    }
  // leaf hashes of every coset
  P.begin_stage();
  for (J &x : js)
    for (uint64_t c = 0; c < x.f; c++) {
      FusedEntry e{};
      e.kind = FK_LEAVES;
      e.src = x.j->lde + c * x.coset_elems;
      e.dst = x.j->trees + c * 8 * x.n;
      e.count = x.n;
      e.cols = x.j->cols;
      e.units = units(x.n);
      x.c_layer[c] = P.counter();
      P.add(e, x.np == 2 ? x.c_fwd1[c] : x.c_fwd0[c], x.c_layer[c], x.layers == 1 ? x.c_trees : NO_COUNTER);
    }
  // node layers: layer l (parent count n >> l) starts at 8n - 8n / 2^l in the subtree buffer
  for (uint32_t l = 1; l < max_layers; l++) {
    P.begin_stage();
    for (J &x : js) {
      if (l >= x.layers) continue;
      for (uint64_t c = 0; c < x.f; c++) {
        uint64_t *tree = x.j->trees + c * 8 * x.n;
        FusedEntry e{};
        e.kind = FK_NODES;
        e.src = tree + (8 * x.n - (8 * x.n >> (l - 1)));
        e.dst = tree + (8 * x.n - (8 * x.n >> l));
        e.count = x.n >> l;
        e.aux = (reinterpret_cast<uintptr_t>(e.src) & 15) == 0;
        e.units = units(e.count);
        const uint32_t prev = x.c_layer[c];
        x.c_layer[c] = P.counter();
        P.add(e, prev, x.c_layer[c], l + 1 == x.layers ? x.c_trees : NO_COUNTER);
      }
    }
  }
  // caps, once every subtree of the job is built
  P.begin_stage();
  for (J &x : js) {
    const uint32_t ccap = 1u << (x.j->log_cap - x.j->log_lde);
    FusedEntry e{};
    e.kind = FK_CAPS;
    e.src = x.j->trees;
    e.dst = x.j->cap;
    e.stride = 8 * x.n;
    e.aux = 8 * x.n - 8ull * ccap;
    e.ccap = ccap;
    e.cols = x.f;
    e.count = 4ull * ccap * x.f;
    e.units = units(e.count);
    P.add(e, x.c_trees, NO_COUNTER);
  }
  return P.finish();
}

}  // namespace glc

namespace glc {

// The work table of a launch lives in a per-device private stream-ordered pool that keeps its
// freed blocks (release threshold: never): from the second call on, the table's allocation is a
// pool hit.  The default pool, whose release threshold is 0, would hand the memory back to the
// driver at every synchronisation and map it again on the next call, which was measured at 0 to
// 90 ms per call on B200.  The pool is created on the first call on a device and destroyed by
// glc_context_destroy.
static std::mutex g_fused_pool_mutex;
static cudaMemPool_t g_fused_pool[MAX_DEVICES];

static cudaError_t fused_pool(int dev, cudaMemPool_t *out) {
  std::lock_guard<std::mutex> lock(g_fused_pool_mutex);
  if (!g_fused_pool[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    cudaError_t e = cudaMemPoolCreate(&p, &props);
    if (e != cudaSuccess) return e;
    uint64_t threshold = UINT64_MAX;
    e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &threshold);
    if (e != cudaSuccess) {
      cudaMemPoolDestroy(p);
      return e;
    }
    g_fused_pool[dev] = p;
  }
  *out = g_fused_pool[dev];
  return cudaSuccess;
}

// Releases the device's work-table pool (its blocks are freed once the launches that use them end).
void fused_forget_device(int dev) {
  std::lock_guard<std::mutex> lock(g_fused_pool_mutex);
  if (g_fused_pool[dev]) cudaMemPoolDestroy(g_fused_pool[dev]);
  g_fused_pool[dev] = nullptr;
}

}  // namespace glc

using namespace glc;

static glc_status commit_batch_fused(const glc_commit_job *jobs, uint32_t n_jobs, unsigned long long *trace,
                                     uint64_t trace_items, const uint32_t *cancel, uint32_t *status, void *stream_) {
  if (n_jobs == 0) return 0;
  if (!jobs) return fail("commit_batch_fused: null jobs");
  for (uint32_t i = 0; i < n_jobs; i++) {
    const int e = commit_check(jobs[i]);
    if (e) return e;
    if (jobs[i].log_n > FUSED_MAX_LOG_N) return fail("commit_batch_fused: log_n must be <= 22");
  }
  const DeviceTables *t = current_tables();
  if (!t) return fail("commit_batch_fused: glc_context_create has not been called on this device");
  FusedPlan P;
  const uint64_t total = fused_plan(t, jobs, n_jobs, P);
  if (P.entries.empty()) return 0;
  cudaStream_t stream = (cudaStream_t)stream_;
  cudaError_t ce = cudaFuncSetAttribute(fused_commit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.smem);
  int dev = 0, sms = 0, per_sm = 0;
  if (ce == cudaSuccess) ce = cudaGetDevice(&dev);
  if (ce == cudaSuccess) ce = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (ce == cudaSuccess)
    ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fused_commit_kernel, FUSED_THREADS, P.smem);
  if (ce != cudaSuccess) return (int)ce;
  if (per_sm < 1) return fail("commit_batch_fused: the kernel does not fit on an SM");
  // one stream-ordered buffer: the entries, then the counters and the item counter (zeroed)
  const size_t eb = P.entries.size() * sizeof(FusedEntry);
  const size_t cb = ((P.target.size() + 3) * sizeof(uint32_t) + 7) / 8 * 8 + sizeof(unsigned long long);
  if (dev < 0 || dev >= MAX_DEVICES) return fail("commit_batch_fused: device ordinal out of range");
  cudaMemPool_t pool = nullptr;
  ce = fused_pool(dev, &pool);
  if (ce != cudaSuccess) return (int)ce;
  char *buf = nullptr;
  ce = cudaMallocFromPoolAsync((void **)&buf, eb + cb, pool, stream);
  if (ce != cudaSuccess) return (int)ce;
  // pageable source: the copy is staged before it returns, so the host table may go
  ce = cudaMemcpyAsync(buf, P.entries.data(), eb, cudaMemcpyHostToDevice, stream);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(buf + eb, 0, cb, stream);
  if (ce == cudaSuccess) {
    const FusedEntry *de = reinterpret_cast<const FusedEntry *>(buf);
    uint32_t *counters = reinterpret_cast<uint32_t *>(buf + eb);
    uint32_t *abort_flag = counters + P.target.size();
    unsigned long long *next = reinterpret_cast<unsigned long long *>(buf + eb + cb - sizeof(unsigned long long));
    uint32_t ne = (uint32_t)P.entries.size();
    uint64_t tu = total;
    const volatile uint32_t *cancel_v = cancel;
    void *args[] = {(void *)&de,   (void *)&ne,    (void *)&tu,          (void *)&counters, (void *)&abort_flag,
                    (void *)&next, (void *)&trace, (void *)&trace_items, (void *)&cancel_v, (void *)&status};
    ce = cudaLaunchCooperativeKernel((const void *)fused_commit_kernel, dim3((unsigned)(per_sm * sms)),
                                     dim3(FUSED_THREADS), args, P.smem, stream);
    count_launches(1);
  }
  const cudaError_t fe = cudaFreeAsync(buf, stream);
  return (int)(ce != cudaSuccess ? ce : fe);
}

extern "C" glc_status glc_commit_batch_fused(const glc_commit_job *jobs, uint32_t n_jobs, void *stream) {
  return commit_batch_fused(jobs, n_jobs, nullptr, 0, nullptr, nullptr, stream);
}

extern "C" glc_status glc_commit_batch_fused_traced(const glc_commit_job *jobs, uint32_t n_jobs, uint64_t *trace,
                                                    uint64_t trace_items, void *stream) {
  if (!trace && trace_items) return fail("commit_batch_fused_traced: null trace buffer");
  return commit_batch_fused(jobs, n_jobs, reinterpret_cast<unsigned long long *>(trace), trace_items, nullptr, nullptr,
                            stream);
}

extern "C" glc_status glc_commit_batch_fused_cancellable(const glc_commit_job *jobs, uint32_t n_jobs,
                                                         const uint32_t *cancel, uint32_t *status, void *stream) {
  if (!cancel) return fail("commit_batch_fused_cancellable: null cancel word");
  return commit_batch_fused(jobs, n_jobs, nullptr, 0, cancel, status, stream);
}

extern "C" glc_status glc_mapped_word_create(uint32_t **host, uint32_t **device) {
  if (!host || !device) return fail("mapped_word_create: null output");
  *host = nullptr;
  *device = nullptr;
  uint32_t *h = nullptr;
  cudaError_t e = cudaHostAlloc((void **)&h, sizeof(uint32_t), cudaHostAllocMapped);
  if (e != cudaSuccess) return (int)e;
  *h = 0;
  uint32_t *d = nullptr;
  e = cudaHostGetDevicePointer((void **)&d, h, 0);
  if (e != cudaSuccess) {
    cudaFreeHost(h);
    return (int)e;
  }
  *host = h;
  *device = d;
  return 0;
}

extern "C" glc_status glc_mapped_word_destroy(uint32_t *host) { return host ? (int)cudaFreeHost(host) : 0; }

extern "C" glc_status glc_commit_batch_fused_timeouts(uint64_t *out) {
  if (!out) return fail("commit_batch_fused_timeouts: null output");
  unsigned long long v = 0;
  const cudaError_t e = cudaMemcpyFromSymbol(&v, g_fused_timeouts, sizeof(v));
  *out = v;
  return (int)e;
}
