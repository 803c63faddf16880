// Fused batch of small commitments: ONE cooperative launch runs every stage of every job.
//
// The per-call form issues about 28 kernels per commitment (NTT passes, bit reversal, one leaf
// launch and node layers per coset, the cap gather); for jobs of 2^12..2^16 rows each of those
// kernels runs for microseconds and cannot fill 148 SMs, so a batch of such jobs is bound by
// launch latency and by the tails of small grids (the reference's per-stage and per-layer
// launches, crates/boojum-cuda/src/ntt.rs:201-241 and src/poseidon2.rs:276-295, are the same
// shape).  Here a persistent grid (as many CTAs as fit on the device at once) walks a table of
// work items, stage by stage:
//   inverse NTT pass 1, pass 2 -> bit reversal -> forward coset NTT pass 1, pass 2 (the coset
//   that transforms the monomials in place last, in steps of its own) -> leaf hashes -> node
//   layer 1, 2, ... -> cap gather,
// with a grid-wide barrier (cooperative groups grid.sync) between steps.  Within a step every
// work item of every job is independent: an NTT tile, 256 rows of a bit reversal, 256 leaves,
// 256 nodes, 256 cap entries.  The items reuse the tile and hash code of the per-call kernels
// (ntt_pass_tile, leaf_hash, hash_node), so the results are the same bits.
//
// Included at the end of poseidon2.cu: it needs that file's __constant__ round constants.
#pragma once
#include <cooperative_groups.h>

#include <vector>

#include "ntt_tile.cuh"

namespace glc {

namespace cg = cooperative_groups;

static constexpr uint32_t FUSED_THREADS = 256;
static constexpr uint32_t FUSED_MAX_LOG_N = 16;

enum FusedKind : uint32_t { FK_NTT = 0, FK_BITREV = 1, FK_LEAVES = 2, FK_NODES = 3, FK_CAPS = 4 };

// One job's share of one step.  Units are numbered across the entries of a step.
struct FusedEntry {
  uint64_t first;          // the step's unit number of this entry's first unit
  uint64_t units;
  uint32_t kind;
  uint32_t log_rows;       // bit reversal: log2 of the rows
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

struct FusedStep {
  uint32_t first_entry, entries;
  uint64_t units;
};

__global__ void __launch_bounds__(FUSED_THREADS, 3) fused_commit_kernel(const FusedEntry *entries, const FusedStep *steps,
                                                                        uint32_t n_steps) {
  extern __shared__ uint64_t smem[];
  cg::grid_group grid = cg::this_grid();
  const uint32_t tid = threadIdx.x;
  for (uint32_t st = 0; st < n_steps; st++) {
    const FusedStep S = steps[st];
    for (uint64_t u = blockIdx.x; u < S.units; u += gridDim.x) {
      // the entry holding unit u: the last one whose first unit is <= u (uniform per CTA)
      uint32_t lo = S.first_entry, hi = S.first_entry + S.entries - 1;
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (entries[mid].first <= u)
          lo = mid;
        else
          hi = mid - 1;
      }
      const FusedEntry &E = entries[lo];
      const uint64_t local = u - E.first;
      const uint32_t kind = E.kind;
      if (kind == FK_NTT) {
        const PassArgs a = E.ntt;
        const uint64_t tpc = E.tiles_per_col;
        __syncthreads();  // the previous item's last reads of shared memory are done
        ntt_pass_tile<4>(a, (uint32_t)(local % tpc), (uint32_t)(local / tpc), smem);
      } else if (kind == FK_BITREV) {
        const uint32_t L = E.log_rows;
        const uint64_t n = 1ull << L, chunks = (n + FUSED_THREADS - 1) / FUSED_THREADS;
        const uint64_t col = local / chunks, i = (local % chunks) * FUSED_THREADS + tid;
        if (i < n) {
          const uint64_t r = brev_low((uint32_t)i, L);
          if (i < r) {
            uint64_t *x = E.dst + col * E.stride;
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
    }
    grid.sync();
  }
}

// Host side: builds the step table of a batch and launches the persistent grid.
struct FusedPlan {
  std::vector<FusedEntry> entries;
  std::vector<FusedStep> steps;
  size_t smem = 0;

  void begin_step() { steps.push_back({(uint32_t)entries.size(), 0, 0}); }
  void add(FusedEntry e) {
    FusedStep &s = steps.back();
    e.first = s.units;
    s.units += e.units;
    s.entries++;
    entries.push_back(e);
  }
  void end_step() {
    if (steps.back().entries == 0) steps.pop_back();
  }
};

static uint32_t fused_brev(uint32_t x, uint32_t bits) {
  uint32_t r = 0;
  for (uint32_t i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

static FusedEntry ntt_entry(const DeviceTables *t, uint32_t log_n, uint32_t q, uint32_t np, const Pass &ps,
                            const uint64_t *in, uint64_t *out, uint64_t in_stride, uint64_t out_stride, uint32_t cols,
                            bool inverse, uint32_t log_ext, uint32_t coset, size_t &smem) {
  FusedEntry e{};
  e.kind = FK_NTT;
  NttTuning tu = ntt_tuning(log_n);
  tu.radix_bits = 4;
  const PassShape sh = make_pass(e.ntt, t, tu, ps, q, np, in, out, in_stride, out_stride, cols, log_n, false, inverse,
                                 log_ext, coset, tu.max_cols_per_cta);
  e.tiles_per_col = sh.tiles_per_col;
  e.units = sh.tiles_per_col * sh.groups;
  smem = std::max(smem, sh.smem);
  return e;
}

static int fused_plan(const DeviceTables *t, const glc_commit_job *jobs, uint32_t n_jobs, FusedPlan &P) {
  auto units = [](uint64_t n) { return (n + FUSED_THREADS - 1) / FUSED_THREADS; };
  struct J {
    const glc_commit_job *j;
    uint64_t n, f, coset_elems;
    uint64_t *mono;
    Pass inv[2], fwd[2];
    uint32_t np;
    uint32_t layers;  // tree layers including the leaves
  };
  std::vector<J> js(n_jobs);
  uint32_t max_layers = 0;
  for (uint32_t i = 0; i < n_jobs; i++) {
    J &x = js[i];
    x.j = &jobs[i];
    x.n = 1ull << jobs[i].log_n;
    x.f = 1ull << jobs[i].log_lde;
    x.coset_elems = x.n * jobs[i].cols;
    x.mono = jobs[i].monomials ? jobs[i].monomials : jobs[i].lde + (x.f - 1) * x.coset_elems;
    const NttTuning &tu = ntt_tuning(jobs[i].log_n);
    x.np = make_plan(jobs[i].log_n, false, tu, x.inv);
    make_plan(jobs[i].log_n, false, tu, x.fwd);
    // tiles of at most 2^12 elements: 96 KB of shared memory at most, two CTAs per SM
    for (uint32_t q = 0; q < x.np; q++) {
      x.inv[q].log_w = std::min(x.inv[q].log_w, SINGLE_PASS_MAX_LOG - x.inv[q].k);
      x.fwd[q].log_w = std::min(x.fwd[q].log_w, SINGLE_PASS_MAX_LOG - x.fwd[q].k);
    }
    x.layers = jobs[i].log_n - (jobs[i].log_cap - jobs[i].log_lde) + 1;
    max_layers = std::max(max_layers, x.layers);
  }
  // inverse NTT (evaluations -> bit-reversed coefficients x N^-1), pass by pass
  for (uint32_t q = 0; q < 2; q++) {
    P.begin_step();
    for (J &x : js)
      if (q < x.np)
        P.add(ntt_entry(t, x.j->log_n, q, x.np, x.inv[q], x.j->evals, x.mono, x.j->evals_stride, x.n, x.j->cols, true, 0,
                        0, P.smem));
    P.end_step();
  }
  // bit reversal: natural-order monomials
  P.begin_step();
  for (J &x : js) {
    FusedEntry e{};
    e.kind = FK_BITREV;
    e.log_rows = x.j->log_n;
    e.dst = x.mono;
    e.stride = x.n;
    e.units = (uint64_t)x.j->cols * units(x.n);
    P.add(e);
  }
  P.end_step();
  // forward coset NTTs; without a monomials buffer the last coset transforms the monomials in
  // place, so it runs after the steps of the other cosets, which read them
  for (int last = 0; last < 2; last++)
    for (uint32_t q = 0; q < 2; q++) {
      P.begin_step();
      for (J &x : js) {
        if (q >= x.np) continue;
        for (uint64_t c = 0; c < x.f; c++) {
          const bool in_place_last = !x.j->monomials && c == x.f - 1;
          if (in_place_last != (last == 1)) continue;
          P.add(ntt_entry(t, x.j->log_n, q, x.np, x.fwd[q], x.mono, x.j->lde + c * x.coset_elems, x.n, x.n, x.j->cols,
                          false, x.j->log_lde, fused_brev((uint32_t)c, x.j->log_lde), P.smem));
        }
      }
      P.end_step();
    }
  // leaf hashes of every coset
  P.begin_step();
  for (J &x : js)
    for (uint64_t c = 0; c < x.f; c++) {
      FusedEntry e{};
      e.kind = FK_LEAVES;
      e.src = x.j->lde + c * x.coset_elems;
      e.dst = x.j->trees + c * 8 * x.n;
      e.count = x.n;
      e.cols = x.j->cols;
      e.units = units(x.n);
      P.add(e);
    }
  P.end_step();
  // node layers: layer l (parent count n >> l) starts at 8n - 8n / 2^l in the subtree buffer
  for (uint32_t l = 1; l < max_layers; l++) {
    P.begin_step();
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
        P.add(e);
      }
    }
    P.end_step();
  }
  // caps
  P.begin_step();
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
    P.add(e);
  }
  P.end_step();
  return 0;
}

}  // namespace glc

using namespace glc;

extern "C" glc_status glc_commit_batch_fused(const glc_commit_job *jobs, uint32_t n_jobs, void *stream_) {
  if (n_jobs == 0) return 0;
  if (!jobs) return fail("commit_batch_fused: null jobs");
  for (uint32_t i = 0; i < n_jobs; i++) {
    const int e = commit_check(jobs[i]);
    if (e) return e;
    if (jobs[i].log_n > FUSED_MAX_LOG_N) return fail("commit_batch_fused: log_n must be <= 16");
  }
  const DeviceTables *t = current_tables();
  if (!t) return fail("commit_batch_fused: glc_context_create has not been called on this device");
  FusedPlan P;
  int e = fused_plan(t, jobs, n_jobs, P);
  if (e) return e;
  cudaStream_t stream = (cudaStream_t)stream_;
  cudaError_t ce = cudaFuncSetAttribute(fused_commit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.smem);
  int dev = 0, sms = 0, per_sm = 0;
  if (ce == cudaSuccess) ce = cudaGetDevice(&dev);
  if (ce == cudaSuccess) ce = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (ce == cudaSuccess)
    ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fused_commit_kernel, FUSED_THREADS, P.smem);
  if (ce != cudaSuccess) return (int)ce;
  if (per_sm < 1) return fail("commit_batch_fused: the kernel does not fit on an SM");
  const size_t eb = P.entries.size() * sizeof(FusedEntry), sb = P.steps.size() * sizeof(FusedStep);
  char *buf = nullptr;
  ce = cudaMallocAsync((void **)&buf, eb + sb, stream);
  if (ce != cudaSuccess) return (int)ce;
  // pageable source: the copies are staged before they return, so the host tables may go
  ce = cudaMemcpyAsync(buf, P.entries.data(), eb, cudaMemcpyHostToDevice, stream);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(buf + eb, P.steps.data(), sb, cudaMemcpyHostToDevice, stream);
  if (ce == cudaSuccess) {
    const FusedEntry *de = reinterpret_cast<const FusedEntry *>(buf);
    const FusedStep *ds = reinterpret_cast<const FusedStep *>(buf + eb);
    uint32_t ns = (uint32_t)P.steps.size();
    void *args[] = {(void *)&de, (void *)&ds, (void *)&ns};
    ce = cudaLaunchCooperativeKernel((const void *)fused_commit_kernel, dim3((unsigned)(per_sm * sms)),
                                     dim3(FUSED_THREADS), args, P.smem, stream);
    count_launches(1);
  }
  const cudaError_t fe = cudaFreeAsync(buf, stream);
  return (int)(ce != cudaSuccess ? ce : fe);
}
