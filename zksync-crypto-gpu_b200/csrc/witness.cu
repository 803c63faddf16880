// Witness-to-trace fill: the trace matrix a commitment starts from, built from the prover's
// witness values.
//
// Replaces boojum-cuda's ops_complex::select (crates/boojum-cuda/src/ops_complex.rs:446-463,
// kernel native/ops_complex.cu:158-164) and the sequence shivini runs around it,
// GenericTraceStorage::fill_from_remote_witness_data (crates/shivini/src/data_structures/
// trace.rs:108-193, with cs/witness.rs:6-31):
//   select:  dst[i] = indexes[i] has bit 31 set (a placeholder) ? 0 : src[indexes[i]]
//   fill:    the variable columns (num_variable_cols x domain_size indexes) and the witness
//            columns are selects from the witness values, stored column after column; the
//            multiplicity column (at most one) holds the lookup multiplicities (u32) as field
//            elements, zero-padded to the domain size.
// A gather: per element 4 bytes of index and 8 of value read (the value at a data-dependent
// address, so a 32-byte sector unless indexes cluster) and 8 bytes written; HBM-bound.  Each
// thread produces 4 consecutive outputs: one 16-byte index load, the 4 value loads issued
// together through the read-only path, two 16-byte streaming stores (scalar accesses when the
// buffers are not 16-byte aligned).  An index past the end of the source (and not a placeholder)
// reads as 0 rather than reading outside the buffer (the reference does not check).  Measured on
// B200 (2^22 rows x 175 gathered columns from 2^28 values): 15.8 ms against 16.4 ms for the
// reference's one-thread-per-index kernel, bit-identical.
#include <algorithm>

#include "glc_internal.h"

namespace glc {

static constexpr uint32_t PLACEHOLDER_BIT = 1u << 31;  // ops_complex.cu:162
static constexpr uint32_t WITNESS_THREADS = 256;

__device__ __forceinline__ uint64_t select_one(uint32_t ix, const uint64_t *src, uint64_t src_len) {
  return (ix & PLACEHOLDER_BIT) || ix >= src_len ? 0ull : __ldg(src + ix);
}

template <bool VEC>
__global__ void __launch_bounds__(WITNESS_THREADS) select_kernel(const uint32_t *indexes, uint64_t count,
                                                                 const uint64_t *src, uint64_t src_len, uint64_t *dst) {
  const uint64_t quads = (count + 3) / 4;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < quads; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i0 = 4 * t;
    if (VEC && i0 + 4 <= count) {
      const uint4 ix = __ldcs(reinterpret_cast<const uint4 *>(indexes) + t);
      const uint64_t v0 = select_one(ix.x, src, src_len), v1 = select_one(ix.y, src, src_len);
      const uint64_t v2 = select_one(ix.z, src, src_len), v3 = select_one(ix.w, src, src_len);
      __stcs(reinterpret_cast<ulonglong2 *>(dst + i0), make_ulonglong2(v0, v1));
      __stcs(reinterpret_cast<ulonglong2 *>(dst + i0 + 2), make_ulonglong2(v2, v3));
    } else {
      for (uint64_t i = i0; i < min(i0 + 4, count); i++) __stcs(dst + i, select_one(__ldcs(indexes + i), src, src_len));
    }
  }
}

// dst[i] = multiplicities[i] (as a field element, u32 < p) for i < n, 0 for n <= i < rows
__global__ void __launch_bounds__(WITNESS_THREADS) multiplicity_kernel(const uint32_t *mult, uint64_t n, uint64_t *dst,
                                                                       uint64_t rows) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (uint64_t)gridDim.x * blockDim.x)
    __stcs(dst + i, i < n ? (uint64_t)__ldcs(mult + i) : 0ull);
}

// grid: one thread per item (the loops stride by the grid only past 2^31 - 1 CTAs).  For the
// gather this beats a grid of a few CTAs per SM looping over the items by 19% on B200: CTAs that
// start while others drain keep more independent loads in flight than a fixed set of threads
// that each wait for their previous quad.
static uint32_t witness_grid(uint64_t items) {
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((items + WITNESS_THREADS - 1) / WITNESS_THREADS, 0x7FFFFFFFull));
}

static int select_launch(const uint32_t *indexes, uint64_t count, const uint64_t *src, uint64_t src_len, uint64_t *dst,
                         cudaStream_t stream) {
  if (count == 0) return 0;
  const bool vec = ((reinterpret_cast<uintptr_t>(indexes) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0;
  const uint32_t grid = witness_grid((count + 3) / 4);
  if (vec)
    select_kernel<true><<<grid, WITNESS_THREADS, 0, stream>>>(indexes, count, src, src_len, dst);
  else
    select_kernel<false><<<grid, WITNESS_THREADS, 0, stream>>>(indexes, count, src, src_len, dst);
  return last_launch_error();
}

}  // namespace glc

using namespace glc;

extern "C" glc_status glc_select(const uint32_t *indexes, uint64_t indexes_len, const uint64_t *src, uint64_t src_len,
                                 uint64_t *dst, uint64_t dst_len, void *stream) {
  // ops_complex.rs:452-455: every length fits in u32; the kernel writes dst[0 .. indexes_len)
  if (indexes_len > 0xFFFFFFFFull || src_len > 0xFFFFFFFFull || dst_len > 0xFFFFFFFFull)
    return fail("select: a length exceeds u32::MAX");
  if (dst_len < indexes_len) return fail("select: dst shorter than indexes");
  if (indexes_len && (!indexes || !dst)) return fail("select: null buffer");
  if (indexes_len && src_len && !src) return fail("select: null source");
  return select_launch(indexes, indexes_len, src, src_len, dst, (cudaStream_t)stream);
}

extern "C" glc_status glc_trace_fill_from_witness(const uint32_t *variable_indexes, uint64_t variable_indexes_len,
                                                  const uint32_t *witness_indexes, uint64_t witness_indexes_len,
                                                  const uint64_t *values, uint64_t values_len,
                                                  const uint32_t *multiplicities, uint64_t multiplicities_len,
                                                  uint64_t *trace, uint64_t trace_len, uint32_t num_variable_cols,
                                                  uint32_t num_witness_cols, uint32_t num_multiplicity_cols,
                                                  uint64_t domain_size, void *stream) {
  cudaStream_t st = (cudaStream_t)stream;
  // trace.rs:117-127: the index arrays cover their columns exactly; at most one multiplicity column
  if ((uint64_t)num_variable_cols * domain_size != variable_indexes_len)
    return fail("trace fill: num_variable_cols * domain_size != variable_indexes_len");
  if ((uint64_t)num_witness_cols * domain_size != witness_indexes_len)
    return fail("trace fill: num_witness_cols * domain_size != witness_indexes_len");
  if (num_multiplicity_cols > 1) return fail("trace fill: at most one multiplicity column");
  // trace.rs:137: the storage holds every column
  const uint64_t cols = (uint64_t)num_variable_cols + num_witness_cols + num_multiplicity_cols;
  if (cols * domain_size != trace_len) return fail("trace fill: trace_len != columns * domain_size");
  // witness.rs:14: values to select from; select's u32 limits
  if ((variable_indexes_len || witness_indexes_len) && (values_len == 0 || !values))
    return fail("trace fill: no witness values");
  if (values_len > 0xFFFFFFFFull || variable_indexes_len > 0xFFFFFFFFull || witness_indexes_len > 0xFFFFFFFFull)
    return fail("trace fill: a length exceeds u32::MAX");
  // trace.rs:157-158: the multiplicities fit their column (ignored without one)
  if (num_multiplicity_cols && multiplicities_len > domain_size)
    return fail("trace fill: more multiplicities than rows");
  if (num_multiplicity_cols && multiplicities_len && !multiplicities) return fail("trace fill: null multiplicities");
  if (trace_len && !trace) return fail("trace fill: null trace");
  if ((variable_indexes_len && !variable_indexes) || (witness_indexes_len && !witness_indexes))
    return fail("trace fill: null indexes");
  int e = select_launch(variable_indexes, variable_indexes_len, values, values_len, trace, st);
  if (!e) e = select_launch(witness_indexes, witness_indexes_len, values, values_len, trace + variable_indexes_len, st);
  if (!e && num_multiplicity_cols && domain_size) {
    multiplicity_kernel<<<witness_grid(domain_size), WITNESS_THREADS, 0, st>>>(
        multiplicities, multiplicities_len, trace + variable_indexes_len + witness_indexes_len, domain_size);
    e = last_launch_error();
  }
  return e;
}
