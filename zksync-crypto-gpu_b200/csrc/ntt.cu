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
#include "ntt_tile.cuh"

namespace glc {

template <uint32_t RB>
__global__ void __launch_bounds__(pass_threads(RB), pass_min_blocks(RB)) ntt_pass_kernel(const PassArgs a) {
  extern __shared__ uint64_t smem[];
  ntt_pass_tile<RB>(a, blockIdx.x, blockIdx.y, smem);
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
      PassArgs a;
      const PassShape sh = make_pass(a, t, tu, ps, q, np, in + (uint64_t)c0 * in_stride, out + (uint64_t)c0 * out_stride,
                                     in_stride, out_stride, cols, log_n, bitrev_inputs, inverse, log_ext, coset_idx,
                                     tu.max_cols_per_cta);
      const uint64_t tiles_per_col = sh.tiles_per_col;
      const uint32_t cpc = a.cols_per_cta, gy = sh.groups, threads = sh.threads;
      const size_t smem = sh.smem;
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
