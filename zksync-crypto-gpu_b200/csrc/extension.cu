// GoldilocksExt2 column layouts: vectorized <-> tuples.
//
// Replaces boojum-cuda's extension_field::convert (crates/boojum-cuda/src/extension_field.rs:60-90;
// kernels native/goldilocks_extension.cu:8-34, accessors native/memory.cuh:545-612):
//   vectorized: extension column k is two base columns, c0 at v[2k*v_stride + row] and c1 at
//               v[(2k+1)*v_stride + row];
//   tuples:     element (row, k) is the 16-byte pair {c0, c1} at t[2*(k*t_stride + row)].
// Pure data movement (16 bytes read and 16 written per element), so the kernel is shaped for
// HBM: each thread moves two consecutive rows, which makes every access a 16-byte vector access
// when the vectorized side is 16-byte aligned (even stride, aligned base), and falls back to
// 8-byte accesses otherwise.
#include <algorithm>

#include "glc_internal.h"

namespace glc {

template <bool TO_TUPLES, bool VEC>
__global__ void __launch_bounds__(256) ef_convert_kernel(const uint64_t *src, uint64_t src_stride, uint64_t *dst,
                                                         uint64_t dst_stride, uint32_t rows, uint32_t cols) {
  const uint32_t pairs = (rows + 1) / 2;
  const uint64_t v_stride = TO_TUPLES ? src_stride : dst_stride;
  const uint64_t t_stride = TO_TUPLES ? dst_stride : src_stride;
  for (uint32_t k = blockIdx.y; k < cols; k += gridDim.y) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pairs) return;
    const uint64_t r = 2ull * i;
    const bool two = r + 1 < rows;
    const uint64_t vc0 = 2ull * k * v_stride + r, vc1 = vc0 + v_stride, tp = 2 * ((uint64_t)k * t_stride + r);
    if (TO_TUPLES) {
      uint64_t a0, a1, b0 = 0, b1 = 0;  // c0, c1 of rows r and r + 1
      if (VEC && two) {
        const ulonglong2 x = __ldcs(reinterpret_cast<const ulonglong2 *>(src + vc0));
        const ulonglong2 y = __ldcs(reinterpret_cast<const ulonglong2 *>(src + vc1));
        a0 = x.x, b0 = x.y, a1 = y.x, b1 = y.y;
      } else {
        a0 = __ldcs(src + vc0), a1 = __ldcs(src + vc1);
        if (two) b0 = __ldcs(src + vc0 + 1), b1 = __ldcs(src + vc1 + 1);
      }
      __stcs(reinterpret_cast<ulonglong2 *>(dst + tp), make_ulonglong2(a0, a1));
      if (two) __stcs(reinterpret_cast<ulonglong2 *>(dst + tp + 2), make_ulonglong2(b0, b1));
    } else {
      const ulonglong2 a = __ldcs(reinterpret_cast<const ulonglong2 *>(src + tp));
      if (VEC && two) {
        const ulonglong2 b = __ldcs(reinterpret_cast<const ulonglong2 *>(src + tp + 2));
        __stcs(reinterpret_cast<ulonglong2 *>(dst + vc0), make_ulonglong2(a.x, b.x));
        __stcs(reinterpret_cast<ulonglong2 *>(dst + vc1), make_ulonglong2(a.y, b.y));
      } else {
        __stcs(dst + vc0, a.x);
        __stcs(dst + vc1, a.y);
        if (two) {
          const ulonglong2 b = __ldcs(reinterpret_cast<const ulonglong2 *>(src + tp + 2));
          __stcs(dst + vc0 + 1, b.x);
          __stcs(dst + vc1 + 1, b.y);
        }
      }
    }
  }
}

static int ef_convert(bool to_tuples, const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride,
                      uint32_t rows, uint32_t cols, cudaStream_t stream) {
  // extension_field.rs:66-77 (rows and columns of both sides agree by construction here)
  if (rows == 0 || cols == 0) return 0;
  if (!src || !dst) return fail("ef convert: null matrix");
  if (src_stride < rows || dst_stride < rows) return fail("ef convert: stride smaller than the rows");
  // the tuple side is read and written as 16-byte pairs
  const uint64_t *t = to_tuples ? dst : src;
  if (reinterpret_cast<uintptr_t>(t) & 15) return fail("ef convert: tuple matrix not 16-byte aligned");
  const uint64_t *v = to_tuples ? src : dst;
  const uint64_t v_stride = to_tuples ? src_stride : dst_stride;
  const bool vec = (reinterpret_cast<uintptr_t>(v) & 15) == 0 && (v_stride & 1) == 0;
  const uint32_t pairs = (rows + 1) / 2;
  const dim3 grid((pairs + 255) / 256, std::min<uint32_t>(cols, 65535));
#define GLC_EF(T, V) ef_convert_kernel<T, V><<<grid, 256, 0, stream>>>(src, src_stride, dst, dst_stride, rows, cols)
  if (to_tuples && vec)
    GLC_EF(true, true);
  else if (to_tuples)
    GLC_EF(true, false);
  else if (vec)
    GLC_EF(false, true);
  else
    GLC_EF(false, false);
#undef GLC_EF
  return last_launch_error();
}

}  // namespace glc

using namespace glc;

extern "C" glc_status glc_ef_vectorized_to_tuples(const uint64_t *src, uint64_t src_stride, uint64_t *dst,
                                                 uint64_t dst_stride, uint32_t rows, uint32_t cols, void *stream) {
  return ef_convert(true, src, src_stride, dst, dst_stride, rows, cols, (cudaStream_t)stream);
}

extern "C" glc_status glc_ef_tuples_to_vectorized(const uint64_t *src, uint64_t src_stride, uint64_t *dst,
                                                 uint64_t dst_stride, uint32_t rows, uint32_t cols, void *stream) {
  return ef_convert(false, src, src_stride, dst, dst_stride, rows, cols, (cudaStream_t)stream);
}
