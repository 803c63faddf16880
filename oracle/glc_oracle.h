/*
 * glc_oracle.h -- CPU oracle for the Goldilocks LDE + Poseidon2 Merkle commitment path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the algorithms of
 * boojum-cuda (crates/boojum-cuda) and of the boojum 0.32.10 CPU routines it is tested
 * against.  Only the test suite, the smoke check and the CPU-baseline leg of the benchmark
 * may load it.  The product library never links it and never falls back to it.
 *
 * Parity status:
 *   - NTT / LDE definitions follow the reference's own test oracle
 *     (crates/boojum-cuda/src/ntt.rs:527-583) with roots of unity
 *     w_{2^k} = 7^((p-1)/2^k) (the multiplicative generator 7, crates/boojum-cuda/src/context.rs:232).
 *     The choice of w is pinned against the reference GPU kernels driven with the same
 *     tables; boojum's own domain_generator_for_size is not available in this environment.
 *   - Poseidon2 follows crates/boojum-cuda/native/poseidon2/gl/.  Its round constants come
 *     from boojum (build/poseidon2_gl.rs:3,34), which is not available here; the oracle takes
 *     the constants as an input (or_p2_set_round_constants), so that it can be run with the
 *     placeholder set shipped with the library or with the real set when a user supplies it.
 *
 * Every element is a uint64_t in [0, 2^64), not necessarily canonical; results are canonical.
 */
#ifndef GLC_ORACLE_H
#define GLC_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_P 0xFFFFFFFF00000001ull

/* ---- field (crates/boojum-cuda/native/goldilocks.cuh:90-185) ---- */
uint64_t or_canon(uint64_t a);
uint64_t or_add(uint64_t a, uint64_t b);
uint64_t or_sub(uint64_t a, uint64_t b);
uint64_t or_mul(uint64_t a, uint64_t b);
uint64_t or_pow(uint64_t a, uint64_t e);
uint64_t or_inv(uint64_t a);
/* w_{2^log_n} = 7^((p-1) >> log_n) */
uint64_t or_root_of_unity(uint32_t log_n);

/* ---- NTT (crates/boojum-cuda/src/ntt.rs:179-369, semantics from ntt.rs:527-583) ----
 * Column k of the input is in[k*in_stride .. k*in_stride + 2^log_n), same for the output.
 * in == out is the in-place form.  Returns 0, or -1 on a contract violation. */
int or_batch_ntt(const uint64_t *in, uint64_t *out, uint32_t log_n, uint32_t num_ntts, uint64_t in_stride,
                 uint64_t out_stride, int bitrev_inputs, int inverse, uint32_t log_extension_degree,
                 uint32_t coset_idx, int threads);

/* O(n^2) direct evaluation of the same definitions, for small-size self checks. */
int or_batch_ntt_naive(const uint64_t *in, uint64_t *out, uint32_t log_n, uint32_t num_ntts, uint64_t in_stride,
                       uint64_t out_stride, int bitrev_inputs, int inverse, uint32_t log_extension_degree,
                       uint32_t coset_idx);

/* ---- bit reverse (crates/boojum-cuda/native/ops_complex.cu:88-156) ---- */
void or_bit_reverse(const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride, uint32_t log_rows,
                    uint32_t cols);

/* ---- Poseidon2, width 12 (crates/boojum-cuda/native/poseidon2/gl/poseidon2_gl_st.cu:9-23) ---- */
void or_p2_set_round_constants(const uint64_t rc[30 * 12]);
void or_p2_permutation(uint64_t state[12]);

/* Leaf hashes (poseidon2_gl_st.cu:25-59, crates/boojum-cuda/src/poseidon2.rs:180-226).
 * results has results_len = 4*count entries, digest element j of leaf i at j*count+i. */
int or_p2_leaves(const uint64_t *values, size_t values_len, uint64_t *results, size_t results_len,
                 uint32_t log_rows_per_hash, int load_intermediate, int store_intermediate, int threads);
/* Node hashes (poseidon2_gl_st.cu:61-82, poseidon2.rs:228-251): values [4][2*count] -> results [4][count]. */
int or_p2_nodes(const uint64_t *values, size_t values_len, uint64_t *results, size_t results_len, int threads);
/* build_merkle_tree (poseidon2.rs:297-314): results_len = 2*4*leaves; unused tail untouched. */
int or_p2_build_merkle_tree(const uint64_t *values, size_t values_len, uint64_t *results, size_t results_len,
                            uint32_t log_rows_per_hash, uint32_t layers_count, int threads);
/* gather_rows (native/poseidon2/queries.cuh:9-19): values is rows x cols column-major with
 * column stride values_stride, result has indexes_count<<log_rows_per_index rows, stride result_stride. */
void or_p2_gather_rows(const uint32_t *indexes, uint32_t indexes_count, uint32_t log_rows_per_index,
                       const uint64_t *values, uint64_t values_stride, uint32_t cols, uint64_t *results,
                       uint64_t result_stride);
/* gather_merkle_paths (queries.cuh:21-37, poseidon2.rs:350-380). */
int or_p2_gather_merkle_paths(const uint32_t *indexes, uint32_t indexes_count, const uint64_t *values,
                              size_t values_len, uint32_t layers_count, uint64_t *results, size_t results_len);

/* Known-answer check on a Merkle opening whose leaf index is not recorded (the query records of
 * crates/shivini/test_data/compression/scheduler_recursive_proof.json): hash leaf_len values as
 * one leaf, climb `depth` levels of `path` ([depth][4] digests) trying both child orders, and
 * return the leaf index whose root equals one of the cap_len cap digests ([cap_len][4]), or -1. */
int64_t or_p2_find_opening(const uint64_t *leaf, uint32_t leaf_len, const uint64_t *path, uint32_t depth,
                           const uint64_t *cap, uint32_t cap_len);

/* ---- commitment job (shivini trace commitment: storage.rs:155-330, cache.rs:353-418) ----
 * evals: cols columns of 2^log_n natural-order evaluations (column stride 2^log_n).
 * monomials_out (optional, may be NULL): cols x 2^log_n natural-order coefficients.
 * lde_out: 2^log_lde cosets, each cols x 2^log_n, bit-reversed evaluations; coset c is at
 *          lde_out + c*cols*2^log_n and uses kernel coset index bitrev(c).
 * trees_out: one Merkle subtree per coset, each 2*4*2^log_n entries, subtree cap 2^(log_cap-log_lde).
 * cap_out: 4*2^log_cap entries, [4][cap] layout (coset caps concatenated). */
/* GoldilocksExt2 column layouts (crates/boojum-cuda/src/extension_field.rs:60-90,
 * native/goldilocks_extension.cu:8-34, native/memory.cuh:545-612).  Vectorized: extension column
 * k is two base columns, c0 at v[2*k*v_stride + row] and c1 at v[(2*k+1)*v_stride + row].
 * Tuples: element (row, k) is the pair {c0, c1} at t[2*(k*t_stride + row)]. */
void or_ef_vectorized_to_tuples(const uint64_t *v, uint64_t v_stride, uint64_t *t, uint64_t t_stride, uint32_t rows,
                                uint32_t cols);
void or_ef_tuples_to_vectorized(const uint64_t *t, uint64_t t_stride, uint64_t *v, uint64_t v_stride, uint32_t rows,
                                uint32_t cols);

/* ops_complex::select (native/ops_complex.cu:158-164): dst[i] = indexes[i] has bit 31 set ? 0 :
 * src[indexes[i]].  An index at or past src_len reads as 0 (the library's defined behaviour for
 * what the reference leaves unchecked). */
void or_select(const uint32_t *indexes, uint64_t count, const uint64_t *src, uint64_t src_len, uint64_t *dst);
/* GenericTraceStorage::fill_from_remote_witness_data (crates/shivini/src/data_structures/
 * trace.rs:108-193): nv variable columns and nw witness columns selected from `values`, then nm
 * (0 or 1) columns of multiplicities zero-padded to n rows; trace is (nv + nw + nm) x n. */
void or_trace_fill(const uint32_t *variable_indexes, const uint32_t *witness_indexes, const uint64_t *values,
                   uint64_t values_len, const uint32_t *multiplicities, uint64_t multiplicities_len, uint64_t *trace,
                   uint32_t nv, uint32_t nw, uint32_t nm, uint64_t n);

int or_commit(const uint64_t *evals, uint32_t log_n, uint32_t cols, uint32_t log_lde, uint32_t log_cap,
              uint64_t *monomials_out, uint64_t *lde_out, uint64_t *trees_out, uint64_t *cap_out, int threads);

#ifdef __cplusplus
}
#endif
#endif
