/*
 * bc_barycentric.h -- C ABI of barycentric evaluation on a coset domain, the
 * replacement of era-boojum-cuda's src/barycentric.rs (kernels
 * native/barycentric.cu), in libbc_ntt.so.
 *
 * A batch of polynomials is given by their values on the coset c * H,
 * H = <w>, |H| = count = 2^k (w = w_{2^k}, the generator-7 roots of
 * bc_ntt.h), and evaluated at a point x of the base field or of its quadratic
 * extension F_p[x]/(x^2 - 7):
 *   L_i(x)  = cf * w^i / (x - c w^i) = cf / (x w^-i - c),
 *   cf      = c (x^count - c^count) / (count c^count),
 *   eval_j  = sum_i y_{i,j} L_i(x).
 * When x lies in c * H every L_i is 0, as in the reference.  Layouts as in
 * the reference (native/memory.cuh:436-590): an extension vector of n
 * elements is all first coordinates then all second coordinates; column j of
 * an extension matrix with `count` rows is the base-field columns 2j (first
 * coordinates) and 2j + 1; the evaluations of extension kind are (c0, c1)
 * pairs, one per polynomial.  Results are canonical.  Asynchronous on the
 * given stream; requires bc_ntt_context_create on the device.
 */
#ifndef BC_BARYCENTRIC_H
#define BC_BARYCENTRIC_H

#include <cuda_runtime_api.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* EvalBaseAtBase, EvalBaseAtExt, EvalExtAtExt (src/barycentric.rs:279-281):
 * values in the base field or the extension, point in the base field or the
 * extension. */
enum {
  BC_EVAL_BASE_AT_BASE = 0,
  BC_EVAL_BASE_AT_EXT = 1,
  BC_EVAL_EXT_AT_EXT = 2
};

/* Replaces precompute_lagrange_coeffs::<PrecomputeAtBase> (src/barycentric.rs:83-126):
 * x and common_factor_storage point to one device word each; lagrange_coeffs
 * receives count = 2^k coefficients, in bit-reversed order when bit_reverse. */
cudaError_t bc_precompute_lagrange_coeffs_at_base(const uint64_t *x, uint64_t *common_factor_storage, uint64_t coset,
                                                  uint64_t *lagrange_coeffs, uint32_t count, bool bit_reverse,
                                                  cudaStream_t stream);

/* The same for PrecomputeAtExt: x and common_factor_storage hold (c0, c1);
 * lagrange_coeffs is an extension vector of count elements (2 * count words). */
cudaError_t bc_precompute_lagrange_coeffs_at_ext(const uint64_t *x, uint64_t *common_factor_storage, uint64_t coset,
                                                 uint64_t *lagrange_coeffs, uint32_t count, bool bit_reverse,
                                                 cudaStream_t stream);

/* Replaces get_batch_eval_temp_storage_sizes (src/barycentric.rs:193-209): the
 * scratch batch_eval needs for `num_polys` polynomials of `count` rows, in
 * u64 words for the partial sums and bytes for the final reduction (0 here). */
cudaError_t bc_get_batch_eval_temp_storage_sizes(int kind, uint32_t count, uint32_t num_polys,
                                                 size_t *partial_reduce_temp_words, size_t *final_reduce_temp_bytes);

/* Replaces batch_eval (src/barycentric.rs:211-260): batch_ys is a column-major
 * matrix of num_polys columns of count rows (stride count; extension kind:
 * 2 * num_polys base-field columns), lagrange_coeffs the vector of the
 * matching precompute, evals num_polys values ((c0, c1) pairs for the
 * extension kinds).  The scratch sizes must be at least those reported above. */
cudaError_t bc_batch_eval(int kind, const uint64_t *batch_ys, uint32_t count, uint32_t num_polys,
                          const uint64_t *lagrange_coeffs, uint64_t *temp_partial_reduce,
                          size_t temp_partial_reduce_words, void *temp_final_reduce, size_t temp_final_reduce_bytes,
                          uint64_t *evals, cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* BC_BARYCENTRIC_H */
