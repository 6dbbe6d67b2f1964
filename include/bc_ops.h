/*
 * bc_ops.h -- C ABI of the vector and matrix operations that sit beside the
 * NTT in era-boojum-cuda's src/ops_complex.rs, in libbc_ntt.so: the
 * bit-reversal permutation of matrix columns, table-driven powers of the
 * domain generators, powers of an arbitrary base (base field and its
 * quadratic extension) and the omega shift.
 *
 * Same conventions as bc_ntt.h: u64 words, column-major matrices (column j at
 * ptr + j * stride), asynchronous on the given stream, cudaErrorInvalidValue
 * where the reference asserts.  The powers and the omega shift read the
 * tables of bc_ntt_context_create and return cudaErrorInitializationError
 * without them.  Outputs are canonical (the reference leaves products
 * unreduced; its values are equal mod p).
 *
 * Domain conventions of the reference (native/context.cuh:9-48): omega is
 * w_{2^24} (OMEGA_LOG_ORDER = 24) and an exponent index is used mod 2^24, so
 * log_degree must be <= 24.  "g" is the multiplicative generator 7.
 *
 * Extension field: F_p[x] / (x^2 - 7) (native/goldilocks_extension.cuh:11).
 * A vector of `count` extension elements is stored as two base-field arrays,
 * all first coordinates then all second coordinates (result[i] and
 * result[i + count]), as the reference's kernels store it
 * (native/ops_complex.cu:53-64).
 */
#ifndef BC_OPS_H
#define BC_OPS_H

#include <cuda_runtime_api.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces bit_reverse (src/ops_complex.rs:271-318, kernels
 * native/ops_complex.cu:89-157): dst[brev(i)] = src[i] in each of `cols`
 * columns of 2^log_rows rows (log_rows <= 31).  src == dst (with equal
 * strides) permutes in place; other overlaps are not allowed. */
cudaError_t bc_bit_reverse(const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride,
                           uint32_t log_rows, uint32_t cols, cudaStream_t stream);

/* Replaces bit_reverse_in_place (src/ops_complex.rs:320-329). */
cudaError_t bc_bit_reverse_in_place(uint64_t *values, uint64_t stride, uint32_t log_rows, uint32_t cols,
                                    cudaStream_t stream);

/* Replaces get_powers_of_w (src/ops_complex.rs:40-85, kernel
 * native/ops_complex.cu:9-20): for i < count, with r = i + offset (u32) and
 * idx = bit_reverse ? brev_{log_degree}(r) : r,
 *   result[i] = w_{2^24}^{+-((idx << (24 - log_degree)) mod 2^24)}
 * (minus when inverse), i.e. powers of w_{2^log_degree}. */
cudaError_t bc_get_powers_of_w(uint32_t log_degree, uint32_t offset, bool inverse, bool bit_reverse,
                               uint64_t *result, uint32_t count, cudaStream_t stream);

/* Replaces get_powers_of_g (src/ops_complex.rs:40-86, kernel native/ops_complex.cu:22-33):
 * as above with base 7 (7^-1 when inverse) and the same exponent, i.e.
 * powers of 7^(2^(24 - log_degree)). */
cudaError_t bc_get_powers_of_g(uint32_t log_degree, uint32_t offset, bool inverse, bool bit_reverse,
                               uint64_t *result, uint32_t count, cudaStream_t stream);

/* Replace get_powers_by_val / get_powers_by_ref for the base field
 * (src/ops_complex.rs:117-205, kernels native/ops_complex.cu:35-52):
 * result[i] = base^e, e = (bit_reverse ? brev_32(i) : i) + offset (u32
 * arithmetic, all 32 bits reversed).  _by_ref reads base from device memory
 * when the kernel runs. */
cudaError_t bc_get_powers_by_val_bf(uint64_t base, uint32_t offset, bool bit_reverse, uint64_t *result,
                                    uint32_t count, cudaStream_t stream);
cudaError_t bc_get_powers_by_ref_bf(const uint64_t *base, uint32_t offset, bool bit_reverse, uint64_t *result,
                                    uint32_t count, cudaStream_t stream);

/* The same for the quadratic extension (kernels native/ops_complex.cu:54-74):
 * base = base_c0 + base_c1 x; result holds 2 * count words (see above).
 * _by_ref reads base_c0, base_c1 from base[0], base[1]. */
cudaError_t bc_get_powers_by_val_ef(uint64_t base_c0, uint64_t base_c1, uint32_t offset, bool bit_reverse,
                                    uint64_t *result, uint32_t count, cudaStream_t stream);
cudaError_t bc_get_powers_by_ref_ef(const uint64_t *base, uint32_t offset, bool bit_reverse, uint64_t *result,
                                    uint32_t count, cudaStream_t stream);

/* Replaces omega_shift (src/ops_complex.rs:207-242, kernel
 * native/ops_complex.cu:76-87): for i < count,
 *   dst[i] = src[i] * w_{2^24}^{+-(((shift * (i + offset)) << (24 - log_degree)) mod 2^24)}
 * (u32 arithmetic before the reduction; minus when inverse).  src == dst is
 * the in-place form. */
cudaError_t bc_omega_shift(const uint64_t *src, uint32_t log_degree, uint32_t offset, bool inverse, uint32_t shift,
                           uint64_t *dst, uint32_t count, cudaStream_t stream);

/* Replaces omega_shift_in_place (src/ops_complex.rs:244-258). */
cudaError_t bc_omega_shift_in_place(uint64_t *values, uint32_t log_degree, uint32_t offset, bool inverse,
                                    uint32_t shift, uint32_t count, cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* BC_OPS_H */
