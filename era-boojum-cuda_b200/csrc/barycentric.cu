// barycentric.cu -- barycentric evaluation on a coset domain (the reference's
// src/barycentric.rs and native/barycentric.cu); C ABI in
// include/bc_barycentric.h.
//
// Lagrange coefficients.  L_i = cf / (x w^-i - c) with
// cf = c (x^N - c^N) / (N c^N) (native/barycentric.cu:12-23, 47-52).  One
// thread computes cf into the caller's storage; the coefficient kernel walks
// w^-i as a running product over indexes 256 apart (w has order N, so the
// product is exact) and inverts its RUN_INV denominators together
// (Montgomery's trick: prefix products, one inversion, a backward pass).  An
// extension denominator is inverted through its norm, c0^2 - 7 c1^2, so the
// batch inversion stays in the base field.  If x lies in c * H a denominator
// is 0, the batch's inverse is 0 and so is cf: every coefficient is 0, as in
// the reference.  The optional bit reversal reuses the tiled kernel of ops.cu.
//
// Batch evaluation.  eval_j = sum_i y_{i,j} L_i: a dot product of every column
// with the coefficient vector, bound by the HBM read of the columns.  Each
// warp takes one column over a chunk of 8192 rows and sums the raw 128-bit
// products y * L in a three-word accumulator (one 64x64 multiply and three
// carry adds an element), reduced mod p once per lane (2^128 = -2^32), then
// summed across the warp; the extension-by-extension kind keeps y1 l1 apart
// and multiplies it by 7 once.  A second kernel sums a column's chunk
// partials with one warp.  Field addition is exact, so the order of the sums
// does not change the result.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/bc_barycentric.h"
#include "../../include/bc_ops.h"
#include "ext.cuh"
#include "ntt_host.cuh"
#include "ntt_pass.cuh"

namespace bc {
namespace {

constexpr uint32_t BT = 256;       // threads per block
constexpr uint32_t RUN_INV = 16;   // coefficients per thread (batch inversion width)
constexpr uint32_t MASK24 = (1u << 24) - 1;

// ---------------------------------------------------------------- common factor
template <bool EXT>
__global__ void common_factor_kernel(const uint64_t *x_ref, uint64_t *cf_ref, uint64_t coset, uint32_t log_count) {
  uint64_t coset_n = coset;
  for (uint32_t k = 0; k < log_count; k++) coset_n = gl::sqr(coset_n);
  const uint64_t den_inv = inv(gl::mul((uint64_t)1 << log_count, coset_n));
  if constexpr (EXT) {
    Ext xn{x_ref[0], x_ref[1]};
    for (uint32_t k = 0; k < log_count; k++) xn = ext_mul(xn, xn);
    const Ext num{gl::mul(gl::sub(xn.c0, coset_n), coset), gl::mul(xn.c1, coset)};
    const Ext cf = ext_mul_base(num, den_inv);
    cf_ref[0] = gl::canon(cf.c0);
    cf_ref[1] = gl::canon(cf.c1);
  } else {
    uint64_t xn = x_ref[0];
    for (uint32_t k = 0; k < log_count; k++) xn = gl::sqr(xn);
    cf_ref[0] = gl::canon(gl::mul(gl::mul(gl::sub(xn, coset_n), coset), den_inv));
  }
}

// ---------------------------------------------------------------- coefficients
// Thread t of a block takes i = i0 + 256 k, k < RUN_INV.
template <bool EXT>
__global__ void __launch_bounds__(BT) lagrange_kernel(const uint64_t *x_ref, const uint64_t *cf_ref, uint64_t coset,
                                                      uint64_t *coeffs, uint32_t log_count, const DevTables tabs) {
  const uint32_t count = 1u << log_count;
  const uint32_t i0 = blockIdx.x * (RUN_INV * BT) + threadIdx.x;
  if (i0 >= count) return;
  const uint32_t d = 24 - log_count;
  uint64_t w = w24_power(tabs, 1, (i0 << d) & MASK24);             // w^-i0
  const uint64_t step = w24_power(tabs, 1, (BT << d) & MASK24);    // w^-256
  const uint64_t x0 = x_ref[0], x1 = EXT ? x_ref[1] : 0;
  // denominators (extension: their norms) and the prefix products
  uint64_t den0[RUN_INV], den1[RUN_INV], norm[RUN_INV], pre[RUN_INV];
  uint64_t acc = 1;
  uint32_t n = 0;
#pragma unroll
  for (uint32_t k = 0; k < RUN_INV; k++) {
    if (i0 + k * BT < count) {
      den0[k] = gl::sub(gl::mul(x0, w), coset);
      if constexpr (EXT) {
        den1[k] = gl::mul(x1, w);
        norm[k] = ext_norm(Ext{den0[k], den1[k]});
      } else {
        norm[k] = den0[k];
      }
      pre[k] = acc;
      acc = gl::mul(acc, norm[k]);
      w = gl::mul(w, step);
      n = k + 1;
    }
  }
  uint64_t inv_acc = inv(acc);
  uint64_t cf0 = cf_ref[0], cf1 = EXT ? cf_ref[1] : 0;
#pragma unroll
  for (int k = RUN_INV - 1; k >= 0; k--) {
    if ((uint32_t)k < n) {
      const uint64_t ninv = gl::mul(inv_acc, pre[k]); // 1 / norm[k]
      inv_acc = gl::mul(inv_acc, norm[k]);
      const uint32_t i = i0 + (uint32_t)k * BT;
      if constexpr (EXT) {
        // 1 / (a0 + a1 x) = (a0 - a1 x) / norm
        const Ext dinv{gl::mul(den0[k], ninv), gl::sub(0, gl::mul(den1[k], ninv))};
        const Ext l = ext_mul(Ext{cf0, cf1}, dinv);
        coeffs[i] = gl::canon(l.c0);
        coeffs[(uint64_t)count + i] = gl::canon(l.c1);
      } else {
        coeffs[i] = gl::canon(gl::mul(cf0, ninv));
      }
    }
  }
}

template <bool EXT>
cudaError_t precompute(const uint64_t *x, uint64_t *cf, uint64_t coset, uint64_t *coeffs, uint32_t count,
                       bool bit_reverse, cudaStream_t stream) {
  if (!x || !cf || !coeffs || count == 0 || (count & (count - 1))) return cudaErrorInvalidValue;
  const uint32_t log_count = 31 - __builtin_clz(count);
  if (log_count > 24) return cudaErrorInvalidValue;
  const DevTables *t = device_tables();
  if (!t) return cudaErrorInitializationError;
  common_factor_kernel<EXT><<<1, 1, 0, stream>>>(x, cf, coset, log_count);
  const uint32_t per_block = RUN_INV * BT;
  lagrange_kernel<EXT><<<(count + per_block - 1) / per_block, BT, 0, stream>>>(x, cf, coset, coeffs, log_count, *t);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !bit_reverse) return e;
  return bc_bit_reverse_in_place(coeffs, count, log_count, EXT ? 2 : 1, stream);
}

// ---------------------------------------------------------------- evaluation
struct KindTraits {
  bool x_ext, y_ext;
};
__host__ __device__ constexpr KindTraits kind_traits(int kind) {
  return {kind != BC_EVAL_BASE_AT_BASE, kind == BC_EVAL_EXT_AT_EXT};
}

constexpr uint32_t EVAL_WARPS = 8;          // columns per block, one per warp
constexpr uint32_t EVAL_ROWS = 8192;        // rows per block (256 per lane)
constexpr uint32_t EVAL_UNROLL = 8;

// Sum of 128-bit products, kept unreduced in three words: up to 2^24 products
// of u64 words stay below 2^152.  Reduced once at the end with
// 2^64 = 2^32 - 1 and 2^128 = -2^32 (mod p).
struct Acc192 {
  uint64_t w0 = 0, w1 = 0, w2 = 0;
  __device__ __forceinline__ void mac(uint64_t a, uint64_t b) {
    const uint64_t lo = a * b, hi = __umul64hi(a, b);
    asm("add.cc.u64 %0, %0, %3;\n\t"
        "addc.cc.u64 %1, %1, %4;\n\t"
        "addc.u64 %2, %2, 0;"
        : "+l"(w0), "+l"(w1), "+l"(w2)
        : "l"(lo), "l"(hi));
  }
  __device__ __forceinline__ uint64_t reduce() const { return gl::sub(gl::reduce128(w0, w1), w2 << 32); }
};

__device__ __forceinline__ uint64_t warp_sum(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = gl::add(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block (row chunk blockIdx.x, column group blockIdx.y); warp w sums column
// blockIdx.y * 8 + w over the chunk's rows (lane: rows lane + 32 k) into
// partial[(p * chunks + chunk) * xw + c].  Coefficients are read per element:
// the 8 warps of a block read the same ones, from L1.
template <int KIND>
__global__ void __launch_bounds__(EVAL_WARPS * 32) eval_partial_kernel(const uint64_t *ys, uint32_t count,
                                                                       uint32_t num_polys, const uint64_t *coeffs,
                                                                       uint64_t *partial, uint32_t chunks) {
  constexpr KindTraits K = kind_traits(KIND);
  constexpr uint32_t xw = K.x_ext ? 2 : 1;
  const uint32_t lane = threadIdx.x & 31, p = blockIdx.y * EVAL_WARPS + (threadIdx.x >> 5);
  if (p >= num_polys) return;
  const uint64_t row0 = (uint64_t)blockIdx.x * EVAL_ROWS;
  const uint64_t rows = min((uint64_t)EVAL_ROWS, count - row0);
  const uint64_t *y0 = ys + (uint64_t)p * count * (K.y_ext ? 2 : 1) + row0;
  const uint64_t *y1 = y0 + count;
  const uint64_t *l0 = coeffs + row0, *l1 = coeffs + count + row0;
  Acc192 a0, a1, a7; // a7: y1 l1 of the extension values (times 7 at the end)
  for (uint64_t r = lane; r < rows; r += 32 * EVAL_UNROLL) {
    uint64_t v0[EVAL_UNROLL], v1[EVAL_UNROLL], c0[EVAL_UNROLL], c1[EVAL_UNROLL];
#pragma unroll
    for (uint32_t k = 0; k < EVAL_UNROLL; k++) {
      const uint64_t i = r + 32 * k;
      const bool in = i < rows;
      v0[k] = in ? __ldcs(y0 + i) : 0;
      c0[k] = in ? __ldg(l0 + i) : 0;
      if constexpr (K.x_ext) c1[k] = in ? __ldg(l1 + i) : 0;
      if constexpr (K.y_ext) v1[k] = in ? __ldcs(y1 + i) : 0;
    }
#pragma unroll
    for (uint32_t k = 0; k < EVAL_UNROLL; k++) {
      a0.mac(v0[k], c0[k]);
      if constexpr (KIND == BC_EVAL_BASE_AT_EXT) a1.mac(v0[k], c1[k]);
      if constexpr (KIND == BC_EVAL_EXT_AT_EXT) {
        a7.mac(v1[k], c1[k]);
        a1.mac(v0[k], c1[k]);
        a1.mac(v1[k], c0[k]);
      }
    }
  }
  uint64_t s0 = a0.reduce(), s1 = 0;
  if constexpr (KIND == BC_EVAL_BASE_AT_EXT) s1 = a1.reduce();
  if constexpr (KIND == BC_EVAL_EXT_AT_EXT) {
    s0 = gl::add(s0, mul7(a7.reduce()));
    s1 = a1.reduce();
  }
  s0 = warp_sum(s0);
  if constexpr (K.x_ext) s1 = warp_sum(s1);
  if (lane == 0) {
    uint64_t *dst = partial + ((uint64_t)p * chunks + blockIdx.x) * xw;
    dst[0] = s0;
    if constexpr (K.x_ext) dst[1] = s1;
  }
}

// One warp per column: evals[p * xw + c] = sum over chunks.
template <int KIND>
__global__ void eval_final_kernel(const uint64_t *partial, uint32_t chunks, uint32_t num_polys, uint64_t *evals) {
  constexpr uint32_t xw = kind_traits(KIND).x_ext ? 2 : 1;
  const uint32_t p = blockIdx.x, lane = threadIdx.x;
  if (p >= num_polys) return;
  uint64_t s[xw] = {};
  for (uint32_t c = lane; c < chunks; c += 32)
#pragma unroll
    for (uint32_t w = 0; w < xw; w++) s[w] = gl::add(s[w], partial[((uint64_t)p * chunks + c) * xw + w]);
#pragma unroll
  for (uint32_t w = 0; w < xw; w++) {
    const uint64_t v = warp_sum(s[w]);
    if (lane == 0) evals[(uint64_t)p * xw + w] = gl::canon(v);
  }
}

uint32_t eval_chunks(uint32_t count) { return (count + EVAL_ROWS - 1) / EVAL_ROWS; }

template <int KIND>
void launch_eval(const uint64_t *ys, uint32_t count, uint32_t num_polys, const uint64_t *coeffs, uint64_t *partial,
                 uint64_t *evals, cudaStream_t stream) {
  const uint32_t chunks = eval_chunks(count);
  const dim3 grid(chunks, (num_polys + EVAL_WARPS - 1) / EVAL_WARPS);
  eval_partial_kernel<KIND><<<grid, EVAL_WARPS * 32, 0, stream>>>(ys, count, num_polys, coeffs, partial, chunks);
  eval_final_kernel<KIND><<<num_polys, 32, 0, stream>>>(partial, chunks, num_polys, evals);
}

} // namespace
} // namespace bc

using namespace bc;

// ---------------------------------------------------------------- C ABI
extern "C" cudaError_t bc_precompute_lagrange_coeffs_at_base(const uint64_t *x, uint64_t *common_factor_storage,
                                                             uint64_t coset, uint64_t *lagrange_coeffs, uint32_t count,
                                                             bool bit_reverse, cudaStream_t stream) {
  return precompute<false>(x, common_factor_storage, coset, lagrange_coeffs, count, bit_reverse, stream);
}

extern "C" cudaError_t bc_precompute_lagrange_coeffs_at_ext(const uint64_t *x, uint64_t *common_factor_storage,
                                                            uint64_t coset, uint64_t *lagrange_coeffs, uint32_t count,
                                                            bool bit_reverse, cudaStream_t stream) {
  return precompute<true>(x, common_factor_storage, coset, lagrange_coeffs, count, bit_reverse, stream);
}

extern "C" cudaError_t bc_get_batch_eval_temp_storage_sizes(int kind, uint32_t count, uint32_t num_polys,
                                                            size_t *partial_reduce_temp_words,
                                                            size_t *final_reduce_temp_bytes) {
  if (kind < BC_EVAL_BASE_AT_BASE || kind > BC_EVAL_EXT_AT_EXT || count == 0 || (count & (count - 1)))
    return cudaErrorInvalidValue;
  if (!partial_reduce_temp_words || !final_reduce_temp_bytes) return cudaErrorInvalidValue;
  *partial_reduce_temp_words = (size_t)eval_chunks(count) * num_polys * (kind_traits(kind).x_ext ? 2 : 1);
  *final_reduce_temp_bytes = 0;
  return cudaSuccess;
}

extern "C" cudaError_t bc_batch_eval(int kind, const uint64_t *batch_ys, uint32_t count, uint32_t num_polys,
                                     const uint64_t *lagrange_coeffs, uint64_t *temp_partial_reduce,
                                     size_t temp_partial_reduce_words, void *temp_final_reduce,
                                     size_t temp_final_reduce_bytes, uint64_t *evals, cudaStream_t stream) {
  (void)temp_final_reduce;
  (void)temp_final_reduce_bytes;
  size_t need_words = 0, need_bytes = 0;
  const cudaError_t e = bc_get_batch_eval_temp_storage_sizes(kind, count, num_polys, &need_words, &need_bytes);
  if (e != cudaSuccess) return e;
  if (num_polys == 0) return cudaSuccess;
  if (!batch_ys || !lagrange_coeffs || !evals || !temp_partial_reduce || temp_partial_reduce_words < need_words)
    return cudaErrorInvalidValue;
  switch (kind) {
  case BC_EVAL_BASE_AT_BASE:
    launch_eval<BC_EVAL_BASE_AT_BASE>(batch_ys, count, num_polys, lagrange_coeffs, temp_partial_reduce, evals, stream);
    break;
  case BC_EVAL_BASE_AT_EXT:
    launch_eval<BC_EVAL_BASE_AT_EXT>(batch_ys, count, num_polys, lagrange_coeffs, temp_partial_reduce, evals, stream);
    break;
  default:
    launch_eval<BC_EVAL_EXT_AT_EXT>(batch_ys, count, num_polys, lagrange_coeffs, temp_partial_reduce, evals, stream);
    break;
  }
  return cudaGetLastError();
}
