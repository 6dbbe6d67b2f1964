// ops.cu -- the operations beside the NTT in the reference's
// src/ops_complex.rs: bit-reversal permutation of matrix columns, table-driven
// powers, powers of an arbitrary base (base field and the quadratic
// extension) and the omega shift.  C ABI in include/bc_ops.h.
//
// Bit reversal.  A column of 2^L rows is indexed i = (a, m, b): a the top
// h = L/2 bits, m the middle bit when L is odd, b the bottom h bits, and
// brev_L(i) = (brev_h(b), m, brev_h(a)).  So the permutation is a transpose
// of the 2^h x 2^h matrix a x b (for each m) with both coordinates
// bit-reversed.  A tile (U, V) holds the 32 rows a with brev_h(a) in
// [32U, 32U + 32) and the 32 columns b in [32V, 32V + 32): it reads 32
// contiguous 256-byte row segments and writes them transposed to rows
// brev_h(b) and the contiguous columns [32U, 32U + 32), i.e. onto the source
// region of tile (V, U).  A CTA loads the pair (U, V), (V, U) into shared
// memory before it writes either, which makes the same kernel an in-place
// permutation; the reference does the same with 32 x 32 tiles
// (native/ops_complex.cu:106-157).  Columns of fewer than 1024 rows swap pairs
// (i, brev(i)) directly.  HBM-bound: 16 bytes per element.
//
// Powers.  Exponents follow native/context.cuh:33-48: omega = w_{2^24}, an
// index mod 2^24, the inverse as w^-e; g = 7 (7^-1 when inverse).  They are
// read from this library's two-level tables (tables.cuh): w_{2^24}^e =
// w_{2^30}^(64 e).  Every kernel but the bit reversal walks a running product
// per thread over indexes 256 apart, exact because the reference's index
// arithmetic is a ring map mod 2^32 (and so mod 2^24): w has order 2^24, and
// the powers of 7 or of a base restart from scratch where their exponent
// wraps (mod 2^24, resp. the u32 exponent).
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/bc_ops.h"
#include "ext.cuh"
#include "ntt_host.cuh"
#include "ntt_pass.cuh"

namespace bc {
namespace {

constexpr uint32_t OPS_THREADS = 256;
constexpr uint32_t RUN = 16;           // elements per thread in the running-product kernels
constexpr uint32_t RUN_POW = 64;       // the same for the powers of a base (amortises its exponentiation)
constexpr uint32_t MASK24 = (1u << 24) - 1;

__device__ __forceinline__ uint32_t brev_n(uint32_t x, uint32_t bits) { return bits ? __brev(x) >> (32 - bits) : 0u; }

// ---------------------------------------------------------------- bit reversal
__global__ void __launch_bounds__(OPS_THREADS) bitrev_swap_kernel(const uint64_t *src, uint64_t ss, uint64_t *dst,
                                                                  uint64_t ds, uint32_t log_rows, uint32_t cols) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (1u << log_rows)) return;
  const uint32_t r = brev_n(i, log_rows);
  if (i > r) return;
  for (uint32_t col = blockIdx.y; col < cols; col += gridDim.y) {
    const uint64_t *s = src + (uint64_t)col * ss;
    uint64_t *d = dst + (uint64_t)col * ds;
    const uint64_t vi = s[i], vr = s[r];
    d[i] = vr;
    d[r] = vi;
  }
}

// Tile pair k of the triangle U <= V (k = V (V + 1) / 2 + U).
__device__ __forceinline__ void decode_tile_pair(uint64_t k, uint32_t &U, uint32_t &V) {
  uint64_t v = (uint64_t)((sqrtf(8.f * (float)k + 1.f) - 1.f) * 0.5f);
  while ((v + 1) * (v + 2) / 2 <= k) v++;
  while (v * (v + 1) / 2 > k) v--;
  U = (uint32_t)(k - v * (v + 1) / 2);
  V = (uint32_t)v;
}

// One CTA: tile pair blockIdx.x (triangular over U <= V), middle bit
// blockIdx.z, columns blockIdx.y + k gridDim.y.  VEC: 16-byte accesses -- a
// warp moves two 32-element row segments per instruction (half-warps on
// consecutive tile rows) and writes each destination row as pairs of
// transposed elements; needs 16-byte aligned columns.  Measured on B200 (64
// columns x 2^22, out of place): 0.644 ms against 0.685 ms with 8-byte
// accesses and 0.667 ms for the reference's kernel.
template <bool VEC>
__global__ void __launch_bounds__(OPS_THREADS) bitrev_tile_kernel(const uint64_t *src, uint64_t ss, uint64_t *dst,
                                                                  uint64_t ds, uint32_t log_rows, uint32_t cols) {
  __shared__ uint64_t tile[2][32][33];
  const uint32_t h = log_rows >> 1, mbit = log_rows & 1;
  uint32_t U, Vv;
  decode_tile_pair(blockIdx.x, U, Vv);
  const uint32_t ntiles = U == Vv ? 1 : 2;
  const uint64_t mid = (uint64_t)blockIdx.z << h;
  // 8-byte: lane = tile column, rows row0 + 8 j.  16-byte: lanes 0-15 / 16-31 of warp w on tile rows
  // 2 (w + 8 j) and 2 (w + 8 j) + 1, two columns 2 l16, 2 l16 + 1 each.
  const uint32_t lane = threadIdx.x & 31, row0 = threadIdx.x >> 5;
  const uint32_t half = (threadIdx.x >> 4) & 1, l16 = threadIdx.x & 15;
  for (uint32_t col = blockIdx.y; col < cols; col += gridDim.y) {
    const uint64_t *s = src + (uint64_t)col * ss + mid;
    uint64_t *d = dst + (uint64_t)col * ds + mid;
    if constexpr (VEC) {
      ulonglong2 v[2][2];
#pragma unroll
      for (uint32_t q = 0; q < 2; q++) {
        if (q < ntiles) {
          const uint32_t tu = q ? Vv : U, tv = q ? U : Vv;
#pragma unroll
          for (uint32_t j = 0; j < 2; j++) {
            const uint64_t a = brev_n(32 * tu + 2 * (row0 + 8 * j) + half, h);
            v[q][j] = __ldcs(reinterpret_cast<const ulonglong2 *>(s + (a << (h + mbit)) + 32 * tv) + l16);
          }
        }
      }
#pragma unroll
      for (uint32_t q = 0; q < 2; q++)
        if (q < ntiles)
#pragma unroll
          for (uint32_t j = 0; j < 2; j++) {
            const uint32_t t = 2 * (row0 + 8 * j) + half;
            tile[q][t][2 * l16] = v[q][j].x;
            tile[q][t][2 * l16 + 1] = v[q][j].y;
          }
      __syncthreads();
#pragma unroll
      for (uint32_t q = 0; q < 2; q++) {
        if (q < ntiles) {
          const uint32_t tu = q ? Vv : U, tv = q ? U : Vv;
#pragma unroll
          for (uint32_t j = 0; j < 2; j++) {
            const uint32_t sidx = 2 * (row0 + 8 * j) + half; // column of the source tile = destination row
            const uint64_t r = brev_n(32 * tv + sidx, h);
            __stcs(reinterpret_cast<ulonglong2 *>(d + (r << (h + mbit)) + 32 * tu) + l16,
                   make_ulonglong2(tile[q][2 * l16][sidx], tile[q][2 * l16 + 1][sidx]));
          }
        }
      }
    } else {
      uint64_t v[2][4];
#pragma unroll
      for (uint32_t q = 0; q < 2; q++) {
        if (q < ntiles) {
          const uint32_t tu = q ? Vv : U, tv = q ? U : Vv;
#pragma unroll
          for (uint32_t j = 0; j < 4; j++) {
            const uint64_t a = brev_n(32 * tu + row0 + 8 * j, h);
            v[q][j] = __ldcs(s + (a << (h + mbit)) + 32 * tv + lane);
          }
        }
      }
#pragma unroll
      for (uint32_t q = 0; q < 2; q++)
        if (q < ntiles)
#pragma unroll
          for (uint32_t j = 0; j < 4; j++) tile[q][row0 + 8 * j][lane] = v[q][j];
      __syncthreads();
#pragma unroll
      for (uint32_t q = 0; q < 2; q++) {
        if (q < ntiles) {
          const uint32_t tu = q ? Vv : U, tv = q ? U : Vv;
#pragma unroll
          for (uint32_t j = 0; j < 4; j++) {
            const uint32_t sidx = row0 + 8 * j; // column of the source tile = destination row
            const uint64_t r = brev_n(32 * tv + sidx, h);
            __stcs(d + (r << (h + mbit)) + 32 * tu + lane, tile[q][lane][sidx]);
          }
        }
      }
    }
    __syncthreads();
  }
}

cudaError_t bit_reverse(const uint64_t *src, uint64_t ss, uint64_t *dst, uint64_t ds, uint32_t log_rows,
                        uint32_t cols, cudaStream_t stream) {
  if (log_rows > 31) return cudaErrorInvalidValue;
  if (cols == 0) return cudaSuccess;
  if (!src || !dst) return cudaErrorInvalidValue;
  const uint64_t rows = 1ull << log_rows;
  if (cols > 1 && (ss < rows || ds < rows)) return cudaErrorInvalidValue;
  if (src == dst && ss != ds) return cudaErrorInvalidValue;
  const uint32_t gy = cols < 65535u ? cols : 65535u;
  if (log_rows < 10) {
    const uint32_t blocks = (uint32_t)((rows + OPS_THREADS - 1) / OPS_THREADS);
    bitrev_swap_kernel<<<dim3(blocks, gy), OPS_THREADS, 0, stream>>>(src, ss, dst, ds, log_rows, cols);
  } else {
    const uint64_t m = 1ull << ((log_rows >> 1) - 5);
    const uint64_t pairs = m * (m + 1) / 2;
    const dim3 grid((uint32_t)pairs, gy, 1u << (log_rows & 1));
    const bool vec = (uintptr_t)src % 16 == 0 && (uintptr_t)dst % 16 == 0 && (cols == 1 || (ss % 2 == 0 && ds % 2 == 0));
    if (vec)
      bitrev_tile_kernel<true><<<grid, OPS_THREADS, 0, stream>>>(src, ss, dst, ds, log_rows, cols);
    else
      bitrev_tile_kernel<false><<<grid, OPS_THREADS, 0, stream>>>(src, ss, dst, ds, log_rows, cols);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------- powers from the tables
__device__ __forceinline__ uint64_t domain_power(const DevTables &t, uint32_t of_g, uint32_t inv, uint32_t e) {
  return of_g ? g_power(t, inv, e) : w24_power(t, inv, e);
}

// Thread t of a block takes indexes i0 + 256 k, k < RUN.  Natural order: the
// exponent advances by de = (256 << (24 - log_degree)) mod 2^24 per step, a
// running product that restarts from the tables where the exponent wraps past
// 2^24 (7 is not of order 2^24).  Bit-reversed order: one table read each.
__global__ void __launch_bounds__(OPS_THREADS) powers_of_kernel(uint32_t log_degree, uint32_t offset, uint32_t inverse,
                                                                uint32_t bit_reverse, uint64_t *result, uint32_t count,
                                                                uint32_t of_g, const DevTables tabs) {
  const uint64_t i0 = (uint64_t)blockIdx.x * (RUN * OPS_THREADS) + threadIdx.x;
  if (i0 >= count) return;
  const uint32_t d = 24 - log_degree;
  if (bit_reverse) {
    for (uint32_t k = 0; k < RUN; k++) {
      const uint64_t i = i0 + (uint64_t)k * OPS_THREADS;
      if (i >= count) break;
      const uint32_t e = (brev_n((uint32_t)i + offset, log_degree) << d) & MASK24;
      __stcs(result + i, gl::canon(domain_power(tabs, of_g, inverse, e)));
    }
    return;
  }
  const uint32_t de = (OPS_THREADS << d) & MASK24;
  const uint64_t step = domain_power(tabs, of_g, inverse, de);
  uint32_t e = (((uint32_t)i0 + offset) << d) & MASK24;
  uint64_t v = domain_power(tabs, of_g, inverse, e);
  for (uint32_t k = 0; k < RUN; k++) {
    const uint64_t i = i0 + (uint64_t)k * OPS_THREADS;
    if (i >= count) break;
    __stcs(result + i, gl::canon(v));
    const uint32_t next = (e + de) & MASK24;
    v = next < e ? domain_power(tabs, of_g, inverse, next) : gl::mul(v, step);
    e = next;
  }
}

cudaError_t powers_of(uint32_t log_degree, uint32_t offset, bool inverse, bool bit_reverse, uint64_t *result,
                      uint32_t count, bool of_g, cudaStream_t stream) {
  if (log_degree > 24) return cudaErrorInvalidValue;
  if (count == 0) return cudaSuccess;
  if (!result) return cudaErrorInvalidValue;
  const DevTables *t = device_tables();
  if (!t) return cudaErrorInitializationError;
  const uint64_t per_block = RUN * OPS_THREADS;
  const uint32_t blocks = (uint32_t)(((uint64_t)count + per_block - 1) / per_block);
  powers_of_kernel<<<blocks, OPS_THREADS, 0, stream>>>(log_degree, offset, inverse, bit_reverse, result, count, of_g,
                                                       *t);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- powers of a base
template <typename F> struct Arith;
template <> struct Arith<uint64_t> {
  static __device__ __forceinline__ uint64_t one() { return 1; }
  static __device__ __forceinline__ uint64_t mul(uint64_t a, uint64_t b) { return gl::mul(a, b); }
  static __device__ __forceinline__ void store(uint64_t *r, uint32_t i, uint32_t, uint64_t v) {
    __stcs(r + i, gl::canon(v));
  }
};
template <> struct Arith<Ext> {
  static __device__ __forceinline__ Ext one() { return {1, 0}; }
  static __device__ __forceinline__ Ext mul(const Ext &a, const Ext &b) { return ext_mul(a, b); }
  static __device__ __forceinline__ void store(uint64_t *r, uint32_t i, uint32_t count, const Ext &v) {
    __stcs(r + i, gl::canon(v.c0));
    __stcs(r + (uint64_t)count + i, gl::canon(v.c1));
  }
};

template <typename F> __device__ __forceinline__ F fpow(F b, uint32_t e) {
  F r = Arith<F>::one();
  while (e) {
    if (e & 1) r = Arith<F>::mul(r, b);
    e >>= 1;
    if (e) b = Arith<F>::mul(b, b);
  }
  return r;
}

// A block covers RUN_POW * 256 consecutive indexes; thread t takes t, t + 256, ...
template <typename F>
__global__ void __launch_bounds__(OPS_THREADS) powers_by_kernel(F base, const uint64_t *base_ref, uint32_t offset,
                                                                uint32_t bit_reverse, uint64_t *result,
                                                                uint32_t count) {
  if (base_ref) {
    if constexpr (sizeof(F) == 8)
      base = (F)base_ref[0];
    else
      base = F{base_ref[0], base_ref[1]};
  }
  const uint64_t i0 = (uint64_t)blockIdx.x * (RUN_POW * OPS_THREADS) + threadIdx.x;
  if (bit_reverse) {
    for (uint32_t k = 0; k < RUN_POW; k++) {
      const uint64_t i = i0 + (uint64_t)k * OPS_THREADS;
      if (i < count) Arith<F>::store(result, (uint32_t)i, count, fpow(base, __brev((uint32_t)i) + offset));
    }
    return;
  }
  if (i0 >= count) return;
  const F step = fpow(base, OPS_THREADS);
  uint32_t e = (uint32_t)i0 + offset;
  F v = fpow(base, e);
  for (uint32_t k = 0; k < RUN_POW; k++) {
    const uint64_t i = i0 + (uint64_t)k * OPS_THREADS;
    if (i >= count) break;
    Arith<F>::store(result, (uint32_t)i, count, v);
    const uint32_t next = e + OPS_THREADS;
    v = next < e ? fpow(base, next) : Arith<F>::mul(v, step); // the u32 exponent wrapped: restart
    e = next;
  }
}

template <typename F>
cudaError_t powers_by(const F &base, const uint64_t *base_ref, uint32_t offset, bool bit_reverse, uint64_t *result,
                      uint32_t count, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  if (!result) return cudaErrorInvalidValue;
  const uint64_t per_block = RUN_POW * OPS_THREADS;
  const uint32_t blocks = (uint32_t)(((uint64_t)count + per_block - 1) / per_block);
  powers_by_kernel<F><<<blocks, OPS_THREADS, 0, stream>>>(base, base_ref, offset, bit_reverse, result, count);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- omega shift
__global__ void __launch_bounds__(OPS_THREADS) omega_shift_kernel(const uint64_t *src, uint32_t log_degree,
                                                                  uint32_t offset, uint32_t inverse, uint32_t shift,
                                                                  uint64_t *dst, uint32_t count, const DevTables tabs) {
  const uint64_t i0 = (uint64_t)blockIdx.x * (RUN * OPS_THREADS) + threadIdx.x;
  if (i0 >= count) return;
  const uint32_t d = 24 - log_degree;
  const uint32_t e0 = ((shift * ((uint32_t)i0 + offset)) << d) & MASK24;
  const uint32_t de = ((shift * OPS_THREADS) << d) & MASK24;
  const uint64_t step = w24_power(tabs, inverse, de);
  uint64_t v = w24_power(tabs, inverse, e0);
  uint64_t x[RUN];
#pragma unroll
  for (uint32_t k = 0; k < RUN; k++) {
    const uint64_t i = i0 + (uint64_t)k * OPS_THREADS;
    x[k] = i < count ? __ldcs(src + i) : 0;
  }
#pragma unroll
  for (uint32_t k = 0; k < RUN; k++) {
    const uint64_t i = i0 + (uint64_t)k * OPS_THREADS;
    if (i < count) __stcs(dst + i, gl::canon(gl::mul(x[k], v)));
    v = gl::mul(v, step);
  }
}

cudaError_t omega_shift(const uint64_t *src, uint32_t log_degree, uint32_t offset, bool inverse, uint32_t shift,
                        uint64_t *dst, uint32_t count, cudaStream_t stream) {
  if (log_degree > 24) return cudaErrorInvalidValue;
  if (count == 0) return cudaSuccess;
  if (!src || !dst) return cudaErrorInvalidValue;
  const DevTables *t = device_tables();
  if (!t) return cudaErrorInitializationError;
  const uint64_t per_block = RUN * OPS_THREADS;
  const uint32_t blocks = (uint32_t)(((uint64_t)count + per_block - 1) / per_block);
  omega_shift_kernel<<<blocks, OPS_THREADS, 0, stream>>>(src, log_degree, offset, inverse, shift, dst, count, *t);
  return cudaGetLastError();
}

} // namespace
} // namespace bc

using namespace bc;

// ---------------------------------------------------------------- C ABI
extern "C" cudaError_t bc_bit_reverse(const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride,
                                      uint32_t log_rows, uint32_t cols, cudaStream_t stream) {
  return bit_reverse(src, src_stride, dst, dst_stride, log_rows, cols, stream);
}

extern "C" cudaError_t bc_bit_reverse_in_place(uint64_t *values, uint64_t stride, uint32_t log_rows, uint32_t cols,
                                               cudaStream_t stream) {
  return bit_reverse(values, stride, values, stride, log_rows, cols, stream);
}

extern "C" cudaError_t bc_get_powers_of_w(uint32_t log_degree, uint32_t offset, bool inverse, bool bit_reverse,
                                          uint64_t *result, uint32_t count, cudaStream_t stream) {
  return powers_of(log_degree, offset, inverse, bit_reverse, result, count, false, stream);
}

extern "C" cudaError_t bc_get_powers_of_g(uint32_t log_degree, uint32_t offset, bool inverse, bool bit_reverse,
                                          uint64_t *result, uint32_t count, cudaStream_t stream) {
  return powers_of(log_degree, offset, inverse, bit_reverse, result, count, true, stream);
}

extern "C" cudaError_t bc_get_powers_by_val_bf(uint64_t base, uint32_t offset, bool bit_reverse, uint64_t *result,
                                               uint32_t count, cudaStream_t stream) {
  return powers_by<uint64_t>(base, nullptr, offset, bit_reverse, result, count, stream);
}

extern "C" cudaError_t bc_get_powers_by_ref_bf(const uint64_t *base, uint32_t offset, bool bit_reverse,
                                               uint64_t *result, uint32_t count, cudaStream_t stream) {
  if (!base) return cudaErrorInvalidValue;
  return powers_by<uint64_t>(0, base, offset, bit_reverse, result, count, stream);
}

extern "C" cudaError_t bc_get_powers_by_val_ef(uint64_t base_c0, uint64_t base_c1, uint32_t offset, bool bit_reverse,
                                               uint64_t *result, uint32_t count, cudaStream_t stream) {
  return powers_by<Ext>(Ext{base_c0, base_c1}, nullptr, offset, bit_reverse, result, count, stream);
}

extern "C" cudaError_t bc_get_powers_by_ref_ef(const uint64_t *base, uint32_t offset, bool bit_reverse,
                                               uint64_t *result, uint32_t count, cudaStream_t stream) {
  if (!base) return cudaErrorInvalidValue;
  return powers_by<Ext>(Ext{0, 0}, base, offset, bit_reverse, result, count, stream);
}

extern "C" cudaError_t bc_omega_shift(const uint64_t *src, uint32_t log_degree, uint32_t offset, bool inverse,
                                      uint32_t shift, uint64_t *dst, uint32_t count, cudaStream_t stream) {
  return omega_shift(src, log_degree, offset, inverse, shift, dst, count, stream);
}

extern "C" cudaError_t bc_omega_shift_in_place(uint64_t *values, uint32_t log_degree, uint32_t offset, bool inverse,
                                               uint32_t shift, uint32_t count, cudaStream_t stream) {
  return omega_shift(values, log_degree, offset, inverse, shift, values, count, stream);
}
