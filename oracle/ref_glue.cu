// ref_glue.cu -- host glue that runs the REFERENCE's own NTT and ops kernels.
//
// TEST / BASELINE INFRASTRUCTURE ONLY (never linked into the product).
// oracle/Makefile (target `ref`) compiles this file together with the
// reference's native/ntt.cu, native/context.cu and native/ops_complex.cu, as
// separate translation units read from where they lie in the reference
// checkout (nothing is copied), with relocatable device code, into
// oracle/_ref/libref_ntt.so.
//
// The reference's host side is Rust (src/context.rs, src/ntt.rs), which cannot
// be built in this image (no Rust toolchain, boojum 0.2.2 not vendored), so
// this file restates, in C++, exactly what that Rust does around the kernels:
//   * ref_context_create   <- Context::create        src/context.rs:171-282
//                             copy_to_symbols        src/context.rs:74-142
//   * ref_batch_ntt        <- batch_ntt_internal     src/ntt.rs:179-290
//                             (PLANS table           src/ntt.rs:74-169,
//                              launch geometry       src/ntt.rs:257-270,
//                              per-stage path        src/ntt.rs:203-241)
//   * ref_bit_reverse, ref_get_powers_of, ref_get_powers_by_val,
//     ref_omega_shift      <- the wrappers of        src/ops_complex.rs:25-304
//   * ref_barycentric_precompute, ref_batch_eval
//                          <- precompute_lagrange_coeffs, batch_eval
//                                                    src/barycentric.rs:83-260
// Roots of unity: boojum's domain_generator_for_size is replaced by the
// generator-7 roots w_{2^k} = (7^((p-1)/2^32))^(2^(32-k)), the same choice the
// C oracle (gl_oracle.c) and the product library make.

#include "context.cuh"

// The reference kernels (native/ntt_n2b.cuh, native/ntt_b2n.cuh), compiled in
// their own translation unit; extern "C" linkage, signature of
// native/ntt_n2b.cuh:104-108.
#define REF_NTT_KERNEL(name)                                                                                           \
  extern "C" __global__ void name(const base_field *, base_field *, const unsigned, const unsigned, const unsigned,   \
                                  const unsigned, const unsigned, const bool, const unsigned, const unsigned,         \
                                  const unsigned);
REF_NTT_KERNEL(n2b_1_stage)
REF_NTT_KERNEL(b2n_1_stage)
REF_NTT_KERNEL(n2b_final_7_stages_warp)
REF_NTT_KERNEL(n2b_final_8_stages_warp)
REF_NTT_KERNEL(n2b_final_9_to_12_stages_block)
REF_NTT_KERNEL(n2b_nonfinal_7_or_8_stages_block)
REF_NTT_KERNEL(b2n_initial_7_stages_warp)
REF_NTT_KERNEL(b2n_initial_8_stages_warp)
REF_NTT_KERNEL(b2n_initial_9_to_12_stages_block)
REF_NTT_KERNEL(b2n_noninitial_7_or_8_stages_block)
#undef REF_NTT_KERNEL

// The reference's ops kernels (native/ops_complex.cu), declared with plain
// structs of the same layout as its by-value parameters: matrix_getter /
// matrix_setter = {T *ptr; size_t stride;} and vector_setter = {T *ptr;}
// (native/memory.cuh:321-422), extension_field = 16-byte aligned pair
// (native/goldilocks_extension.cuh:8-9).
struct RefMat {
  const void *ptr;
  size_t stride;
};
struct RefVec {
  void *ptr;
};
struct __align__(16) RefExt {
  uint64_t c0, c1;
};
extern "C" __global__ void bit_reverse_naive_kernel(RefMat, RefMat, const unsigned);
extern "C" __global__ void bit_reverse_kernel(RefMat, RefMat, const unsigned);
extern "C" __global__ void get_powers_of_w_kernel(const unsigned, const unsigned, const bool, const bool, RefVec,
                                                  const unsigned);
extern "C" __global__ void get_powers_of_g_kernel(const unsigned, const unsigned, const bool, const bool, RefVec,
                                                  const unsigned);
extern "C" __global__ void get_powers_by_val_bf_kernel(const uint64_t, const unsigned, const bool, uint64_t *,
                                                       const unsigned);
extern "C" __global__ void get_powers_by_val_ef_kernel(const RefExt, const unsigned, const bool, RefExt *,
                                                       const unsigned);
extern "C" __global__ void omega_shift_kernel(const uint64_t *, const unsigned, const unsigned, const bool,
                                              const unsigned, uint64_t *, const unsigned);
// native/barycentric.cu; ef_double_vector/matrix accessors wrap one matrix
// accessor {ptr, stride} (native/memory.cuh:436-590), i.e. RefMat.
extern "C" __global__ void barycentric_precompute_common_factor_bf_kernel(const uint64_t *, uint64_t *, const uint64_t,
                                                                          const unsigned);
extern "C" __global__ void barycentric_precompute_common_factor_ef_kernel(const RefExt *, RefExt *, const uint64_t,
                                                                          const unsigned);
extern "C" __global__ void barycentric_precompute_lagrange_coeffs_bf_kernel(const uint64_t *, const uint64_t *,
                                                                            const uint64_t, const uint64_t, RefVec,
                                                                            const unsigned);
extern "C" __global__ void barycentric_precompute_lagrange_coeffs_ef_kernel(const RefExt *, const RefExt *,
                                                                            const uint64_t, const uint64_t, RefMat,
                                                                            const unsigned);
extern "C" __global__ void batch_barycentric_partial_reduce_bf_bf_kernel(RefMat, RefVec, RefMat, const unsigned,
                                                                         const unsigned);
extern "C" __global__ void batch_barycentric_partial_reduce_bf_ef_kernel(RefMat, RefMat, RefMat, const unsigned,
                                                                         const unsigned);
extern "C" __global__ void batch_barycentric_partial_reduce_ef_ef_kernel(RefMat, RefMat, RefMat, const unsigned,
                                                                         const unsigned);

#include <cstdint>
#include <cstring>
#include <vector>

namespace refglue {

static constexpr uint64_t P = 0xffffffff00000001ull;
typedef unsigned __int128 u128;

static uint64_t mul(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a * b) % P); }
static uint64_t pw(uint64_t b, uint64_t e) {
  uint64_t r = 1;
  b %= P;
  while (e) {
    if (e & 1) r = mul(r, b);
    b = mul(b, b);
    e >>= 1;
  }
  return r;
}
static uint64_t inv(uint64_t a) { return pw(a, P - 2); }
// domain_generator_for_size(2^k) restated with the generator-7 root choice.
static uint64_t domain_generator(uint64_t size) {
  unsigned k = 0;
  while ((1ull << k) < size) k++;
  return pw(pw(7, (P - 1) >> 32), 1ull << (32 - k));
}
static unsigned brev(unsigned x, unsigned bits) {
  unsigned r = 0;
  for (unsigned i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}
// generate_powers_dev (src/context.rs:144-155): distribute_powers from ONE,
// then the optional bitreverse_enumeration_inplace over log2(len) bits.
static cudaError_t upload_powers(uint64_t base, size_t len, bool bit_reverse, base_field **dst) {
  std::vector<uint64_t> h(len);
  uint64_t acc = 1;
  for (size_t i = 0; i < len; i++) {
    h[i] = acc;
    acc = mul(acc, base);
  }
  if (bit_reverse) {
    unsigned bits = 0;
    while ((1ull << bits) < len) bits++;
    std::vector<uint64_t> t(h);
    for (size_t i = 0; i < len; i++) h[brev((unsigned)i, bits)] = t[i];
  }
  cudaError_t e = cudaMalloc(dst, len * sizeof(uint64_t));
  if (e != cudaSuccess) return e;
  return cudaMemcpy(*dst, h.data(), len * sizeof(uint64_t), cudaMemcpyHostToDevice);
}

static base_field *g_tables[10] = {};

static powers_data make_pd(base_field *fine, unsigned fine_log, base_field *coarse, unsigned coarse_log) {
  powers_data d;
  d.fine.values = fine;
  d.fine.mask = (1u << fine_log) - 1;
  d.fine.log_count = fine_log;
  d.coarse.values = coarse;
  d.coarse.mask = (1u << coarse_log) - 1;
  d.coarse.log_count = coarse_log;
  return d;
}

} // namespace refglue

using namespace refglue;

extern "C" cudaError_t ref_context_destroy() {
  for (auto &t : g_tables) {
    if (t) cudaFree(t);
    t = nullptr;
  }
  return cudaGetLastError();
}

extern "C" cudaError_t ref_context_create(unsigned w_coarse_log, unsigned g_coarse_log) {
  if (w_coarse_log > OMEGA_LOG_ORDER || g_coarse_log > OMEGA_LOG_ORDER) return cudaErrorInvalidValue;
  ref_context_destroy();
  cudaError_t e;
#define CK(x)                                                                                                          \
  if ((e = (x)) != cudaSuccess) return e;
  const uint64_t w24 = domain_generator(1ull << OMEGA_LOG_ORDER);
  size_t len_fine = 1ull << (OMEGA_LOG_ORDER - w_coarse_log), len_coarse = 1ull << w_coarse_log;
  CK(upload_powers(w24, len_fine, false, &g_tables[0]));                            // powers_of_w_fine
  CK(upload_powers(domain_generator(len_coarse), len_coarse, false, &g_tables[1])); // powers_of_w_coarse
  len_fine = 1ull << (OMEGA_LOG_ORDER - w_coarse_log - 1);
  CK(upload_powers(w24, len_fine, true, &g_tables[2]));                                     // w fine bitrev
  CK(upload_powers(domain_generator(len_coarse * 2), len_coarse, true, &g_tables[3]));      // w coarse bitrev
  CK(upload_powers(inv(w24), len_fine, true, &g_tables[4]));                                // w inv fine bitrev
  CK(upload_powers(inv(domain_generator(len_coarse * 2)), len_coarse, true, &g_tables[5])); // w inv coarse bitrev
  len_fine = 1ull << (OMEGA_LOG_ORDER - g_coarse_log);
  len_coarse = 1ull << g_coarse_log;
  CK(upload_powers(7, len_fine, false, &g_tables[6]));               // g_f fine
  CK(upload_powers(pw(7, len_fine), len_coarse, false, &g_tables[7])); // g_f coarse
  const uint64_t g_inv = inv(7);
  CK(upload_powers(g_inv, len_fine, false, &g_tables[8]));               // g_i fine
  CK(upload_powers(pw(g_inv, len_fine), len_coarse, false, &g_tables[9])); // g_i coarse

  // copy_to_symbols (src/context.rs:74-142), including its swapped fine/coarse
  // log counts for powers_data_g_i (harmless when both splits are equal).
  unsigned coarse_log = w_coarse_log, fine_log = OMEGA_LOG_ORDER - coarse_log;
  powers_data d = make_pd(g_tables[0], fine_log, g_tables[1], coarse_log);
  CK(cudaMemcpyToSymbol(powers_data_w, &d, sizeof(d)));
  fine_log -= 1;
  d = make_pd(g_tables[2], fine_log, g_tables[3], coarse_log);
  CK(cudaMemcpyToSymbol(powers_data_w_bitrev_for_ntt, &d, sizeof(d)));
  d = make_pd(g_tables[4], fine_log, g_tables[5], coarse_log);
  CK(cudaMemcpyToSymbol(powers_data_w_inv_bitrev_for_ntt, &d, sizeof(d)));
  coarse_log = g_coarse_log;
  fine_log = OMEGA_LOG_ORDER - coarse_log;
  d = make_pd(g_tables[6], fine_log, g_tables[7], coarse_log);
  CK(cudaMemcpyToSymbol(powers_data_g_f, &d, sizeof(d)));
  d = make_pd(g_tables[8], coarse_log, g_tables[9], fine_log);
  CK(cudaMemcpyToSymbol(powers_data_g_i, &d, sizeof(d)));
  uint64_t inv_sizes_host[OMEGA_LOG_ORDER + 1];
  const uint64_t two_inv = inv(2);
  uint64_t acc = 1;
  for (unsigned i = 0; i <= OMEGA_LOG_ORDER; i++) {
    inv_sizes_host[i] = acc;
    acc = mul(acc, two_inv);
  }
  CK(cudaMemcpyToSymbol(inv_sizes, inv_sizes_host, sizeof(inv_sizes_host)));
#undef CK
  return cudaDeviceSynchronize();
}

namespace refglue {
enum Kern { N2B_F7W, N2B_F8W, N2B_F912B, N2B_NF78B, B2N_I7W, B2N_I8W, B2N_I912B, B2N_NI78B, NONE };
struct Step {
  Kern k;
  unsigned stages;
};
// PLANS, src/ntt.rs:74-169: [bitrev_inputs][log_n - 16][3]
static const Step PLANS[2][9][3] = {
    {{{N2B_NF78B, 8}, {N2B_F8W, 8}, {NONE, 0}},
     {{N2B_NF78B, 8}, {N2B_F912B, 9}, {NONE, 0}},
     {{N2B_NF78B, 8}, {N2B_F912B, 10}, {NONE, 0}},
     {{N2B_NF78B, 8}, {N2B_F912B, 11}, {NONE, 0}},
     {{N2B_NF78B, 8}, {N2B_F912B, 12}, {NONE, 0}},
     {{N2B_NF78B, 7}, {N2B_NF78B, 7}, {N2B_F7W, 7}},
     {{N2B_NF78B, 7}, {N2B_NF78B, 7}, {N2B_F8W, 8}},
     {{N2B_NF78B, 7}, {N2B_NF78B, 8}, {N2B_F8W, 8}},
     {{N2B_NF78B, 8}, {N2B_NF78B, 8}, {N2B_F8W, 8}}},
    {{{B2N_I8W, 8}, {B2N_NI78B, 8}, {NONE, 0}},
     {{B2N_I912B, 9}, {B2N_NI78B, 8}, {NONE, 0}},
     {{B2N_I912B, 10}, {B2N_NI78B, 8}, {NONE, 0}},
     {{B2N_I912B, 11}, {B2N_NI78B, 8}, {NONE, 0}},
     {{B2N_I912B, 12}, {B2N_NI78B, 8}, {NONE, 0}},
     {{B2N_I7W, 7}, {B2N_NI78B, 7}, {B2N_NI78B, 7}},
     {{B2N_I8W, 8}, {B2N_NI78B, 7}, {B2N_NI78B, 7}},
     {{B2N_I8W, 8}, {B2N_NI78B, 8}, {B2N_NI78B, 7}},
     {{B2N_I8W, 8}, {B2N_NI78B, 8}, {B2N_NI78B, 8}}}};
static const unsigned NTTS_PER_BLOCK_HOST = 8; // src/ntt.rs:174
} // namespace refglue

// batch_ntt_internal, src/ntt.rs:179-290.  Argument violations (asserts in the
// Rust) return cudaErrorInvalidValue; launches are asynchronous on `stream`.
extern "C" cudaError_t ref_batch_ntt(const uint64_t *inputs_ptr_in, uint64_t *outputs_ptr, unsigned log_n,
                                     unsigned num_ntts, unsigned stride_in, unsigned stride_out, bool bitrev_inputs,
                                     bool inverse, unsigned log_ext, unsigned coset_index, cudaStream_t stream) {
  if (log_n < 1 || log_n + log_ext > OMEGA_LOG_ORDER) return cudaErrorInvalidValue;
  const unsigned n = 1u << log_n;
  if (n > stride_in || n > stride_out) return cudaErrorInvalidValue;
  if (coset_index > 0 && (log_ext == 0 || coset_index >= (1u << log_ext))) return cudaErrorInvalidValue;
  if (num_ntts == 0) return cudaSuccess;
  const base_field *in0 = reinterpret_cast<const base_field *>(inputs_ptr_in);
  base_field *out = reinterpret_cast<base_field *>(outputs_ptr);
  if (log_n < 16) {
    const unsigned threads = 128;
    const unsigned blocks_per_ntt = (n + 2 * threads - 1) / (2 * threads);
    const unsigned blocks = blocks_per_ntt * num_ntts;
    for (unsigned stage = 0; stage < log_n; stage++) {
      const base_field *in = stage == 0 ? in0 : out;
      const unsigned sin = stage == 0 ? stride_in : stride_out;
      if (bitrev_inputs)
        b2n_1_stage<<<blocks, threads, 0, stream>>>(in, out, sin, stride_out, stage, 1, log_n, inverse,
                                                         blocks_per_ntt, log_ext, coset_index);
      else
        n2b_1_stage<<<blocks, threads, 0, stream>>>(in, out, sin, stride_out, stage, 1, log_n, inverse,
                                                         blocks_per_ntt, log_ext, coset_index);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  const Step *plan = PLANS[bitrev_inputs ? 1 : 0][log_n - 16];
  unsigned stage = 0;
  const unsigned num_chunks = (num_ntts + NTTS_PER_BLOCK_HOST - 1) / NTTS_PER_BLOCK_HOST;
  for (int i = 0; i < 3; i++) {
    const Step st = plan[i];
    if (st.k == NONE) continue;
    const unsigned start_stage = stage;
    const base_field *in = stage == 0 ? in0 : out;
    const unsigned sin = stage == 0 ? stride_in : stride_out;
    stage += st.stages;
    dim3 block, grid;
    void (*fn)(const base_field *, base_field *, unsigned, unsigned, unsigned, unsigned, unsigned, bool, unsigned,
               unsigned, unsigned) = nullptr;
    switch (st.k) {
    case N2B_F7W: fn = n2b_final_7_stages_warp; grid = dim3(n / (4 * 128), num_chunks); block = 128; break;
    case N2B_F8W: fn = n2b_final_8_stages_warp; grid = dim3(n / (4 * 256), num_chunks); block = 128; break;
    case N2B_F912B: fn = n2b_final_9_to_12_stages_block; grid = dim3(n / 4096, num_chunks); block = 512; break;
    case N2B_NF78B: fn = n2b_nonfinal_7_or_8_stages_block; grid = dim3(n / 4096, num_chunks); block = 512; break;
    case B2N_I7W: fn = b2n_initial_7_stages_warp; grid = dim3(n / (4 * 128), num_chunks); block = 128; break;
    case B2N_I8W: fn = b2n_initial_8_stages_warp; grid = dim3(n / (4 * 256), num_chunks); block = 128; break;
    case B2N_I912B: fn = b2n_initial_9_to_12_stages_block; grid = dim3(n / 4096, num_chunks); block = 512; break;
    case B2N_NI78B: fn = b2n_noninitial_7_or_8_stages_block; grid = dim3(n / 4096, num_chunks); block = 512; break;
    default: return cudaErrorInvalidValue;
    }
    fn<<<grid, block, 0, stream>>>(in, out, sin, stride_out, start_stage, st.stages, log_n, inverse, num_ntts, log_ext,
                                   coset_index);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return stage == log_n ? cudaSuccess : cudaErrorUnknown;
}

// ---------------------------------------------------------------- ops (src/ops_complex.rs)
// Launch geometry of the reference's wrappers: get_launch_dims = 128-thread
// blocks (src/ops_complex.rs:25-27, src/utils.rs:6-13).
static dim3 ref_grid(unsigned count, unsigned &block) {
  block = count < 128 ? (count ? count : 1) : 128;
  return dim3((count + block - 1) / block);
}

// launch_bit_reverse (src/ops_complex.rs:271-304).
extern "C" cudaError_t ref_bit_reverse(const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride,
                                       unsigned log_rows, unsigned cols, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  const RefMat a{src, (size_t)src_stride}, b{dst, (size_t)dst_stride};
  const unsigned half = log_rows >> 1;
  if (half < 5) {
    unsigned block;
    dim3 grid = ref_grid(1u << log_rows, block);
    grid.y = cols;
    bit_reverse_naive_kernel<<<grid, block, 0, s>>>(a, b, log_rows);
  } else {
    const unsigned tiles = 1u << (half - 5);
    const dim3 grid(tiles * (tiles + 1) / 2, log_rows - (half << 1) + 1, cols), block(32, 2, 2);
    bit_reverse_kernel<<<grid, block, 0, s>>>(a, b, log_rows);
  }
  return cudaGetLastError();
}

// get_powers_of (src/ops_complex.rs:40-56); of_g selects get_powers_of_g.
extern "C" cudaError_t ref_get_powers_of(unsigned log_degree, unsigned offset, bool inverse, bool bit_reverse,
                                         bool of_g, uint64_t *result, unsigned count, void *stream) {
  unsigned block;
  const dim3 grid = ref_grid(count, block);
  if (of_g)
    get_powers_of_g_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(log_degree, offset, inverse, bit_reverse,
                                                                       RefVec{result}, count);
  else
    get_powers_of_w_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(log_degree, offset, inverse, bit_reverse,
                                                                       RefVec{result}, count);
  return cudaGetLastError();
}

// get_powers_by_val (src/ops_complex.rs:117-131) for the base field (ext = false)
// or the extension (result holds 2 * count words).
extern "C" cudaError_t ref_get_powers_by_val(uint64_t base_c0, uint64_t base_c1, bool ext, unsigned offset,
                                             bool bit_reverse, uint64_t *result, unsigned count, void *stream) {
  unsigned block;
  const dim3 grid = ref_grid(count, block);
  if (ext)
    get_powers_by_val_ef_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(RefExt{base_c0, base_c1}, offset,
                                                                            bit_reverse, (RefExt *)result, count);
  else
    get_powers_by_val_bf_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(base_c0, offset, bit_reverse, result,
                                                                            count);
  return cudaGetLastError();
}

// omega_shift (src/ops_complex.rs:220-242).
extern "C" cudaError_t ref_omega_shift(const uint64_t *src, unsigned log_degree, unsigned offset, bool inverse,
                                       unsigned shift, uint64_t *dst, unsigned count, void *stream) {
  unsigned block;
  const dim3 grid = ref_grid(count, block);
  omega_shift_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(src, log_degree, offset, inverse, shift, dst, count);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- barycentric (src/barycentric.rs)
static uint64_t addp(uint64_t a, uint64_t b) {
  a %= P;
  b %= P;
  const uint64_t s = a + b;
  return (s < a || s >= P) ? s - P : s;
}

// precompute_lagrange_coeffs (src/barycentric.rs:83-126): the common-factor kernel, the coefficient kernel with
// 128-thread blocks and INV_BATCH_SIZE 10 (base) / 6 (extension) elements per thread, w_inv_step =
// w_N^-(128 * grid), then the optional bit reversal of the coefficient vector as a matrix of 1 (2) columns.
extern "C" cudaError_t ref_barycentric_precompute(bool ext, const uint64_t *x, uint64_t *cf, uint64_t coset,
                                                  uint64_t *coeffs, unsigned count, bool bit_reverse, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (ext)
    barycentric_precompute_common_factor_ef_kernel<<<1, 1, 0, s>>>((const RefExt *)x, (RefExt *)cf, coset, count);
  else
    barycentric_precompute_common_factor_bf_kernel<<<1, 1, 0, s>>>(x, cf, coset, count);
  unsigned log_count = 0;
  while ((1u << log_count) < count) log_count++;
  const unsigned inv_batch = ext ? 6 : 10, block = 128;
  const unsigned grid = (count + inv_batch * block - 1) / (inv_batch * block);
  const uint64_t w_inv = inv(domain_generator(count));
  const uint64_t w_inv_step = pw(w_inv, (uint64_t)block * grid);
  if (ext)
    barycentric_precompute_lagrange_coeffs_ef_kernel<<<grid, block, 0, s>>>(
        (const RefExt *)x, (const RefExt *)cf, w_inv_step, coset, RefMat{coeffs, (size_t)count}, log_count);
  else
    barycentric_precompute_lagrange_coeffs_bf_kernel<<<grid, block, 0, s>>>(x, cf, w_inv_step, coset,
                                                                            RefVec{coeffs}, log_count);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !bit_reverse) return e;
  return ref_bit_reverse(coeffs, count, coeffs, count, log_count, ext ? 2 : 1, stream);
}

// batch_eval (src/barycentric.rs:183-260): the partial-reduce kernel with blocks of 32 x 32 threads and 12
// (base at base) / 6 elements per thread, then the column sums that the Rust side hands to CUB, done here
// on the host; evals_host gets one word per polynomial (kind 0) or (c0, c1) pairs.  Synchronous.
extern "C" cudaError_t ref_batch_eval(int kind, const uint64_t *ys, unsigned count, unsigned num_polys,
                                      const uint64_t *coeffs, uint64_t *evals_host, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned ept = kind == 0 ? 12 : 6, bx = 32;
  const unsigned grid = (count + ept * bx - 1) / (ept * bx);
  const unsigned grid_size_x = bx * grid;
  const unsigned rows = count < grid_size_x ? count : grid_size_x;
  const unsigned xw = kind == 0 ? 1 : 2;
  uint64_t *partial = nullptr;
  cudaError_t e = cudaMalloc(&partial, (size_t)rows * num_polys * xw * sizeof(uint64_t));
  if (e != cudaSuccess) return e;
  unsigned log_count = 0;
  while ((1u << log_count) < count) log_count++;
  const dim3 block(bx, 32);
  const RefMat y{ys, (size_t)count}, part{partial, (size_t)rows};
  if (kind == 0)
    batch_barycentric_partial_reduce_bf_bf_kernel<<<grid, block, 0, s>>>(y, RefVec{(void *)coeffs}, part, log_count,
                                                                         num_polys);
  else if (kind == 1)
    batch_barycentric_partial_reduce_bf_ef_kernel<<<grid, block, 0, s>>>(y, RefMat{coeffs, (size_t)count}, part,
                                                                         log_count, num_polys);
  else
    batch_barycentric_partial_reduce_ef_ef_kernel<<<grid, block, 0, s>>>(y, RefMat{coeffs, (size_t)count}, part,
                                                                         log_count, num_polys);
  e = cudaGetLastError();
  std::vector<uint64_t> h((size_t)rows * num_polys * xw);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMemcpy(h.data(), partial, h.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost);
  cudaFree(partial);
  if (e != cudaSuccess) return e;
  // base-field column k of the partial matrix (extension: column j = base columns 2j, 2j + 1) -> evals[k]
  for (size_t k = 0; k < (size_t)num_polys * xw; k++) {
    uint64_t acc = 0;
    for (unsigned r = 0; r < rows; r++) acc = addp(acc, h[k * rows + r]);
    evals_host[k] = acc;
  }
  return cudaSuccess;
}

// The partial-reduce kernel of batch_eval alone (asynchronous), into `partial` of at least
// min(count, 32 * grid) * num_polys * (1 or 2) words: what the reference runs on the GPU before the CUB
// column sums (timing only).
extern "C" cudaError_t ref_batch_eval_partial(int kind, const uint64_t *ys, unsigned count, unsigned num_polys,
                                              const uint64_t *coeffs, uint64_t *partial, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned ept = kind == 0 ? 12 : 6, bx = 32;
  const unsigned grid = (count + ept * bx - 1) / (ept * bx);
  const unsigned rows = count < bx * grid ? count : bx * grid;
  unsigned log_count = 0;
  while ((1u << log_count) < count) log_count++;
  const dim3 block(bx, 32);
  const RefMat y{ys, (size_t)count}, part{partial, (size_t)rows};
  if (kind == 0)
    batch_barycentric_partial_reduce_bf_bf_kernel<<<grid, block, 0, s>>>(y, RefVec{(void *)coeffs}, part, log_count,
                                                                         num_polys);
  else if (kind == 1)
    batch_barycentric_partial_reduce_bf_ef_kernel<<<grid, block, 0, s>>>(y, RefMat{coeffs, (size_t)count}, part,
                                                                         log_count, num_polys);
  else
    batch_barycentric_partial_reduce_ef_ef_kernel<<<grid, block, 0, s>>>(y, RefMat{coeffs, (size_t)count}, part,
                                                                         log_count, num_polys);
  return cudaGetLastError();
}
