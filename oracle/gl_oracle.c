/*
 * gl_oracle.c -- CPU oracle for the batched Goldilocks NTT / coset LDE path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke
 * check in __graft_entry__.py and the cpu_baseline leg of bench.py may load
 * it; the product library (era-boojum-cuda_b200/csrc) never links or calls it.
 *
 * It restates, from the mathematics, the transform that the reference's
 * batch entry points compute (src/ntt.rs:179-369) with the conventions of its
 * kernels:
 *   - field p = 2^64 - 2^32 + 1; values may arrive non-canonical (any u64),
 *     src/ntt.rs:424 feeds raw rng.gen() words; outputs here are canonical.
 *   - coset c = g * w_{n*2^e}^k with g = 7 (src/ntt.rs:527-538,
 *     native/context.cuh:33-48: power index k << (24 - log_n - e)).
 *   - forward : y[m] = sum_i x[i] c^i w_n^{i m}
 *     inverse : z[i] = n^-1 c^-i sum_m y[m] w_n^{-i m}
 *     (native/ntt_n2b.cuh:551-579, native/ntt_b2n.cuh:562-590: the coset
 *      factor always uses the NATURAL index i).
 *   - ordering: bitrev_inputs = false (n2b) reads natural order and writes
 *     bit-reversed order; bitrev_inputs = true (b2n) reads bit-reversed order
 *     and writes natural order (src/ntt.rs:561-582).
 *   - roots of unity: w_{2^32} = 7^((p-1)/2^32), w_{2^k} = w_{2^32}^{2^(32-k)}.
 *     boojum's own domain_generator_for_size is not vendored with the
 *     reference, so this choice of root is fixed here and fed to the
 *     reference kernels by oracle/ref_glue.cu as well.
 *
 * The transform is computed with a textbook natural-order Cooley-Tukey NTT
 * (bit-reverse permutation followed by log_n butterfly levels with the powers
 * w^j), deliberately a different factorisation from the product kernels, and
 * with an O(n^2) definition-based DFT for tiny sizes so tests can pin the
 * fast path.
 *
 * Pinning: against the reference's own CUDA kernels, compiled from its
 * sources into oracle/_ref (GPU tests, same inputs), and without a GPU
 * against the SHA-256 digests of those kernels' outputs on 176 seeded cases
 * (tests/golden/, tests/test_golden.py).  Unpinned: boojum's own root of
 * unity (above), for which no source or vector exists here.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define GL_P 0xffffffff00000001ull
#define GL_EPS 0xffffffffull

typedef unsigned __int128 u128;

static inline uint64_t gl_canon(uint64_t x) { return x >= GL_P ? x - GL_P : x; }

static inline uint64_t gl_add(uint64_t a, uint64_t b) {
  /* a, b canonical */
  uint64_t s = a + b;
  if (s < a || s >= GL_P) s -= GL_P;
  return s;
}

static inline uint64_t gl_sub(uint64_t a, uint64_t b) {
  /* a, b canonical */
  return a >= b ? a - b : a + (GL_P - b);
}

/* a * b mod p for canonical a, b: x = lo + 2^64 hl + 2^96 hh = lo - hh + hl * (2^32 - 1) (mod p). */
static inline uint64_t gl_mul(uint64_t a, uint64_t b) {
  u128 x = (u128)a * b;
  uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
  uint64_t hh = hi >> 32, hl = hi & GL_EPS;
  uint64_t t0 = lo - hh;
  if (lo < hh) t0 -= GL_EPS;
  uint64_t t1 = hl * GL_EPS;
  uint64_t r = t0 + t1;
  if (r < t1) r += GL_EPS;
  return gl_canon(r);
}

uint64_t gl_oracle_mul(uint64_t a, uint64_t b) { return gl_mul(gl_canon(a), gl_canon(b)); }

uint64_t gl_oracle_pow(uint64_t base, uint64_t e) {
  uint64_t r = 1, b = gl_canon(base);
  while (e) {
    if (e & 1) r = gl_mul(r, b);
    b = gl_mul(b, b);
    e >>= 1;
  }
  return r;
}

uint64_t gl_oracle_inv(uint64_t a) { return gl_oracle_pow(a, GL_P - 2); }

/* w_{2^log_size}: primitive 2^log_size-th root of unity, log_size <= 32. */
uint64_t gl_oracle_root_of_unity(unsigned log_size) {
  uint64_t w32 = gl_oracle_pow(7, (GL_P - 1) >> 32);
  return gl_oracle_pow(w32, 1ull << (32 - log_size));
}

/* Coset shift c of src/ntt.rs:527-538: 1 when log_ext == 0, else 7 * w_{n 2^e}^k. */
uint64_t gl_oracle_coset(unsigned log_n, unsigned log_ext, unsigned coset_idx) {
  if (log_ext == 0) return 1;
  uint64_t w = gl_oracle_root_of_unity(log_n + log_ext);
  return gl_mul(7, gl_oracle_pow(w, coset_idx));
}

static inline uint32_t brev(uint32_t x, unsigned bits) {
  if (bits == 0) return 0;
  x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
  x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
  x = ((x >> 4) & 0x0f0f0f0fu) | ((x & 0x0f0f0f0fu) << 4);
  x = ((x >> 8) & 0x00ff00ffu) | ((x & 0x00ff00ffu) << 8);
  x = (x >> 16) | (x << 16);
  return x >> (32 - bits);
}

/* In-place natural-order NTT: a[m] <- sum_i a[i] w^{i m}, w of order 2^log_n.
 * powers[j] = w^j for j < n/2. */
static void ntt_natural(uint64_t *a, unsigned log_n, const uint64_t *powers) {
  const uint32_t n = 1u << log_n;
  for (uint32_t i = 0; i < n; i++) {
    uint32_t j = brev(i, log_n);
    if (i < j) {
      uint64_t t = a[i];
      a[i] = a[j];
      a[j] = t;
    }
  }
  for (unsigned lvl = 1; lvl <= log_n; lvl++) {
    const uint32_t len = 1u << lvl, half = len >> 1, step = n >> lvl;
    for (uint32_t base = 0; base < n; base += len) {
      for (uint32_t j = 0; j < half; j++) {
        uint64_t u = a[base + j];
        uint64_t v = gl_mul(a[base + j + half], powers[(uint64_t)j * step]);
        a[base + j] = gl_add(u, v);
        a[base + j + half] = gl_sub(u, v);
      }
    }
  }
}

typedef struct {
  const uint64_t *in;
  uint64_t *out;
  unsigned log_n;
  uint32_t num_ntts;
  uint64_t stride_in, stride_out;
  int bitrev_inputs, inverse;
  uint64_t coset;     /* c (forward) or c^-1 (inverse) */
  uint64_t scale;     /* 1 (forward) or n^-1 (inverse) */
  const uint64_t *powers;
  uint32_t col_begin, col_step;
} job_t;

static void run_columns(const job_t *jb) {
  const uint32_t n = 1u << jb->log_n;
  uint64_t *buf = (uint64_t *)malloc(sizeof(uint64_t) * n);
  for (uint32_t col = jb->col_begin; col < jb->num_ntts; col += jb->col_step) {
    const uint64_t *src = jb->in + (uint64_t)col * jb->stride_in;
    uint64_t *dst = jb->out + (uint64_t)col * jb->stride_out;
    for (uint32_t i = 0; i < n; i++) buf[i] = gl_canon(src[jb->bitrev_inputs ? brev(i, jb->log_n) : i]);
    if (!jb->inverse && jb->coset != 1) {
      uint64_t c = 1;
      for (uint32_t i = 0; i < n; i++) {
        buf[i] = gl_mul(buf[i], c);
        c = gl_mul(c, jb->coset);
      }
    }
    ntt_natural(buf, jb->log_n, jb->powers);
    if (jb->inverse) {
      uint64_t c = jb->scale;
      for (uint32_t i = 0; i < n; i++) {
        buf[i] = gl_mul(buf[i], c);
        c = gl_mul(c, jb->coset);
      }
    }
    for (uint32_t m = 0; m < n; m++) dst[jb->bitrev_inputs ? m : brev(m, jb->log_n)] = buf[m];
  }
  free(buf);
}

static void *thread_main(void *arg) {
  run_columns((const job_t *)arg);
  return NULL;
}

/*
 * Batched NTT with the argument meaning of batch_ntt_internal
 * (src/ntt.rs:179-191), 64-bit strides, `threads` host threads over columns.
 * Returns 0, or -1 on invalid arguments (same checks as src/ntt.rs:192-200).
 * in == out is allowed (each column is staged through a private buffer).
 */
int gl_oracle_batch_ntt(const uint64_t *in, uint64_t *out, unsigned log_n, uint32_t num_ntts, uint64_t stride_in,
                        uint64_t stride_out, int bitrev_inputs, int inverse, unsigned log_ext, unsigned coset_idx,
                        int threads) {
  if (log_n < 1 || log_n + log_ext > 32) return -1;
  const uint64_t n = 1ull << log_n;
  if (n > stride_in || n > stride_out) return -1;
  if (coset_idx > 0 && (log_ext == 0 || coset_idx >= (1u << log_ext))) return -1;
  if (num_ntts == 0) return 0;
  if (threads < 1) threads = 1;
  if ((uint32_t)threads > num_ntts) threads = (int)num_ntts;

  uint64_t w = gl_oracle_root_of_unity(log_n);
  if (inverse) w = gl_oracle_inv(w);
  uint64_t *powers = (uint64_t *)malloc(sizeof(uint64_t) * (n / 2));
  powers[0] = 1;
  for (uint64_t j = 1; j < n / 2; j++) powers[j] = gl_mul(powers[j - 1], w);

  uint64_t c = gl_oracle_coset(log_n, log_ext, coset_idx);
  job_t base = {in, out, log_n, num_ntts, stride_in, stride_out, bitrev_inputs, inverse,
                inverse ? gl_oracle_inv(c) : c, inverse ? gl_oracle_inv(n % GL_P) : 1, powers, 0, 1};

  /* in-place calls: other columns must not be overwritten before they are read, which holds because
   * every column is read and written only by its own thread, but columns may overlap when strides
   * are tiny; the reference asserts n <= stride, so columns are disjoint. */
  if (threads == 1) {
    run_columns(&base);
  } else {
    pthread_t *tid = (pthread_t *)malloc(sizeof(pthread_t) * threads);
    job_t *jobs = (job_t *)malloc(sizeof(job_t) * threads);
    for (int t = 0; t < threads; t++) {
      jobs[t] = base;
      jobs[t].col_begin = (uint32_t)t;
      jobs[t].col_step = (uint32_t)threads;
      pthread_create(&tid[t], NULL, thread_main, &jobs[t]);
    }
    for (int t = 0; t < threads; t++) pthread_join(tid[t], NULL);
    free(tid);
    free(jobs);
  }
  free(powers);
  return 0;
}

/*
 * Coset LDE as the reference's callers compose it (src/ntt.rs:527-583 with
 * benches/ntt.rs:114-116): bit-reversed evaluations on H -> inverse NTT (b2n,
 * natural coefficients) -> for each coset k < 2^log_blowup a forward n2b NTT
 * with (log_ext = log_blowup, coset_idx = k).  Coset k of column j is written
 * at out + k * coset_stride + j * stride_out, in bit-reversed order.
 */
int gl_oracle_lde(const uint64_t *in, uint64_t *out, unsigned log_n, uint32_t num_cols, uint64_t stride_in,
                  uint64_t stride_out, uint64_t coset_stride, unsigned log_blowup, int threads) {
  const uint64_t n = 1ull << log_n;
  if (log_n < 1 || log_n + log_blowup > 32 || n > stride_in || n > stride_out) return -1;
  uint64_t *coef = (uint64_t *)malloc(sizeof(uint64_t) * n * (num_cols ? num_cols : 1));
  int rc = gl_oracle_batch_ntt(in, coef, log_n, num_cols, stride_in, n, 1, 1, 0, 0, threads);
  for (unsigned k = 0; rc == 0 && k < (1u << log_blowup); k++)
    rc = gl_oracle_batch_ntt(coef, out + k * coset_stride, log_n, num_cols, n, stride_out, 0, 0, log_blowup, k,
                             threads);
  free(coef);
  return rc;
}

/* O(n^2) DFT straight from the definition, natural order in and out, used to
 * pin the fast path on tiny sizes: y[m] = sum_i x[i] w^{i m}. */
void gl_oracle_dft_naive(const uint64_t *x, uint64_t *y, unsigned log_n, int inverse) {
  const uint64_t n = 1ull << log_n;
  uint64_t w = gl_oracle_root_of_unity(log_n);
  if (inverse) w = gl_oracle_inv(w);
  for (uint64_t m = 0; m < n; m++) {
    uint64_t acc = 0, wm = gl_oracle_pow(w, m), t = 1;
    for (uint64_t i = 0; i < n; i++) {
      acc = gl_add(acc, gl_mul(gl_canon(x[i]), t));
      t = gl_mul(t, wm);
    }
    y[m] = acc;
  }
}

void gl_oracle_canonicalize(uint64_t *x, uint64_t count) {
  for (uint64_t i = 0; i < count; i++) x[i] = gl_canon(x[i]);
}

/* ------------------------------------------------------------------ ops beside the NTT
 * Restatements of the reference's src/ops_complex.rs operations with the
 * index conventions of its kernels (native/ops_complex.cu:9-157) and of its
 * power tables (native/context.cuh:9-48: omega = w_{2^24}, exponents mod
 * 2^24, inverse = w^-e; g = 7).  Element by element, with full
 * exponentiations, so they share nothing with the product's tables or running
 * products. */

static inline uint32_t brev32(uint32_t x) { return brev(x, 32); }

/* dst[brev_{log_rows}(i)] = src[i] in each column (src and dst distinct). */
void gl_oracle_bit_reverse(const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride,
                           unsigned log_rows, uint32_t cols) {
  const uint64_t rows = 1ull << log_rows;
  for (uint32_t c = 0; c < cols; c++)
    for (uint64_t i = 0; i < rows; i++) dst[c * dst_stride + brev((uint32_t)i, log_rows)] = src[c * src_stride + i];
}

/* native/ops_complex.cu:9-33: r = i + offset (u32), idx = bit_reverse ?
 * brev_{log_degree}(r) : r, e = (idx << (24 - log_degree)) mod 2^24; the
 * value is w_{2^24}^e (of_g = 0) or 7^e (of_g = 1), inverted bases when
 * inverse. */
void gl_oracle_powers_of(unsigned log_degree, uint32_t offset, int inverse, int bit_reverse, int of_g,
                         uint64_t *result, uint32_t count) {
  uint64_t base = of_g ? 7 : gl_oracle_root_of_unity(24);
  if (inverse) base = gl_oracle_inv(base);
  for (uint32_t i = 0; i < count; i++) {
    const uint32_t r = i + offset;
    const uint32_t idx = bit_reverse ? brev(r & (log_degree ? (uint32_t)((1ull << log_degree) - 1) : 0u), log_degree) : r;
    const uint32_t e = (uint32_t)(idx << (24 - log_degree)) & ((1u << 24) - 1);
    result[i] = gl_oracle_pow(base, e);
  }
}

/* Quadratic extension F_p[x] / (x^2 - 7) (native/goldilocks_extension.cuh:11-80). */
static void ext_mul(const uint64_t a[2], const uint64_t b[2], uint64_t r[2]) {
  const uint64_t c0 = gl_add(gl_mul(a[0], b[0]), gl_mul(7, gl_mul(a[1], b[1])));
  const uint64_t c1 = gl_add(gl_mul(a[0], b[1]), gl_mul(a[1], b[0]));
  r[0] = c0;
  r[1] = c1;
}

static void ext_pow(const uint64_t base[2], uint32_t e, uint64_t r[2]) {
  uint64_t acc[2] = {1, 0}, b[2] = {gl_canon(base[0]), gl_canon(base[1])};
  while (e) {
    if (e & 1) ext_mul(acc, b, acc);
    ext_mul(b, b, b);
    e >>= 1;
  }
  r[0] = acc[0];
  r[1] = acc[1];
}

/* native/ops_complex.cu:35-74: e = (bit_reverse ? brev_32(i) : i) + offset
 * (u32), result[i] = base^e; the extension version stores its two
 * coordinates at result[i] and result[i + count]. */
void gl_oracle_powers_by(uint64_t base_c0, uint64_t base_c1, int ext, uint32_t offset, int bit_reverse,
                         uint64_t *result, uint32_t count) {
  const uint64_t base[2] = {base_c0, base_c1};
  for (uint32_t i = 0; i < count; i++) {
    const uint32_t e = (bit_reverse ? brev32(i) : i) + offset;
    if (ext) {
      uint64_t v[2];
      ext_pow(base, e, v);
      result[i] = v[0];
      result[(uint64_t)count + i] = v[1];
    } else {
      result[i] = gl_oracle_pow(base_c0, e);
    }
  }
}

/* native/ops_complex.cu:76-87: dst[i] = src[i] * w_{2^24}^{+-e},
 * e = ((shift * (i + offset)) << (24 - log_degree)) mod 2^24 in u32 arithmetic. */
void gl_oracle_omega_shift(const uint64_t *src, unsigned log_degree, uint32_t offset, int inverse, uint32_t shift,
                           uint64_t *dst, uint32_t count) {
  uint64_t w = gl_oracle_root_of_unity(24);
  if (inverse) w = gl_oracle_inv(w);
  for (uint32_t i = 0; i < count; i++) {
    const uint32_t e = (uint32_t)((shift * (i + offset)) << (24 - log_degree)) & ((1u << 24) - 1);
    dst[i] = gl_mul(gl_canon(src[i]), gl_oracle_pow(w, e));
  }
}

/* ------------------------------------------------------------------ barycentric evaluation
 * src/barycentric.rs, native/barycentric.cu: L_i(x) = cf * w^i / (x - c w^i),
 * cf = c (x^N - c^N) / (N c^N), w = w_N, N = 2^log_count; x in the base field
 * (ext = 0) or in F_p[x]/(x^2 - 7).  Element by element with a full inversion
 * each (the reference's zero convention: inv(0) = 0). */

static void ext_inv(const uint64_t a[2], uint64_t r[2]) {
  /* (a0 + a1 x)^-1 = (a0 - a1 x) / (a0^2 - 7 a1^2) */
  const uint64_t a0 = gl_canon(a[0]), a1 = gl_canon(a[1]);
  const uint64_t nrm = gl_sub(gl_mul(a0, a0), gl_mul(7, gl_mul(a1, a1)));
  const uint64_t ni = gl_oracle_inv(nrm);
  r[0] = gl_mul(a0, ni);
  r[1] = gl_sub(0, gl_mul(a1, ni));
}

/* out: N values (base) or 2N words, all c0 then all c1 (extension); natural
 * order, bit-reversed when bit_reverse. */
void gl_oracle_lagrange_coeffs(uint64_t x0, uint64_t x1, int ext, uint64_t coset, unsigned log_count, int bit_reverse,
                               uint64_t *out) {
  const uint64_t n = 1ull << log_count;
  const uint64_t c = gl_canon(coset);
  const uint64_t x[2] = {gl_canon(x0), ext ? gl_canon(x1) : 0};
  uint64_t xn[2];
  ext_pow(x, (uint32_t)n, xn); /* x^N; N <= 2^31 */
  const uint64_t cn = gl_oracle_pow(c, n);
  const uint64_t den_inv = gl_oracle_inv(gl_mul(n % GL_P, cn));
  const uint64_t cf[2] = {gl_mul(gl_mul(gl_sub(xn[0], cn), c), den_inv), gl_mul(gl_mul(xn[1], c), den_inv)};
  const uint64_t w = gl_oracle_root_of_unity(log_count);
  uint64_t wi = 1;
  for (uint64_t i = 0; i < n; i++) {
    const uint64_t cw = gl_mul(c, wi);
    const uint64_t d[2] = {gl_sub(x[0], cw), x[1]};
    uint64_t di[2], l[2];
    ext_inv(d, di);
    const uint64_t cfw[2] = {gl_mul(cf[0], wi), gl_mul(cf[1], wi)};
    ext_mul(cfw, di, l);
    const uint64_t pos = bit_reverse ? brev((uint32_t)i, log_count) : i;
    out[pos] = l[0];
    if (ext) out[n + pos] = l[1];
    wi = gl_mul(wi, w);
  }
}

/* eval_j = sum_i y_{i,j} L_i.  kind 0: base values, base coefficients; 1: base
 * values, extension coefficients; 2: extension values (column j = base columns
 * 2j, 2j + 1) and extension coefficients.  out: one word (kind 0) or a (c0, c1)
 * pair per polynomial. */
void gl_oracle_batch_eval(int kind, const uint64_t *ys, uint32_t count, uint32_t num_polys, const uint64_t *coeffs,
                          uint64_t *out) {
  for (uint32_t j = 0; j < num_polys; j++) {
    uint64_t acc[2] = {0, 0};
    for (uint32_t i = 0; i < count; i++) {
      uint64_t y[2], l[2], pr[2];
      if (kind == 2) {
        y[0] = gl_canon(ys[(uint64_t)2 * j * count + i]);
        y[1] = gl_canon(ys[(uint64_t)(2 * j + 1) * count + i]);
      } else {
        y[0] = gl_canon(ys[(uint64_t)j * count + i]);
        y[1] = 0;
      }
      l[0] = gl_canon(coeffs[i]);
      l[1] = kind == 0 ? 0 : gl_canon(coeffs[count + i]);
      ext_mul(y, l, pr);
      acc[0] = gl_add(acc[0], pr[0]);
      acc[1] = gl_add(acc[1], pr[1]);
    }
    if (kind == 0) {
      out[j] = acc[0];
    } else {
      out[2 * j] = acc[0];
      out[2 * j + 1] = acc[1];
    }
  }
}

/* sum_i a_{i,j} x^i for num_polys coefficient columns of count rows (Horner);
 * x and the coefficients in the base field or the extension as above. */
void gl_oracle_poly_eval(int ext_coeffs, const uint64_t *coeffs, uint32_t count, uint32_t num_polys, uint64_t x0,
                         uint64_t x1, uint64_t *out) {
  const uint64_t x[2] = {gl_canon(x0), gl_canon(x1)};
  for (uint32_t j = 0; j < num_polys; j++) {
    uint64_t acc[2] = {0, 0};
    for (int64_t i = (int64_t)count - 1; i >= 0; i--) {
      uint64_t t[2];
      ext_mul(acc, x, t);
      if (ext_coeffs) {
        acc[0] = gl_add(t[0], gl_canon(coeffs[(uint64_t)2 * j * count + i]));
        acc[1] = gl_add(t[1], gl_canon(coeffs[(uint64_t)(2 * j + 1) * count + i]));
      } else {
        acc[0] = gl_add(t[0], gl_canon(coeffs[(uint64_t)j * count + i]));
        acc[1] = t[1];
      }
    }
    out[2 * j] = acc[0];
    out[2 * j + 1] = acc[1];
  }
}
