// ntt_pass.cuh -- one multi-stage pass of a batched Goldilocks NTT (sm_100a).
//
// Index bits of a length-2^log_n column are processed in passes.  A pass owns
// a window of K consecutive bits [lb, lb + K) and runs every radix-2 stage
// that pairs indices differing in one of those bits:
//   * natural -> bit-reversed (n2b, the reference's DIT kernels,
//     native/ntt_n2b.cuh): stages go from the window's top bit down, with the
//     butterfly (a, b) -> (a + b*t, a - b*t);
//   * bit-reversed -> natural (b2n, native/ntt_b2n.cuh): stages go from the
//     window's bottom bit up, with (a, b) -> (a + b, (a - b)*t).
// For a stage on index bit a, the pair whose index has upper part
// r = idx >> (a + 1) uses twiddle T[r] (see tables.cuh); T[r] does not depend
// on the stage, exactly as in the reference (native/ntt.cu:23-35).
//
// Plain tile loads bypass L1 (ld.global.cg): a tile is read once.  The 8-byte
// cp.async tile copies can only be .ca (the padded slots are not 16-byte
// aligned); in the persistent batch kernel, where another SM may have written
// a tile during the launch, a CTA reads a job's tiles only after an
// ld.acquire.gpu of the producing kernel's counter and a barrier, which
// orders those reads after the writes in the PTX memory model.
//
// Tile.  A CTA owns one tile position: the bits above the window (H) and a
// run of C consecutive values of the bits below it (l0 .. l0 + C - 1), and
// walks over columns G at a time.  A tile is G x 2^K x C elements, loaded
// with coalesced 16-byte accesses into padded shared memory (one pad word
// every 16 words keeps the strided radix-16 accesses conflict-free), then
// processed in rounds of up to 4 stages held in registers (16 values per
// thread), then stored.  A round multiplies by powers s^j of one twiddle per
// group and then runs a fixed network of shift multiplications (see the
// factored rounds below); the 2^K - 1 powers a tile position needs are
// computed once per CTA into shared memory and reused for all its columns.
//
// Column groups.  Columns may come in 2^log_groups groups (group k at
// group_stride from group 0) whose transforms carry an extra index prefix
// brev(k) above bit log_n: group k then computes block brev(k) of a transform
// of size 2^(log_n + log_groups) whose input is zero outside block 0.  The
// fused LDE uses this for its coset blocks (lde.cu); a plain transform has one
// group.
//
// Fused scaling (same places as the reference): a forward LDE pass multiplies
// element i by c^i on load (native/ntt_n2b.cuh:369-400); the last pass of an
// inverse transform multiplies by n^-1 * c^-i on store
// (native/ntt_n2b.cuh:68-99), i being the NATURAL index of the element.
// The last pass also reduces its outputs to canonical form.
#pragma once
#include "gl.cuh"
#include "tables.cuh"

// Resident CTAs per SM the pass kernels are compiled for (256 threads each):
// natural->bit-reversed passes 2 (128 registers a thread), bit-reversed->natural
// ones 3 (80 registers; measured ~9 % faster on B200, while the n2b ones gain
// nothing from the third CTA) for windows of 9 bits and more (smaller windows
// spill at 80 registers).
#ifndef BC_PASS_MIN_BLOCKS
#define BC_PASS_MIN_BLOCKS 2
#endif
#ifndef BC_PASS_MIN_BLOCKS_B2N
#define BC_PASS_MIN_BLOCKS_B2N 3
#endif
// The same for the fused LDE's top-window kernel (lde.cu).
#ifndef BC_TOP_MIN_BLOCKS
#define BC_TOP_MIN_BLOCKS 2
#endif

namespace bc {

struct PassParams {
  const uint64_t *in;
  uint64_t *out;
  uint64_t stride_in;
  uint64_t stride_out;
  uint64_t group_stride_in;  // distance between column groups (elements)
  uint64_t group_stride_out;
  uint32_t group_cols;       // columns per group
  uint32_t chunks_per_group; // grid.y = groups * chunks_per_group
  uint32_t log_groups;       // group k carries index prefix brev(k)
  uint32_t log_n;
  uint32_t lb;           // lowest index bit of the window
  uint32_t log_g;        // columns per tile iteration = 2^log_g
  uint32_t cols_per_cta; // multiple of 2^log_g
  uint32_t inverse;      // inverse twiddles
  uint32_t load_scale;   // multiply by c^i on load
  uint32_t store_scale;  // multiply by n^-1 c^-i on store
  uint32_t canon_out;    // canonical outputs
  uint32_t has_coset;    // c != 1 (log_extension_degree > 0)
  uint32_t coset_kshift; // coset_idx << (PW_LOG - log_n - log_ext)
  uint32_t vec_in;       // 16-byte loads allowed (alignment checked on the host)
  uint32_t vec_out;      // 16-byte stores allowed
  DevTables tabs;
};

__device__ __forceinline__ uint64_t ld_tab(const uint64_t *p) { return __ldg(p); }

// T[r] for the forward (inv = 0) or inverse (inv = 1) twiddle table.
__device__ __forceinline__ uint64_t twiddle(const DevTables &t, uint32_t inv, uint32_t r) {
  const uint64_t lo = ld_tab(t.tw_lo[inv] + (r & ((1u << TW_FINE) - 1)));
  const uint32_t rh = r >> TW_FINE;
  return rh ? gl::mul(lo, ld_tab(t.tw_hi[inv] + rh)) : lo;
}

// g^i (inv = 0) or g^-i (inv = 1).
__device__ __forceinline__ uint64_t g_power(const DevTables &t, uint32_t inv, uint32_t i) {
  uint64_t r = ld_tab(t.g_lo[inv] + (i & ((1u << G_FINE) - 1)));
  const uint32_t ih = i >> G_FINE;
  return ih ? gl::mul(r, ld_tab(t.g_hi[inv] + ih)) : r;
}

// c^i (inv = 0) or c^-i (inv = 1), c = g * w_{n*2^e}^k.  kshift = k << (PW_LOG - log_n - e).
__device__ __forceinline__ uint64_t coset_power(const DevTables &t, uint32_t inv, uint32_t i, uint32_t kshift) {
  uint64_t r = g_power(t, inv, i);
  if (kshift) {
    const uint32_t e = (i * kshift) & ((1u << PW_LOG) - 1);
    uint64_t w = ld_tab(t.w_lo[inv] + (e & ((1u << PW_FINE) - 1)));
    const uint32_t eh = e >> PW_FINE;
    if (eh) w = gl::mul(w, ld_tab(t.w_hi[inv] + eh));
    r = gl::mul(r, w);
  }
  return r;
}

// w_{2^24}^e (inv = 1: w^-e) for e < 2^24, the reference's omega and index
// convention (native/context.cuh:9-48): w_{2^24} = w_{2^PW_LOG}^(2^(PW_LOG-24)).
__device__ __forceinline__ uint64_t w24_power(const DevTables &t, uint32_t inv, uint32_t e) {
  const uint32_t e30 = e << (PW_LOG - 24);
  const uint64_t w = ld_tab(t.w_lo[inv] + (e30 & ((1u << PW_FINE) - 1)));
  const uint32_t eh = e30 >> PW_FINE;
  return eh ? gl::mul(w, ld_tab(t.w_hi[inv] + eh)) : w;
}

__device__ __forceinline__ uint32_t pad16(uint32_t x) { return x + (x >> 4); }

// Asynchronous global -> shared copies (cp.async); completion by cp_async_wait
// (then a barrier before other threads read the data).
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ uint32_t brev_bits(uint32_t x, uint32_t bits) { return bits ? __brev(x) >> (32 - bits) : 0; }

// ---------------------------------------------------------------- factored rounds
// A round holds V window bits [B, B + V) of 16 / 2^V groups per thread in
// registers: x[q * 2^V + j] is element j of the thread's q-th group (j is the
// value of the round's bits, its top bit the round's top stage bit).
//
// Factoring.  In a round, the pair of stage bit a = B + qq uses
// T[(R << (V-1-qq)) + u]: R = idx >> (B + V) is the upper part of the group
// (one value for its 2^V elements) and u = j >> (qq + 1) < 2^(V-1-qq) are the
// round bits above a.  Bit-reversed twiddles multiply over disjoint bit fields,
// T[(R << m) + u] = T[R << m] T[u], and T[2r]^2 = T[r] gives
// T[R << m] = s^(2^(V-1-m)) with s = T[R << (V-1)].  A DIT round is therefore
//     x_j <- x_j s^j  (j = 1 .. 2^V - 1),  then the same network with R = 0,
// and a DIF round (its inverse, stage by stage, with the inverse table) is the
// R = 0 network followed by x_j <- x_j s^j.  The R = 0 network's twiddles
// T[u], u < 8, are signed powers of two (small_tw_exp), applied with shifts
// (gl::mul_pow2): a round costs 2^V - 1 general multiplications instead of
// V 2^(V-1), plus shift multiplications.  Both networks use Cooley-Tukey
// butterflies (cstage); one by -2^e swaps its sum and difference.
//
// Power table of one tile position.  The window's rounds partition its bits
// into full rounds [K - 4(i+1), K - 4i) from the top and a short round
// [0, K mod 4).  The round on [B, B + V) has NR = 2^(K-B-V) values of
// R_local (the window bits above it; R = (H << (K-B-V)) + R_local) and keeps
// s^j of R_local at entry (NR - 1) + R_local (2^V - 1) + j - 1: the rounds
// above it hold exactly NR - 1 entries, and the table 2^K - 1.  The odd
// stride 2^V - 1 keeps a half-warp's reads of distinct R_local on distinct
// banks.

// Tile index of element 0 of group gi, and its window value w (bits [B, B+V) zero).
// Which index runs fastest across consecutive threads of a round: runs of C
// low positions first keeps a half-warp on 16 distinct banks for every full
// round; a short round on the window's bottom bits with C > 1 instead needs
// the other window bits first (group stride 2^V * C <= 16 words).
template <int C, int B, int V> struct GroupOrder {
  static constexpr bool window_first = (V < 4) && (B == 0) && (C > 1) && ((1 << V) * C <= 16);
};

template <int K, int C, int B, int V>
__device__ __forceinline__ uint32_t group_base(uint32_t gi, uint32_t &w) {
  constexpr int W = 1 << K;
  uint32_t lc, g, wo;
  if constexpr (GroupOrder<C, B, V>::window_first) {
    wo = gi & ((1u << (K - V)) - 1);
    const uint32_t rest = gi >> (K - V);
    lc = rest % C;
    g = rest / C;
  } else {
    lc = gi % C;
    const uint32_t rest = gi / C;
    g = rest >> (K - V);
    wo = rest & ((1u << (K - V)) - 1);
  }
  w = (wo & ((1u << B) - 1)) | ((wo >> B) << (B + V));
  return (g * W + w) * C + lc;
}

template <int K, int C, int B, int V>
__device__ __forceinline__ void load_groups(const uint64_t *tile, uint64_t (&x)[16], uint32_t tid, uint32_t nthreads) {
  constexpr int NV = 1 << V, NG = 16 / NV;
#pragma unroll
  for (int q = 0; q < NG; q++) {
    uint32_t w;
    const uint32_t eb = group_base<K, C, B, V>(tid + nthreads * q, w);
#pragma unroll
    for (int j = 0; j < NV; j++) x[q * NV + j] = tile[pad16(eb + ((uint32_t)j << B) * C)];
  }
}

template <int K, int C, int B, int V>
__device__ __forceinline__ void store_groups(uint64_t *tile, const uint64_t (&x)[16], uint32_t tid, uint32_t nthreads) {
  constexpr int NV = 1 << V, NG = 16 / NV;
#pragma unroll
  for (int q = 0; q < NG; q++) {
    uint32_t w;
    const uint32_t eb = group_base<K, C, B, V>(tid + nthreads * q, w);
#pragma unroll
    for (int j = 0; j < NV; j++) tile[pad16(eb + ((uint32_t)j << B) * C)] = x[q * NV + j];
  }
}

// Round ri of K window bits.  DIT rounds run top-down with the short round
// last; DIF rounds run bottom-up, short round last or (RAGGED_FIRST) first.
template <int K, bool DIF, bool RAGGED_FIRST, int RI> struct RoundShape {
  static constexpr int R = K % 4;
  static constexpr int lo_dif = (RAGGED_FIRST && R) ? (RI == 0 ? 0 : R + 4 * (RI - 1)) : 4 * RI;
  static constexpr int v_dif = (RAGGED_FIRST && R) ? (RI == 0 ? R : 4) : ((K - 4 * RI) < 4 ? (K - 4 * RI) : 4);
  static constexpr int hi_dit = K - 4 * RI;
  static constexpr int V = DIF ? v_dif : (hi_dit < 4 ? hi_dit : 4);
  static constexpr int B = DIF ? lo_dif : hi_dit - V;
  static constexpr int NR = (K + 3) / 4;
};

// The other partition of a window, used by the top-window kernel's direct
// path (lde.cuh): the short round on the window's top bits [K - R, K), full
// rounds below it down to bit 0.  Rounds are listed top-down (RI = 0 is the
// top one); with R = 0 it is RoundShape's DIT partition.
template <int K, int RI> struct ShortTopShape {
  static constexpr int R = K % 4;
  static constexpr int V = (R && RI == 0) ? R : 4;
  static constexpr int B = R ? (RI == 0 ? K - R : K - R - 4 * RI) : K - 4 - 4 * RI;
  static constexpr int NR = K / 4 + (R ? 1 : 0);
};

// Round RI of partition PART (0: RoundShape's DIT partition, short round at
// the bottom; 1: ShortTopShape).
template <int K, int RI, int PART> struct PartShape {
  using type = RoundShape<K, false, false, RI>;
};
template <int K, int RI> struct PartShape<K, RI, 1> {
  using type = ShortTopShape<K, RI>;
};

// Words of a tile position's power table, and its fill tasks (R_local values
// over all rounds).
template <int K> struct PowWords {
  static constexpr uint32_t words = 1u << K;
  static constexpr uint32_t tasks = ((1u << (4 * (K / 4))) - 1) / 15 + (K % 4 ? (1u << (K - K % 4)) : 0);
};

// Powers s^1 .. s^(2^V - 1) of every R_local of the round on [B, B + V).
// Tasks start at thread `first` so that consecutive rounds use different threads.
template <int K, int B, int V>
__device__ __forceinline__ void fill_round_powers(uint64_t *pw, const DevTables &tabs, uint32_t inv, uint32_t H,
                                                  uint32_t first, uint32_t tid, uint32_t nthreads) {
  constexpr uint32_t NR = 1u << (K - B - V);
  constexpr int NP = (1 << V) - 1;
  uint64_t *base = pw + (NR - 1);
  for (uint32_t r = (tid + nthreads - first) % nthreads; r < NR; r += nthreads) {
    uint64_t sp[NP + 1];
    sp[1] = twiddle(tabs, inv, (H << (K - B - 1)) + (r << (V - 1)));
#pragma unroll
    for (int j = 2; j <= NP; j++) sp[j] = (j & 1) ? gl::mul(sp[j - 1], sp[1]) : gl::sqr(sp[j / 2]);
#pragma unroll
    for (int j = 1; j <= NP; j++) base[r * NP + j - 1] = sp[j];
  }
}

// The power table of tile position H (window bits above the window, group
// prefix included) for the forward (inv = 0) or inverse (inv = 1) twiddles,
// for the rounds of partition PART (PartShape).  The layout rule (a round's
// entries after the NR - 1 of the rounds above it) holds for either.
template <int K, int RI = 0, int PART = 0>
__device__ __forceinline__ void fill_powers(uint64_t *pw, const DevTables &tabs, uint32_t inv, uint32_t H,
                                            uint32_t tid, uint32_t nthreads, uint32_t first = 0) {
  using S = typename PartShape<K, RI, PART>::type;
  if constexpr (RI < S::NR) {
    fill_round_powers<K, S::B, S::V>(pw, tabs, inv, H, first % nthreads, tid, nthreads);
    fill_powers<K, RI + 1, PART>(pw, tabs, inv, H, tid, nthreads, first + (1u << (K - S::B - S::V)));
  }
}

// Butterflies by the constant twiddle 2^E (E < 192).  DIT: the product is
// reduced to [0, p), so the sum and difference need one correction each;
// with E = 0 b itself is reduced first unless it is known canonical (BCAN):
// 6 + 8 instructions against 16 for the add and subtract of two arbitrary
// operands.
template <int E, bool BCAN = false> __device__ __forceinline__ void cdit(uint64_t &a, uint64_t &b) {
  const uint64_t a0 = a;
  if constexpr (E == 0 && BCAN) {
    a = gl::add_bc(a0, b);
    b = gl::sub_bc(a0, b);
  } else if constexpr (E == 0) {
    const uint64_t m = gl::canon(b);
    a = gl::add_bc(a0, m);
    b = gl::sub_bc(a0, m);
  } else if constexpr (E < 96) {
    const uint64_t m = gl::mul_pow2<E, true>(b);
    a = gl::add_bc(a0, m);
    b = gl::sub_bc(a0, m);
  } else {
    const uint64_t m = gl::mul_pow2<E - 96, true>(b);
    a = gl::sub_bc(a0, m);
    b = gl::add_bc(a0, m);
  }
}

// One stage (pair bit QQ of a V-bit round) of the R = 0 network on
// x[OFF .. OFF + 2^V), Cooley-Tukey butterflies (twiddle, then sum and
// difference).  DIT network: stages top bit first, the pair's twiddle is T[u]
// of the round bits u above QQ.  DIF network: stages bottom bit first, twiddle
// w_{2^(QQ+1)}^(-+j) of the round bits j below QQ (ct_tw_exp).  The DIF
// network, the stage-by-stage inverse of the DIT one with the other table,
// is 2^V N_DIT^-1 = DFT(w^-+1) composed with the bit-reversal of its input,
// and the in-place Cooley-Tukey iteration computes exactly that map on the
// same registers; its butterflies (canonical shift product, one correction per
// add and subtract) cost fewer instructions than sum-then-twiddle ones.
// BCAN: the stage's second operands are canonical.
template <bool DIF, bool INV, int V, int OFF, int QQ, bool BCAN, int J0 = 0>
__device__ __forceinline__ void cstage(uint64_t (&x)[16]) {
  if constexpr (J0 < (1 << V)) {
    if constexpr (!(J0 & (1 << QQ))) {
      constexpr int E = DIF ? ct_tw_exp(INV, QQ, J0 & ((1 << QQ) - 1)) : small_tw_exp(INV, J0 >> (QQ + 1));
      cdit<E, BCAN>(x[OFF + J0], x[OFF + (J0 | (1 << QQ))]);
    }
    cstage<DIF, INV, V, OFF, QQ, BCAN, J0 + 1>(x);
  }
}

// The R = 0 network of a V-bit round: DIT top bit first, DIF bottom bit first.
// Either way the first stage's twiddles are all 1: DIT rounds enter with their
// upper half canonical (dit_prepare), DIF rounds reduce their odd elements
// here, so that stage takes one carry correction per add and subtract.
template <bool DIF, bool INV, int V, int OFF, int S = 0>
__device__ __forceinline__ void cnet(uint64_t (&x)[16]) {
  if constexpr (DIF && S == 0) {
#pragma unroll
    for (int j = 1; j < (1 << V); j += 2) x[OFF + j] = gl::canon(x[OFF + j]);
  }
  if constexpr (S < V) {
    cstage<DIF, INV, V, OFF, DIF ? S : V - 1 - S, S == 0>(x);
    cnet<DIF, INV, V, OFF, S + 1>(x);
  }
}

// x[OFF + j] *= pp[j - 1] for j = 1 .. 2^V - 1 (independent products: the
// multiply-add chain form, gl::mul_chain).
template <int V, int OFF>
__device__ __forceinline__ void mul_powers(uint64_t (&x)[16], const uint64_t *pp) {
#pragma unroll
  for (int j = 1; j < (1 << V); j++) x[OFF + j] = gl::mul_chain(x[OFF + j], pp[j - 1]);
}

// Entry of a DIT round: with scale, x[OFF + j] *= pp[j - 1] (the upper half
// reduced to [0, p)); without, the upper half is only reduced.  Either way the
// first stage's second operands are canonical (see cnet).
template <int V, int OFF>
__device__ __forceinline__ void dit_prepare(uint64_t (&x)[16], const uint64_t *pp, bool scale) {
  constexpr int H = 1 << (V - 1);
  if (scale) {
#pragma unroll
    for (int j = 1; j < H; j++) x[OFF + j] = gl::mul_chain(x[OFF + j], pp[j - 1]);
#pragma unroll
    for (int j = H; j < 2 * H; j++) x[OFF + j] = gl::mul_chain_canon(x[OFF + j], pp[j - 1]);
  } else {
#pragma unroll
    for (int j = H; j < 2 * H; j++) x[OFF + j] = gl::canon(x[OFF + j]);
  }
}

// One round of V bits at a compile-time offset B on every group of the thread.
template <int K, int C, bool DIF, bool INV, int B, int V, int Q = 0>
__device__ __forceinline__ void compute_groups(uint64_t (&x)[16], const uint64_t *pw, uint32_t tid,
                                               uint32_t nthreads) {
  constexpr int NV = 1 << V, NG = 16 / NV;
  if constexpr (Q < NG) {
    uint32_t w;
    group_base<K, C, B, V>(tid + nthreads * Q, w);
    const uint64_t *pp = pw + ((1u << (K - B - V)) - 1) + (NV - 1) * (w >> (B + V));
    if constexpr (!DIF) dit_prepare<V, Q * NV>(x, pp, true);
    cnet<DIF, INV, V, Q * NV>(x);
    if constexpr (DIF) mul_powers<V, Q * NV>(x, pp);
    compute_groups<K, C, DIF, INV, B, V, Q + 1>(x, pw, tid, nthreads);
  }
}

// Rounds [RI, END) through shared memory, each followed by a barrier
// (END = -1: through the last round).  DIF rounds run short-round-first, the
// partition the power table is laid out for.
template <int K, int C, bool DIF, bool INV, bool RAGGED_FIRST, int RI, int END = -1>
__device__ __forceinline__ void rounds_from(uint64_t *tile, const uint64_t *pw, uint32_t tid, uint32_t nthreads) {
  static_assert(!DIF || RAGGED_FIRST || K % 4 == 0 || K < 4, "DIF rounds must take the short round first");
  using S = RoundShape<K, DIF, RAGGED_FIRST, RI>;
  constexpr int STOP = END < 0 ? S::NR : END;
  if constexpr (RI < STOP) {
    uint64_t x[16];
    load_groups<K, C, S::B, S::V>(tile, x, tid, nthreads);
    compute_groups<K, C, DIF, INV, S::B, S::V>(x, pw, tid, nthreads);
    store_groups<K, C, S::B, S::V>(tile, x, tid, nthreads);
    __syncthreads();
    rounds_from<K, C, DIF, INV, RAGGED_FIRST, RI + 1, END>(tile, pw, tid, nthreads);
  }
}

// ---------------------------------------------------------------- full rounds at a runtime bit offset
// A full round holds 4 window bits [B, B + 4) of one group per thread.  The
// network below is written once per direction and reused for every full
// round of a pass (looped with `#pragma unroll 1`), which keeps a kernel to one
// copy of the register network instead of one per round.

// Tile index of element 0 of group gi (runs of C fastest) and its window value w.
template <int K, int C>
__device__ __forceinline__ uint32_t gbase16(uint32_t gi, uint32_t B, uint32_t &w) {
  const uint32_t lc = gi % C;
  const uint32_t rest = gi / C;
  const uint32_t g = rest >> (K - 4);
  const uint32_t wo = rest & ((1u << (K - 4)) - 1);
  w = (wo & ((1u << B) - 1)) | ((wo >> B) << (B + 4));
  return ((g << K) | w) * C + lc;
}

// Padded tile slots of the 16 elements of a group: element j sits at tile
// index eb + j * S, S = C << B.
__device__ __forceinline__ void slots16(uint32_t eb, uint32_t S, uint32_t (&a)[16]) {
  if (S >= 16) { // S is a multiple of 16: the padding advances by S / 16 per element
    const uint32_t p0 = pad16(eb), s17 = S + (S >> 4);
#pragma unroll
    for (int j = 0; j < 16; j++) a[j] = p0 + (uint32_t)j * s17;
  } else {
#pragma unroll
    for (int j = 0; j < 16; j++) a[j] = pad16(eb + (uint32_t)j * S);
  }
}

// A full round on x[16] (element j at window w | j << B).  scale = false skips
// the multiplications by s^j, for a caller that knows s = 1 (R = 0) or has
// folded s^j into its own scaling.
template <int K, bool DIF, bool INV>
__device__ __forceinline__ void net16(uint64_t (&x)[16], const uint64_t *pw, uint32_t w, uint32_t B, bool scale) {
  const uint64_t *pp = pw + ((1u << (K - 4 - B)) - 1) + 15 * (w >> (B + 4));
  if constexpr (!DIF) dit_prepare<4, 0>(x, pp, scale);
  cnet<DIF, INV, 4, 0>(x);
  if (DIF && scale) mul_powers<4, 0>(x, pp);
}

// Full rounds at bit offsets B0, B0 + dB, ... (count rounds) through shared
// memory, each followed by a barrier.  One thread per group.
template <int K, int C, bool DIF, bool INV>
__device__ __forceinline__ void full_rounds(uint64_t *tile, const uint64_t *pw, int B0, int dB, int count,
                                            uint32_t tid) {
#pragma unroll 1
  for (int r = 0; r < count; r++) {
    const uint32_t B = (uint32_t)(B0 + r * dB);
    uint32_t w;
    const uint32_t eb = gbase16<K, C>(tid, B, w);
    uint32_t a[16];
    slots16(eb, (uint32_t)C << B, a);
    uint64_t x[16];
#pragma unroll
    for (int j = 0; j < 16; j++) x[j] = tile[a[j]];
    net16<K, DIF, INV>(x, pw, w, B, true);
#pragma unroll
    for (int j = 0; j < 16; j++) tile[a[j]] = x[j];
    __syncthreads();
  }
}

template <int C> struct LogC {
  static constexpr int v = C == 1 ? 0 : C == 2 ? 1 : C == 4 ? 2 : 3;
};

// Tile geometry shared by the pass kernels: decodes blockIdx into the tile
// position and the column range of this CTA.
struct TileGeom {
  uint32_t H;        // bits above the window (within the log_n-bit index)
  uint64_t base_off; // column-relative index of (w = 0, lc = 0)
  uint32_t group;    // column group
  uint32_t col_begin, col_end;
};

template <int K, int C>
__device__ __forceinline__ TileGeom tile_geom(const PassParams &p, uint32_t bx, uint32_t by) {
  TileGeom t;
  const uint32_t lblocks_log = p.lb - LogC<C>::v;
  const uint32_t tp = bx;
  t.H = tp >> lblocks_log;
  t.base_off = ((uint64_t)t.H << (p.lb + K)) + ((uint64_t)(tp & ((1u << lblocks_log) - 1)) << LogC<C>::v);
  t.group = by / p.chunks_per_group;
  const uint32_t chunk = by - t.group * p.chunks_per_group;
  t.col_begin = chunk * p.cols_per_cta;
  t.col_end = min(p.group_cols, t.col_begin + p.cols_per_cta);
  return t;
}

// Element e of the tile (e even) and its neighbour e + 1 are adjacent in
// memory: next lc when C > 1, next w when C == 1 (then the window starts at 0).
template <int K, int C>
__device__ __forceinline__ void tile_elem(uint32_t e, uint32_t &g, uint64_t &off, uint64_t base_off, uint32_t lb) {
  constexpr uint32_t WC = (1u << K) * C;
  g = e / WC;
  const uint32_t rem = e % WC;
  off = base_off + ((uint64_t)(rem / C) << lb) + rem % C;
}

// One CTA's work of a pass: tile position bx, column chunk by (blockIdx of the
// standalone launch, or a work item of the persistent batch kernel).  Needs
// blockDim.x == 2^log_g * 2^K * C / 16 and the shared memory of pass_smem_words.
//
// Round order.  Natural->bit-reversed: the first full round (top 4 window
// bits) is loaded straight from global memory into registers (consecutive
// threads read consecutive addresses), the remaining full rounds run from the
// top down through shared memory, the short round (K mod 4 bits at the bottom)
// last, then the tile is stored with 16-byte stores.  Bit-reversed->natural:
// the tile is loaded with 16-byte loads, the short round runs first at the
// bottom, the full rounds upwards, and the last full round (top 4 bits) is
// stored straight from registers.
//
// Twiddles.  INV selects the inverse table (p.inverse); the power table of the
// tile position sits after the tile.  The window's top round has R = H: for
// H = 0 its s is 1 and its multiplications are skipped, and where the pass
// scales on load (n2b) or on store (b2n) the top round's s^j is folded into
// that scaling's running product.
template <int K, int C, bool B2N, bool INV>
__device__ __forceinline__ void pass_body(const PassParams &p, uint32_t bx, uint32_t by, uint64_t *smem) {
  constexpr int W = 1 << K;
  constexpr int R = K % 4, NF = K / 4;
  const uint32_t G = 1u << p.log_g;
  const uint32_t TILE = G * W * C;
  const uint32_t T = TILE / 16; // == blockDim.x
  uint64_t *tile = smem;
  uint64_t *pw = smem + TILE + TILE / 16;
  const uint32_t tid = threadIdx.x;
  const TileGeom tg = tile_geom<K, C>(p, bx, by);
  const uint32_t Hbig = tg.H + (brev_bits(tg.group, p.log_groups) << (p.log_n - p.lb - K));
  // Bit-reversed -> natural passes fill the power table in their first column
  // group while that group's tile copy is in flight (cp.async); the others
  // fill it here.
  if constexpr (!B2N && NF > 0) fill_powers<K>(pw, p.tabs, INV, Hbig, tid, T);
  const bool top_s = Hbig != 0; // the top round's s differs from 1

  const uint64_t *in = p.in + tg.group * p.group_stride_in;
  uint64_t *out = p.out + tg.group * p.group_stride_out;
  const uint32_t mask_n = (1u << p.log_n) - 1;

  // global offset (within the column) and column of element 0 of a full-round group
  auto group_origin = [&](uint32_t eb, uint32_t c0, uint64_t &off0, uint32_t &col) {
    uint32_t g;
    tile_elem<K, C>(eb, g, off0, tg.base_off, p.lb);
    col = c0 + g;
  };

  // 8-byte cp.async copy of column group c's tile (padded slots are only
  // 8-byte aligned); slots of columns past the chunk are zeroed
  auto copy_tile_async = [&](uint32_t c) {
#pragma unroll 1
    for (int j = 0; j < 8; j++) {
      const uint32_t e = 2 * (tid + T * j);
      uint32_t g;
      uint64_t off;
      tile_elem<K, C>(e, g, off, tg.base_off, p.lb);
      const uint32_t col = c + g;
      if (col < tg.col_end) {
        const uint64_t *src = in + (uint64_t)col * p.stride_in + off;
        cp_async8(tile + pad16(e), src);
        cp_async8(tile + pad16(e) + 1, src + 1);
      } else {
        tile[pad16(e)] = 0;
        tile[pad16(e) + 1] = 0;
      }
    }
    cp_async_commit();
  };
  // bit-reversed -> natural with a plain copy: the last round has the whole
  // tile in registers, so the next group's copy is issued into the tile then
  // and overlaps that round's arithmetic and stores
  bool prefetched = false;

  for (uint32_t c0 = tg.col_begin; c0 < tg.col_end; c0 += G) {
    if constexpr (!B2N && NF > 0) {
      __syncthreads(); // powers ready; previous column group's stores done
      // first full round straight from global memory
      constexpr uint32_t B = K - 4;
      uint32_t w;
      const uint32_t eb = gbase16<K, C>(tid, B, w);
      uint64_t off0;
      uint32_t col;
      group_origin(eb, c0, off0, col);
      uint64_t x[16];
      if (col < tg.col_end) {
        const uint64_t *src = in + (uint64_t)col * p.stride_in + off0;
        const uint64_t step = 1ull << (B + p.lb);
#pragma unroll
        for (int j = 0; j < 16; j++) x[j] = __ldcg(src + j * step);
        if (p.load_scale) { // c^i s^j for i = off0 + j * step: a running product
          uint64_t c_step = coset_power(p.tabs, 0, (uint32_t)step, p.coset_kshift);
          if (top_s) c_step = gl::mul(c_step, pw[0]);
          uint64_t c = coset_power(p.tabs, 0, (uint32_t)off0, p.coset_kshift);
#pragma unroll
          for (int j = 0; j < 16; j++) {
            x[j] = gl::mul(x[j], c);
            if (j + 1 < 16) c = gl::mul(c, c_step);
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < 16; j++) x[j] = 0;
      }
      net16<K, false, INV>(x, pw, w, B, top_s && !p.load_scale);
      uint32_t a[16];
      slots16(eb, (uint32_t)C << B, a);
#pragma unroll
      for (int j = 0; j < 16; j++) tile[a[j]] = x[j];
      __syncthreads();
      full_rounds<K, C, false, INV>(tile, pw, (int)B - 4, -4, NF - 1, tid);
      if constexpr (R > 0) rounds_from<K, C, false, INV, false, NF>(tile, pw, tid, T);
    } else {
      // the tile: a plain copy goes by cp.async (8-byte: padded slots are only
      // 8-byte aligned), completed after the first group's table fill
      const bool async_copy = !p.load_scale;
#pragma unroll
      for (int j = 0; j < 8 && !prefetched; j++) {
        const uint32_t e = 2 * (tid + T * j);
        uint32_t g;
        uint64_t off;
        tile_elem<K, C>(e, g, off, tg.base_off, p.lb);
        const uint32_t col = c0 + g;
        if (col < tg.col_end && async_copy) {
          const uint64_t *src = in + (uint64_t)col * p.stride_in + off;
          cp_async8(tile + pad16(e), src);
          cp_async8(tile + pad16(e) + 1, src + 1);
          continue;
        }
        uint64_t v0 = 0, v1 = 0;
        if (col < tg.col_end) {
          const uint64_t *src = in + (uint64_t)col * p.stride_in + off;
          if (p.vec_in) {
            const ulonglong2 v = __ldcg(reinterpret_cast<const ulonglong2 *>(src));
            v0 = v.x;
            v1 = v.y;
          } else {
            v0 = __ldcg(src);
            v1 = __ldcg(src + 1);
          }
          const uint32_t i0 = (uint32_t)off, i1 = (uint32_t)off + 1; // load_scale
          const uint32_t n0 = B2N ? brev_bits(i0, p.log_n) : i0;
          const uint32_t n1 = B2N ? brev_bits(i1 & mask_n, p.log_n) : i1;
          v0 = gl::mul(v0, coset_power(p.tabs, 0, n0, p.coset_kshift));
          v1 = gl::mul(v1, coset_power(p.tabs, 0, n1, p.coset_kshift));
        }
        tile[pad16(e)] = v0;
        tile[pad16(e) + 1] = v1;
      }
      cp_async_commit();
      if (c0 == tg.col_begin) fill_powers<K>(pw, p.tabs, INV, Hbig, tid, T);
      cp_async_wait<0>();
      __syncthreads();
      if constexpr (!B2N) {
        rounds_from<K, C, false, INV, false, 0>(tile, pw, tid, T); // K < 4: one short round
      } else if constexpr (NF == 0) {
        rounds_from<K, C, true, INV, true, 0>(tile, pw, tid, T);
      } else {
        if constexpr (R > 0) rounds_from<K, C, true, INV, true, 0, 1>(tile, pw, tid, T);
        full_rounds<K, C, true, INV>(tile, pw, R, 4, NF - 1, tid);
        // last full round (top 4 bits) stored straight from registers
        constexpr uint32_t B = K - 4;
        uint32_t w;
        const uint32_t eb = gbase16<K, C>(tid, B, w);
        uint32_t a[16];
        slots16(eb, (uint32_t)C << B, a);
        uint64_t x[16];
#pragma unroll
        for (int j = 0; j < 16; j++) x[j] = tile[a[j]];
        prefetched = async_copy && c0 + G < tg.col_end;
        if (prefetched) {
          __syncthreads(); // every thread holds its values: the tile is free
          copy_tile_async(c0 + G);
        }
        net16<K, true, INV>(x, pw, w, B, top_s && !p.store_scale);
        uint64_t off0;
        uint32_t col;
        group_origin(eb, c0, off0, col);
        if (col < tg.col_end) {
          uint64_t *dst = out + (uint64_t)col * p.stride_out + off0;
          const uint64_t step = 1ull << (B + p.lb);
          if (p.store_scale) { // n^-1 c^-i s^j for the natural index i = off0 + j * step: a running product
            uint64_t s = p.tabs.inv_pow2[p.log_n], s_step = 1;
            if (p.has_coset) {
              s = gl::mul(s, coset_power(p.tabs, 1, (uint32_t)off0, p.coset_kshift));
              s_step = coset_power(p.tabs, 1, (uint32_t)step, p.coset_kshift);
            }
            if (top_s) s_step = p.has_coset ? gl::mul(s_step, pw[0]) : pw[0];
#pragma unroll
            for (int j = 0; j < 16; j++) {
              x[j] = gl::mul(x[j], s);
              if (j + 1 < 16) s = gl::mul(s, s_step);
            }
          }
#pragma unroll
          for (int j = 0; j < 16; j++) __stcg(dst + j * step, p.canon_out ? gl::canon(x[j]) : x[j]);
        }
        if (!prefetched) __syncthreads();
        continue;
      }
    }

#pragma unroll
    for (int j = 0; j < 8; j++) {
      const uint32_t e = 2 * (tid + T * j);
      uint32_t g;
      uint64_t off;
      tile_elem<K, C>(e, g, off, tg.base_off, p.lb);
      const uint32_t col = c0 + g;
      if (col >= tg.col_end) continue;
      uint64_t v0 = tile[pad16(e)], v1 = tile[pad16(e) + 1];
      if (p.store_scale) {
        const uint32_t i0 = (uint32_t)off, i1 = (uint32_t)off + 1;
        const uint32_t n0 = B2N ? i0 : brev_bits(i0, p.log_n);
        const uint32_t n1 = B2N ? i1 : brev_bits(i1 & mask_n, p.log_n);
        const uint64_t s = p.tabs.inv_pow2[p.log_n];
        if (p.has_coset) {
          v0 = gl::mul(v0, gl::mul(s, coset_power(p.tabs, 1, n0, p.coset_kshift)));
          v1 = gl::mul(v1, gl::mul(s, coset_power(p.tabs, 1, n1, p.coset_kshift)));
        } else {
          v0 = gl::mul(v0, s);
          v1 = gl::mul(v1, s);
        }
      }
      if (p.canon_out) {
        v0 = gl::canon(v0);
        v1 = gl::canon(v1);
      }
      uint64_t *dst = out + (uint64_t)col * p.stride_out + off;
      if (p.vec_out) {
        *reinterpret_cast<ulonglong2 *>(dst) = make_ulonglong2(v0, v1);
      } else {
        dst[0] = v0;
        dst[1] = v1;
      }
    }
    __syncthreads();
  }
}

// Shared memory (u64 words) of pass_body for a tile of `tile` elements.
__host__ __device__ constexpr uint32_t pass_smem_words(uint32_t tile, int K) { return tile + tile / 16 + (1u << K); }

// One kernel per twiddle direction (INV == p.inverse, chosen on the host): a
// kernel carrying both bodies behind a branch on p.inverse measured 4-10 us
// slower per small launch in its second body.  MINB > 0 compiles the kernel for
// MINB resident CTAs per SM instead of the default (the autotuner's occupancy
// knob).
template <int K, int C, bool B2N, bool INV, int MINB = 0>
__global__ void __launch_bounds__(256, MINB ? MINB : ((B2N && K >= 9) ? BC_PASS_MIN_BLOCKS_B2N : BC_PASS_MIN_BLOCKS))
    ntt_pass_kernel(const PassParams p) {
  extern __shared__ uint64_t smem[];
  pass_body<K, C, B2N, INV>(p, blockIdx.x, blockIdx.y, smem);
}

} // namespace bc
