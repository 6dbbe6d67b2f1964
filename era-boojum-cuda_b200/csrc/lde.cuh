// lde.cuh -- the fused LDE's top-window kernel body and its step description.
//
// See lde.cu for the algorithm.  The body is shared by the standalone
// lde_top_kernel launch and by the persistent batch kernel (lde_batch.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/bc_ntt.h"
#include "ntt_host.cuh"
#include "ntt_pass.cuh"

namespace bc {

enum : uint32_t { TOP_TABLES_REFILL = 0, TOP_TABLES_RESIDENT = 1, TOP_TABLES_PREFETCH = 2 };

// Word offset of the power tables after `tiles` padded tiles, rounded up to
// an even word so that 16-byte copies into them are aligned.
__host__ __device__ constexpr uint32_t top_tables_offset(uint32_t tile, uint32_t tiles) {
  return (tiles * (tile + tile / 16) + 1) & ~1u;
}

// Copies a 2^K-word power table (16-byte aligned both sides) into shared memory:
// plain 16-byte loads, or cp.async (ASYNC: completion by cp_async_wait).
template <int K, bool ASYNC>
__device__ __forceinline__ void copy_table(uint64_t *dst, const uint64_t *src, uint32_t tid, uint32_t nthreads) {
  for (uint32_t c = tid; c < (1u << (K - 1)); c += nthreads) {
    if constexpr (ASYNC)
      cp_async16(dst + 2 * c, src + 2 * c);
    else
      reinterpret_cast<ulonglong2 *>(dst)[c] = __ldg(reinterpret_cast<const ulonglong2 *>(src) + c);
  }
}

struct LdeTopParams {
  const uint64_t *in; // T (or the evaluations when the plan has one pass)
  uint64_t *out;      // coset block 0
  uint64_t stride_in;
  uint64_t stride_out;
  uint64_t coset_stride;
  uint32_t num_cols;
  uint32_t log_n;
  uint32_t lb; // = log_n - K
  uint32_t log_blowup;
  uint32_t log_g;
  uint32_t cols_per_cta;
  uint32_t canon_out; // single-pass plan: this kernel writes final values
  uint32_t vec_in, vec_out;
  // forward power tables in shared memory: TOP_TABLES_RESIDENT (all cosets',
  // filled once per CTA), TOP_TABLES_PREFETCH (two slots, the next coset's
  // table copied with cp.async from fwd_tables during this coset's rounds) or
  // TOP_TABLES_REFILL (one slot, computed again for every coset)
  uint32_t fwd_mode;
  const uint64_t *fwd_tables; // precomputed forward tables of the cosets (or nullptr)
  const uint64_t *inv_table;  // precomputed inverse table (or nullptr)
  uint32_t dbuf;              // two tiles, the next column group copied (cp.async) during this one;
                              // honoured by the 8-column kernels only (C == 8)
  uint32_t scale_off;         // windows of 4 bits or more: word offset in shared memory of the
                              // threads' scale factors n^-1 g^i (16 per thread, computed once per CTA
                              // and reused by every column group it walks); 0: recomputed per group
  DevTables tabs;
};

// Stores coset k of the tile (16-byte stores; canonical when this kernel ends the LDE).
template <int K, int C>
__device__ __forceinline__ void top_store_t(const LdeTopParams &p, const uint64_t *tile, uint32_t c0, uint32_t col_end,
                                            uint32_t k, uint64_t base_off, uint32_t tid, uint32_t T) {
  uint64_t *out = p.out + (uint64_t)k * p.coset_stride;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const uint32_t e = 2 * (tid + T * j);
    uint32_t g;
    uint64_t off;
    tile_elem<K, C>(e, g, off, base_off, p.lb);
    const uint32_t col = c0 + g;
    if (col >= col_end) continue;
    uint64_t v0 = tile[pad16(e)], v1 = tile[pad16(e) + 1];
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
}
#define top_store top_store_t<K, C>

// top_store_t from the values v[2j], v[2j + 1] of tile elements 2 (tid + T j), + 1.
template <int K, int C>
__device__ __forceinline__ void top_store_regs(const LdeTopParams &p, const uint64_t (&v)[16], uint32_t c0,
                                               uint32_t col_end, uint32_t k, uint64_t base_off, uint32_t tid,
                                               uint32_t T) {
  uint64_t *out = p.out + (uint64_t)k * p.coset_stride;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const uint32_t e = 2 * (tid + T * j);
    uint32_t g;
    uint64_t off;
    tile_elem<K, C>(e, g, off, base_off, p.lb);
    const uint32_t col = c0 + g;
    if (col >= col_end) continue;
    uint64_t v0 = v[2 * j], v1 = v[2 * j + 1];
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
}

// The top-window kernel takes its direct path (top_body_direct) for windows of
// 4 bits or more over runs of C >= 4 low positions (a run fills a 32-byte
// sector, so a warp's 8-byte accesses to one window position are whole
// sectors); its power tables use the short-round-on-top partition
// (ShortTopShape) when K mod 4 != 0.
__host__ __device__ constexpr bool top_direct(int K, int C) { return K >= 4 && C >= 4; }

// The top round of the direct path on every group of the thread: NV = 2^V
// values per group, the same powers for all (R_local = 0).  DIT: with scale,
// x_j *= pp[j - 1] first; DIF: no powers (the inverse top round has s = 1).
template <bool DIF, bool INV, int V, int Q = 0>
__device__ __forceinline__ void top_round_groups(uint64_t (&x)[16], const uint64_t *pp, bool scale) {
  constexpr int NV = 1 << V;
  if constexpr (Q < 16 / NV) {
    if constexpr (!DIF) dit_prepare<V, Q * NV>(x, pp, scale);
    cnet<DIF, INV, V, Q * NV>(x);
    top_round_groups<DIF, INV, V, Q + 1>(x, pp, scale);
  }
}

// Direct path of the top-window kernel (top_direct(K, C)).  The window's
// rounds are the full rounds [0, 4), [4, 8), ... and on top a short round of
// K mod 4 bits (or the last full round when K mod 4 = 0).  The inverse runs
// them bottom-up: the bottom round is loaded straight from global memory into
// registers (thread: 16 consecutive window positions of one low position;
// C consecutive threads: one run), the rounds above go through the tile, and
// the top round stays in registers, where the scale n^-1 g^i is applied.
// Each coset's forward runs top-down from those registers: the top round
// (powers of the coset prefix brev(k); none for k = 0), the rounds below
// through the tile, and the bottom round is stored straight from registers.
// Against top_body this saves the tile's fill, the top_store round trip, two
// barriers per coset and, with a short round, its two shared-memory round
// trips per direction.  The tile region a CTA reads is the one it writes (the
// intermediate T may be coset block 2^b - 1), and every thread loads its
// values before the first barrier of the column group.
template <int K, int C>
__device__ __forceinline__ void top_body_direct(const LdeTopParams &p, uint32_t bx, uint32_t by, uint64_t *smem) {
  constexpr int W = 1 << K;
  constexpr int R = K % 4, NF = K / 4;
  constexpr int NB = R ? NF : NF - 1;   // full rounds below the top round
  constexpr int TB = R ? K - R : K - 4; // the top round's bits [TB, K)
  constexpr int TV = K - TB;
  constexpr int NV = 1 << TV, NG = 16 / NV;
  const uint32_t G = 1u << p.log_g;
  const uint32_t TILE = G * W * C;
  const uint32_t T = TILE / 16;
  uint64_t *const tile = smem;
  uint64_t *pw_inv = smem + top_tables_offset(TILE, 1);
  uint64_t *pw_fwd = pw_inv + PowWords<K>::words;
  constexpr uint32_t PW = PowWords<K>::words;
  const uint32_t tid = threadIdx.x;

  const uint64_t base_off = (uint64_t)bx << LogC<C>::v;
  const uint32_t col_begin = by * p.cols_per_cta;
  const uint32_t col_end = min(p.num_cols, col_begin + p.cols_per_cta);
  const uint32_t nb = 1u << p.log_blowup;
  if (p.inv_table)
    copy_table<K, false>(pw_inv, p.inv_table, tid, T);
  else
    fill_powers<K, 0, 1>(pw_inv, p.tabs, 1, 0, tid, T);
  if (p.fwd_mode == TOP_TABLES_RESIDENT) {
    for (uint32_t k = 0; k < nb; k++) {
      if (p.fwd_tables)
        copy_table<K, false>(pw_fwd + k * PW, p.fwd_tables + k * PW, tid, T);
      else
        fill_powers<K, 0, 1>(pw_fwd + k * PW, p.tabs, 0, brev_bits(k, p.log_blowup), tid, T,
                             (k + 1) * PowWords<K>::tasks);
    }
  } else if (p.fwd_mode == TOP_TABLES_PREFETCH) {
    copy_table<K, true>(pw_fwd, p.fwd_tables, tid, T); // coset 0 of the first column
    cp_async_commit();
  }
  uint32_t step = 0; // cosets done so far: PREFETCH keeps step's table in slot step & 1
  const uint64_t inv_n = p.tabs.inv_pow2[p.log_n];

  // the thread's bottom-round group: window positions w0 + j, low position
  // base_off + lc, column c0 + g0 of each column group
  uint32_t w0;
  const uint32_t eb0 = gbase16<K, C>(tid, 0, w0);
  const uint32_t lc = tid % C, g0 = (tid / C) >> (K - 4);

  // scale n^-1 g^i of the top round's registers: register q NV + j holds
  // window position w_q + (j << TB) (group q = tid + T q of that round)
  auto scale_factors = [&](auto &&use) {
    const uint64_t g_step = g_power(p.tabs, 0, 1u << (p.lb + TB));
    if constexpr (R > 0) {
#pragma unroll
      for (int q = 0; q < NG; q++) {
        uint32_t w;
        group_base<K, C, TB, TV>(tid + T * (uint32_t)q, w);
        uint64_t s = gl::mul(inv_n, g_power(p.tabs, 0, (uint32_t)base_off + lc + (w << p.lb)));
#pragma unroll
        for (int j = 0; j < NV; j++) {
          use(q * NV + j, s);
          if (j + 1 < NV) s = gl::mul(s, g_step);
        }
      }
    } else {
      uint32_t w;
      gbase16<K, C>(tid, TB, w);
      uint64_t s = gl::mul(inv_n, g_power(p.tabs, 0, (uint32_t)base_off + lc + (w << p.lb)));
#pragma unroll
      for (int j = 0; j < 16; j++) {
        use(j, s);
        if (j + 1 < 16) s = gl::mul(s, g_step);
      }
    }
  };
  uint64_t *const scale_tab = p.scale_off ? smem + p.scale_off : nullptr;
  if (scale_tab) scale_factors([&](int j, uint64_t s) { scale_tab[j * T + tid] = s; });
  __syncthreads(); // the tables are complete before the first round reads them

  for (uint32_t c0 = col_begin; c0 < col_end; c0 += G) {
    const uint32_t col = c0 + g0;
    const bool live = col < col_end;
    uint64_t coef[16];
    {
      // inverse, bottom round: straight from global memory
      uint64_t x[16];
      if (live) {
        const uint64_t *src = p.in + (uint64_t)col * p.stride_in + base_off + lc;
#pragma unroll
        for (int j = 0; j < 16; j++) x[j] = __ldcg(src + ((uint64_t)(w0 + (uint32_t)j) << p.lb));
      } else {
#pragma unroll
        for (int j = 0; j < 16; j++) x[j] = 0;
      }
      if constexpr (NB == 0) {
        net16<K, true, true>(x, pw_inv, w0, 0, false); // the bottom round is the top round: s = 1
#pragma unroll
        for (int j = 0; j < 16; j++) coef[j] = x[j];
      } else {
        net16<K, true, true>(x, pw_inv, w0, 0, true);
        uint32_t a[16];
        slots16(eb0, (uint32_t)C, a);
        __syncthreads(); // the previous column group's last round has read the tile
#pragma unroll
        for (int j = 0; j < 16; j++) tile[a[j]] = x[j];
        __syncthreads();
        full_rounds<K, C, true, true>(tile, pw_inv, 4, 4, NB - 1, tid);
        if constexpr (R > 0) {
          load_groups<K, C, TB, TV>(tile, coef, tid, T);
          top_round_groups<true, true, TV>(coef, pw_inv, false);
        } else {
          uint32_t w;
          const uint32_t eb = gbase16<K, C>(tid, TB, w);
          slots16(eb, (uint32_t)C << TB, a);
#pragma unroll
          for (int j = 0; j < 16; j++) coef[j] = tile[a[j]];
          net16<K, true, true>(coef, pw_inv, w, TB, false);
        }
      }
    }
    if (scale_tab) {
#pragma unroll
      for (int j = 0; j < 16; j++) coef[j] = gl::mul_chain(coef[j], scale_tab[j * T + tid]);
    } else {
      scale_factors([&](int j, uint64_t s) { coef[j] = gl::mul(coef[j], s); });
    }

    for (uint32_t k = 0; k < nb; k++) {
      __syncthreads(); // the previous round has read the tile and the powers
      const uint64_t *pwk = pw_fwd;
      if (p.fwd_mode == TOP_TABLES_RESIDENT) {
        pwk = pw_fwd + k * PW;
      } else if (p.fwd_mode == TOP_TABLES_PREFETCH) {
        // the slot of the previous step is free: start the next step's copy,
        // then wait for this step's (all but the newest group)
        pwk = pw_fwd + (step & 1) * PW;
        const bool more = k + 1 < nb || c0 + G < col_end;
        if (more) copy_table<K, true>(pw_fwd + ((step + 1) & 1) * PW, p.fwd_tables + ((k + 1) % nb) * PW, tid, T);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
      } else {
        fill_powers<K, 0, 1>(pw_fwd, p.tabs, 0, brev_bits(k, p.log_blowup), tid, T);
        __syncthreads();
      }
      step++;
      uint64_t x[16];
#pragma unroll
      for (int j = 0; j < 16; j++) x[j] = coef[j];
      if constexpr (NB == 0) {
        net16<K, false, false>(x, pwk, w0, 0, k != 0);
      } else {
        if constexpr (R > 0) {
          top_round_groups<false, false, TV>(x, pwk, k != 0);
          store_groups<K, C, TB, TV>(tile, x, tid, T);
        } else {
          uint32_t w;
          const uint32_t eb = gbase16<K, C>(tid, TB, w);
          net16<K, false, false>(x, pwk, w, TB, k != 0);
          uint32_t a[16];
          slots16(eb, (uint32_t)C << TB, a);
#pragma unroll
          for (int j = 0; j < 16; j++) tile[a[j]] = x[j];
        }
        __syncthreads();
        full_rounds<K, C, false, false>(tile, pwk, 4 * (NB - 1), -4, NB - 1, tid);
        uint32_t a[16];
        slots16(eb0, (uint32_t)C, a);
#pragma unroll
        for (int j = 0; j < 16; j++) x[j] = tile[a[j]];
        net16<K, false, false>(x, pwk, w0, 0, true);
      }
      // forward, bottom round: straight to global memory
      if (live) {
        uint64_t *dst = p.out + (uint64_t)k * p.coset_stride + (uint64_t)col * p.stride_out + base_off + lc;
#pragma unroll
        for (int j = 0; j < 16; j++)
          __stcg(dst + ((uint64_t)(w0 + (uint32_t)j) << p.lb), p.canon_out ? gl::canon(x[j]) : x[j]);
      }
    }
  }
  cp_async_wait<0>(); // nothing in flight past the body
}

// One CTA's work of the top-window kernel: tile position bx (run of low
// positions), column chunk by.  blockDim.x == 2^log_g * 2^K * C / 16.
template <int K, int C>
__device__ __forceinline__ void top_body(const LdeTopParams &p, uint32_t bx, uint32_t by, uint64_t *smem) {
  if constexpr (top_direct(K, C)) {
    top_body_direct<K, C>(p, bx, by, smem);
    return;
  }
  constexpr int W = 1 << K;
  constexpr int R = K % 4, NF = K / 4;
  const uint32_t G = 1u << p.log_g;
  const uint32_t TILE = G * W * C;
  const uint32_t T = TILE / 16;
  // two tiles only in the 8-column kernels (short windows, many column groups
  // per CTA); the wider windows keep one tile and the registers it saves
  const bool dbuf = C == 8 && p.dbuf;
  uint64_t *const tiles[2] = {smem, smem + TILE + TILE / 16};
  // power tables (ntt_pass.cuh): the inverse one, then the forward ones of
  // fwd_mode (see LdeTopParams); 16-byte aligned (copied 16 bytes at a time)
  uint64_t *pw_inv = smem + top_tables_offset(TILE, dbuf ? 2 : 1);
  uint64_t *pw_fwd = pw_inv + PowWords<K>::words;
  constexpr uint32_t PW = PowWords<K>::words;
  const uint32_t tid = threadIdx.x;

  // top window: H = 0, the tile position is the run of low positions
  const uint64_t base_off = (uint64_t)bx << LogC<C>::v;
  const uint32_t col_begin = by * p.cols_per_cta;
  const uint32_t col_end = min(p.num_cols, col_begin + p.cols_per_cta);
  const uint32_t nb = 1u << p.log_blowup;
  if (p.inv_table)
    copy_table<K, false>(pw_inv, p.inv_table, tid, T);
  else
    fill_powers<K>(pw_inv, p.tabs, 1, 0, tid, T);
  if (p.fwd_mode == TOP_TABLES_RESIDENT) {
    for (uint32_t k = 0; k < nb; k++) {
      if (p.fwd_tables)
        copy_table<K, false>(pw_fwd + k * PW, p.fwd_tables + k * PW, tid, T);
      else
        fill_powers<K>(pw_fwd + k * PW, p.tabs, 0, brev_bits(k, p.log_blowup), tid, T, (k + 1) * PowWords<K>::tasks);
    }
  } else if (p.fwd_mode == TOP_TABLES_PREFETCH) {
    copy_table<K, true>(pw_fwd, p.fwd_tables, tid, T); // coset 0 of the first column
    cp_async_commit();
  }
  uint32_t step = 0; // cosets done so far: PREFETCH keeps step's table in slot step & 1
  // the column loop's first barrier orders these fills before any use

  const uint64_t inv_n = p.tabs.inv_pow2[p.log_n];

  // scale n^-1 g^i of the inverse window's output: element j of the thread's
  // group (after the last inverse round) has natural index
  // i0 + (j << (lb + K - 4)), i0 = base_off + tid % C + (w << lb); one factor
  // to start and 15 running products
  auto scale_factors = [&](uint32_t w, auto &&use) {
    const uint32_t i0 = (uint32_t)base_off + tid % C + (w << p.lb);
    const uint64_t g_step = g_power(p.tabs, 0, 1u << (p.lb + K - 4));
    uint64_t s = gl::mul(inv_n, g_power(p.tabs, 0, i0));
#pragma unroll
    for (int j = 0; j < 16; j++) {
      use(j, s);
      if (j + 1 < 16) s = gl::mul(s, g_step);
    }
  };
  uint64_t *const scale_tab = (NF > 0 && p.scale_off) ? smem + p.scale_off : nullptr;
  if constexpr (NF > 0) {
    if (scale_tab) {
      // each thread reads back only its own factors: no barrier needed
      uint32_t w;
      gbase16<K, C>(tid, K - 4, w);
      scale_factors(w, [&](int j, uint64_t s) { scale_tab[j * T + tid] = s; });
    }
  }

  // the tile of column group c by loads and stores
  auto load_tile = [&](uint64_t *dst, uint32_t c) {
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const uint32_t e = 2 * (tid + T * j);
      uint32_t g;
      uint64_t off;
      tile_elem<K, C>(e, g, off, base_off, p.lb);
      const uint32_t col = c + g;
      uint64_t v0 = 0, v1 = 0;
      if (col < col_end) {
        const uint64_t *src = p.in + (uint64_t)col * p.stride_in + off;
        if (p.vec_in) {
          const ulonglong2 v = __ldcg(reinterpret_cast<const ulonglong2 *>(src));
          v0 = v.x;
          v1 = v.y;
        } else {
          v0 = __ldcg(src);
          v1 = __ldcg(src + 1);
        }
      }
      dst[pad16(e)] = v0;
      dst[pad16(e) + 1] = v1;
    }
  };
  // ... or by 8-byte cp.async (padded slots are 8-byte aligned), rolled so
  // that it holds no addresses across the transform it overlaps
  auto load_tile_async = [&](uint64_t *dst, uint32_t c) {
#pragma unroll 1
    for (int j = 0; j < 8; j++) {
      const uint32_t e = 2 * (tid + T * j);
      uint32_t g;
      uint64_t off;
      tile_elem<K, C>(e, g, off, base_off, p.lb);
      const uint32_t col = c + g;
      if (col < col_end) {
        const uint64_t *src = p.in + (uint64_t)col * p.stride_in + off;
        cp_async8(dst + pad16(e), src);
        cp_async8(dst + pad16(e) + 1, src + 1);
      } else {
        dst[pad16(e)] = 0;
        dst[pad16(e) + 1] = 0;
      }
    }
  };
  if (dbuf) {
    load_tile_async(tiles[0], col_begin);
    cp_async_commit();
  }

  bool prefetched = false; // this group's tile was copied during the previous group
  uint32_t it = 0;
  for (uint32_t c0 = col_begin; c0 < col_end; c0 += G, it++) {
    uint64_t *const tile = tiles[dbuf ? (it & 1) : 0];
    if (dbuf) {
      cp_async_wait<0>();
      __syncthreads(); // this group's tile is complete; the other tile is free
      if (c0 + G < col_end) {
        load_tile_async(tiles[(it + 1) & 1], c0 + G);
        cp_async_commit();
      }
    } else if (prefetched) {
      cp_async_wait<0>(); // copied during the previous group's last store
      __syncthreads();
    } else {
      load_tile(tile, c0);
      __syncthreads();
    }
    prefetched = false;

    if constexpr (NF == 0) {
      // window of fewer than 4 bits: one short round each way, in registers
      using S = RoundShape<K, false, false, 0>;
      uint64_t coef[16];
      load_groups<K, C, S::B, S::V>(tile, coef, tid, T);
      compute_groups<K, C, true, true, S::B, S::V>(coef, pw_inv, tid, T);
      constexpr int NV = 1 << S::V, NG = 16 / NV;
#pragma unroll
      for (int q = 0; q < NG; q++) {
        uint32_t w;
        const uint32_t gi = tid + T * q;
        group_base<K, C, S::B, S::V>(gi, w);
        const uint32_t i0 = (uint32_t)base_off + gi % C + (w << p.lb);
        const uint64_t g_step = g_power(p.tabs, 0, 1u << p.lb);
        uint64_t s = gl::mul(inv_n, g_power(p.tabs, 0, i0));
#pragma unroll
        for (int j = 0; j < NV; j++) {
          coef[q * NV + j] = gl::mul(coef[q * NV + j], s);
          if (j + 1 < NV) s = gl::mul(s, g_step);
        }
      }
      for (uint32_t k = 0; k < nb; k++) {
        __syncthreads();
        const uint64_t *pwk = pw_fwd + (p.fwd_mode == TOP_TABLES_RESIDENT ? k * PW : 0);
        if (p.fwd_mode != TOP_TABLES_RESIDENT) { // windows under 4 bits never prefetch
          fill_powers<K>(pw_fwd, p.tabs, 0, brev_bits(k, p.log_blowup), tid, T);
          __syncthreads();
        }
        uint64_t x[16];
#pragma unroll
        for (int j = 0; j < 16; j++) x[j] = coef[j];
        compute_groups<K, C, false, false, S::B, S::V>(x, pwk, tid, T);
        store_groups<K, C, S::B, S::V>(tile, x, tid, T);
        __syncthreads();
        top_store(p, tile, c0, col_end, k, base_off, tid, T);
      }
    } else {
      // inverse stages of the window (bottom-up): the short round first, then the
      // full rounds; the last full round (top 4 bits, R = 0: no powers) stays in
      // registers, scaled
      if constexpr (R > 0) rounds_from<K, C, true, true, true, 0, 1>(tile, pw_inv, tid, T);
      uint32_t w;
      const uint32_t eb = gbase16<K, C>(tid, K - 4, w);
      uint64_t coef[16];
#pragma unroll 1
      for (int r = 0; r < NF; r++) {
        const uint32_t B = (uint32_t)(R + 4 * r);
        uint32_t wr;
        const uint32_t ebr = gbase16<K, C>(tid, B, wr);
        uint32_t a[16];
        slots16(ebr, (uint32_t)C << B, a);
        uint64_t x[16];
#pragma unroll
        for (int j = 0; j < 16; j++) x[j] = tile[a[j]];
        net16<K, true, true>(x, pw_inv, wr, B, r + 1 < NF);
        if (r + 1 < NF) {
#pragma unroll
          for (int j = 0; j < 16; j++) tile[a[j]] = x[j];
          __syncthreads();
        } else {
#pragma unroll
          for (int j = 0; j < 16; j++) coef[j] = x[j];
        }
      }
      // scale n^-1 g^i
      if (scale_tab) {
#pragma unroll
        for (int j = 0; j < 16; j++) coef[j] = gl::mul_chain(coef[j], scale_tab[j * T + tid]);
      } else {
        scale_factors(w, [&](int j, uint64_t s) { coef[j] = gl::mul(coef[j], s); });
      }
      for (uint32_t k = 0; k < nb; k++) {
        __syncthreads(); // previous coset's stores have read the tile (and the powers)
        const uint64_t *pwk = pw_fwd;
        if (p.fwd_mode == TOP_TABLES_RESIDENT) {
          pwk = pw_fwd + k * PW;
        } else if (p.fwd_mode == TOP_TABLES_PREFETCH) {
          // the slot of the previous step is free: start the next step's copy,
          // then wait for this step's (all but the newest group)
          pwk = pw_fwd + (step & 1) * PW;
          const bool more = k + 1 < nb || c0 + G < col_end;
          if (more) copy_table<K, true>(pw_fwd + ((step + 1) & 1) * PW, p.fwd_tables + ((k + 1) % nb) * PW, tid, T);
          cp_async_commit();
          cp_async_wait<1>();
          __syncthreads();
        } else {
          fill_powers<K>(pw_fwd, p.tabs, 0, brev_bits(k, p.log_blowup), tid, T);
          __syncthreads();
        }
        step++;
        // forward stages (top-down): the first full round starts from the registers
        // (its R is the coset prefix brev(k): s = 1 for k = 0)
#pragma unroll 1
        for (int r = 0; r < NF; r++) {
          const uint32_t B = (uint32_t)(K - 4 - 4 * r);
          uint32_t wr;
          const uint32_t ebr = gbase16<K, C>(tid, B, wr);
          uint32_t a[16];
          slots16(ebr, (uint32_t)C << B, a);
          uint64_t x[16];
          if (r == 0) {
#pragma unroll
            for (int j = 0; j < 16; j++) x[j] = coef[j];
          } else {
#pragma unroll
            for (int j = 0; j < 16; j++) x[j] = tile[a[j]];
          }
          net16<K, false, false>(x, pwk, wr, B, r > 0 || k != 0);
#pragma unroll
          for (int j = 0; j < 16; j++) tile[a[j]] = x[j];
          __syncthreads();
        }
        if constexpr (R > 0) rounds_from<K, C, false, false, false, NF>(tile, pwk, tid, T);
        if (k + 1 == nb && !dbuf && p.fwd_mode != TOP_TABLES_PREFETCH && c0 + G < col_end) {
          // last coset: the values go to registers, then the next group's tile
          // is copied into the tile while they are stored (not with prefetched
          // tables, whose next copy the tile's wait would then also wait for:
          // 2^23 x 64 columns, blowup 4 measured 2.4 % slower)
          uint64_t v[16];
#pragma unroll
          for (int j = 0; j < 8; j++) {
            const uint32_t e = 2 * (tid + T * j);
            v[2 * j] = tile[pad16(e)];
            v[2 * j + 1] = tile[pad16(e) + 1];
          }
          __syncthreads();
          load_tile_async(tile, c0 + G);
          cp_async_commit();
          prefetched = true;
          top_store_regs<K, C>(p, v, c0, col_end, k, base_off, tid, T);
        } else {
          top_store(p, tile, c0, col_end, k, base_off, tid, T);
        }
      }
    }
    if (!prefetched) __syncthreads(); // the tile is read; a prefetch already waited for that
  }
  cp_async_wait<0>(); // nothing in flight past the body
}

// Shared memory (u64 words) of top_body: one or two padded tiles, the
// inverse power table and fwd_tables forward ones (or slots).
__host__ __device__ constexpr uint32_t top_smem_words(uint32_t tile, int K, uint32_t fwd_tables, uint32_t tiles = 1) {
  return top_tables_offset(tile, tiles) + (1 + fwd_tables) * (1u << K);
}

// Largest shared memory of a top-window kernel whose forward tables stay
// resident: that of a 4096-element tile of 12 bits with one forward table
// (98 KB), which keeps two CTAs on an SM and fits the persistent kernel.
constexpr uint32_t TOP_RESIDENT_SMEM_MAX = top_smem_words(4096, 12, 1) * 8;

// One kernel of a fused LDE: either a pass (ntt_pass_kernel) or the top-window
// kernel, with its parameters and launch shape.
struct LdeStep {
  bool top = false;
  int K = 0, C = 1;
  bool b2n = false;
  int occ = 0; // occupancy variant of a pass kernel (Knobs::occ)
  PassParams pass{};
  LdeTopParams topp{};
  dim3 grid;
  uint32_t threads = 0;
  size_t smem = 0;
};

// Steps of one fused LDE (inverse passes below the top window, the top-window
// kernel, forward passes below it).  full_tile: 4096-element tiles (256
// threads) for every step; pass_walk / top_walk: column groups a pass CTA /
// a top-window CTA walks at most.  The plan's other knobs (top-window table
// mode, double-buffering, pass occupancy) apply where the kernel allows them.
bool build_lde_steps(const Plan &pl, const uint64_t *in, uint64_t *out, uint32_t log_n, uint32_t num_cols,
                     uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride, uint32_t log_blowup,
                     bool full_tile, int pass_walk, int top_walk, std::vector<LdeStep> &steps);

bool lde_args_ok(uint32_t log_n, uint32_t num_cols, uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride,
                 uint32_t log_blowup);

// Launches one step (pass or top-window kernel) on `stream`.
cudaError_t launch_lde_step(const LdeStep &st, cudaStream_t stream);

// Enqueues a batch of LDE jobs (bc_lde_job, include/bc_ntt.h) as one
// persistent launch with its schedule in caller-owned device scratch, staged
// through caller-owned pinned memory (lde_batch.cu).
cudaError_t batch_enqueue_into(const bc_lde_job *jobs, uint32_t n_jobs, void *dev_scratch, void *host_staging,
                               size_t scratch_bytes, cudaStream_t stream);

// Launches the fused LDE's kernels on `stream`; events (optional): ev[0] is
// recorded before the first kernel and ev[j + 1] after kernel j.
cudaError_t lde_fused(const Plan &pl, const uint64_t *in, uint64_t *out, uint32_t log_n, uint32_t num_cols,
                      uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride, uint32_t log_blowup,
                      cudaStream_t stream, cudaEvent_t *ev = nullptr, uint32_t n_ev = 0);

} // namespace bc
