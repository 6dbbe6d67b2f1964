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
// Tile loads bypass L1 (ld.global.cg): a tile is read once, and in the
// persistent batch kernel another SM may have written it during this launch.
//
// Tile.  A CTA owns one tile position: the bits above the window (H) and a
// run of C consecutive values of the bits below it (l0 .. l0 + C - 1), and
// walks over columns G at a time.  A tile is G x 2^K x C elements, loaded
// with coalesced 16-byte accesses into padded shared memory (one pad word
// every 16 words keeps the strided radix-16 accesses conflict-free), then
// processed in rounds of up to 4 stages held in registers (16 values per
// thread), then stored.  The 2^K - 1 twiddles a tile position needs are
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

// Resident CTAs per SM the pass kernels are compiled for (256 threads each);
// 2 leaves each thread 128 registers, enough for 16 values without spills.
#ifndef BC_PASS_MIN_BLOCKS
#define BC_PASS_MIN_BLOCKS 2
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

__device__ __forceinline__ uint32_t pad16(uint32_t x) { return x + (x >> 4); }

__device__ __forceinline__ uint32_t brev_bits(uint32_t x, uint32_t bits) { return bits ? __brev(x) >> (32 - bits) : 0; }

__device__ __forceinline__ void dit(uint64_t &a, uint64_t &b, uint64_t t) {
  const uint64_t bt = gl::mul(b, t);
  const uint64_t a0 = a;
  a = gl::add(a0, bt);
  b = gl::sub(a0, bt);
}

__device__ __forceinline__ void dif(uint64_t &a, uint64_t &b, uint64_t t) {
  const uint64_t a0 = a;
  a = gl::add(a0, b);
  b = gl::mul(gl::sub(a0, b), t);
}

// ---------------------------------------------------------------- rounds
// A round holds the V window bits [B, B + V) of 16 / 2^V groups per thread in
// registers: x[q * 2^V + j] is element j of the thread's q-th group.

// Which index runs fastest across consecutive threads of a round.  Runs of C
// low positions first keeps a half-warp on 16 distinct banks for every full
// round; a short round on the window's bottom bits with C > 1 instead needs
// the other window bits first (group stride 2^V * C <= 16 words).
template <int C, int B, int V> struct GroupOrder {
  static constexpr bool window_first = (V < 4) && (B == 0) && (C > 1) && ((1 << V) * C <= 16);
};

// Tile index of element 0 of group gi, and its window value w (bits [B, B+V) zero).
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

// Shared-memory twiddle slot of entry i: level L (2^L entries) starts at 2^L
// (entry 0 unused) and one pad word follows every 16, which keeps every
// round's twiddle reads on distinct banks.
__device__ __forceinline__ uint32_t tw_slot(uint32_t i) { return i + (i >> 4); }
template <int K> struct TwSlots {
  static constexpr uint32_t words = (1u << K) + (1u << K) / 16;
};

// Stages of one round.  DIF: bottom bit first, (a+b, (a-b)t); DIT: top bit
// first, (a+bt, a-bt).  Twiddle of window bit qb for upper window part u:
// entry 2^(K-1-qb) + u of the tile's twiddle table.
template <int K, int C, bool DIF, int B, int V>
__device__ __forceinline__ void compute_groups(uint64_t (&x)[16], const uint64_t *tws, uint32_t tid,
                                               uint32_t nthreads) {
  constexpr int NV = 1 << V, NG = 16 / NV;
#pragma unroll
  for (int q = 0; q < NG; q++) {
    uint32_t w;
    group_base<K, C, B, V>(tid + nthreads * q, w);
#pragma unroll
    for (int s = 0; s < V; s++) {
      const int qq = DIF ? s : V - 1 - s;
      const int qb = B + qq;
#pragma unroll
      for (int j0 = 0; j0 < NV; j0++) {
        if (j0 & (1 << qq)) continue;
        const uint32_t u = (w | ((uint32_t)j0 << B)) >> (qb + 1);
        const uint64_t t = tws[tw_slot((1u << (K - 1 - qb)) + u)];
        if (DIF)
          dif(x[q * NV + j0], x[q * NV + (j0 | (1 << qq))], t);
        else
          dit(x[q * NV + j0], x[q * NV + (j0 | (1 << qq))], t);
      }
    }
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

// Rounds [RI, END) through shared memory, each followed by a barrier
// (END = -1: through the last round).
template <int K, int C, bool DIF, bool RAGGED_FIRST, int RI, int END = -1>
__device__ __forceinline__ void rounds_from(uint64_t *tile, const uint64_t *tws, uint32_t tid, uint32_t nthreads) {
  using S = RoundShape<K, DIF, RAGGED_FIRST, RI>;
  constexpr int STOP = END < 0 ? S::NR : END;
  if constexpr (RI < STOP) {
    uint64_t x[16];
    load_groups<K, C, S::B, S::V>(tile, x, tid, nthreads);
    compute_groups<K, C, DIF, S::B, S::V>(x, tws, tid, nthreads);
    store_groups<K, C, S::B, S::V>(tile, x, tid, nthreads);
    __syncthreads();
    rounds_from<K, C, DIF, RAGGED_FIRST, RI + 1, END>(tile, tws, tid, nthreads);
  }
}

// Shared-memory twiddles of one tile position: entry 2^(K-1-q) + u holds
// T[(H << (K-1-q)) + u], q = window bit.
template <int K>
__device__ __forceinline__ void fill_twiddles(uint64_t *tws, const DevTables &tabs, uint32_t inv, uint32_t H,
                                              uint32_t tid, uint32_t nthreads) {
  for (uint32_t t = tid + 1; t < (1u << K); t += nthreads) {
    const uint32_t level = 31 - __clz(t); // = K - 1 - (window bit)
    const uint32_t u = t - (1u << level);
    tws[tw_slot(t)] = twiddle(tabs, inv, (H << level) + u);
  }
}

// ---------------------------------------------------------------- full rounds at a runtime bit offset
// A full round holds 4 window bits [B, B + 4) of one group per thread.  The
// network below is written once per direction and reused for every full
// round of a pass (looped with `#pragma unroll 1`), which keeps a kernel to one
// copy of the 32-butterfly register network instead of one per round.

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

// The four stages of a full round on x[16] (element j at window w | j << B).
// The twiddle of stage bit qb for element pair j0 is entry
// 2^(K-1-qb) + (w >> (qb+1)) + (j0 >> (qq+1)) of the tile's table; the last
// term never carries across a pad word, so one base pointer per stage serves
// all its pairs with constant offsets.
template <int K, bool DIF>
__device__ __forceinline__ void net16(uint64_t (&x)[16], const uint64_t *tws, uint32_t w, uint32_t B) {
  const uint64_t *tp[4];
#pragma unroll
  for (int qq = 0; qq < 4; qq++) {
    const uint32_t qb = B + qq;
    tp[qq] = tws + tw_slot((1u << (K - 1 - qb)) + (w >> (qb + 1)));
  }
#pragma unroll
  for (int st = 0; st < 4; st++) {
    const int qq = DIF ? st : 3 - st;
#pragma unroll
    for (int j0 = 0; j0 < 16; j0++) {
      if (j0 & (1 << qq)) continue;
      const uint64_t t = tp[qq][j0 >> (qq + 1)];
      if (DIF)
        dif(x[j0], x[j0 | (1 << qq)], t);
      else
        dit(x[j0], x[j0 | (1 << qq)], t);
    }
  }
}

// Full rounds at bit offsets B0, B0 + dB, ... (count rounds) through shared
// memory, each followed by a barrier.  One thread per group.
template <int K, int C, bool DIF>
__device__ __forceinline__ void full_rounds(uint64_t *tile, const uint64_t *tws, int B0, int dB, int count,
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
    net16<K, DIF>(x, tws, w, B);
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
template <int K, int C, bool B2N>
__device__ __forceinline__ void pass_body(const PassParams &p, uint32_t bx, uint32_t by, uint64_t *smem) {
  constexpr int W = 1 << K;
  constexpr int R = K % 4, NF = K / 4;
  const uint32_t G = 1u << p.log_g;
  const uint32_t TILE = G * W * C;
  const uint32_t T = TILE / 16; // == blockDim.x
  uint64_t *tile = smem;
  uint64_t *tws = smem + TILE + TILE / 16;
  const uint32_t tid = threadIdx.x;
  const TileGeom tg = tile_geom<K, C>(p, bx, by);
  const uint32_t Hbig = tg.H + (brev_bits(tg.group, p.log_groups) << (p.log_n - p.lb - K));
  fill_twiddles<K>(tws, p.tabs, p.inverse, Hbig, tid, T);

  const uint64_t *in = p.in + tg.group * p.group_stride_in;
  uint64_t *out = p.out + tg.group * p.group_stride_out;
  const uint32_t mask_n = (1u << p.log_n) - 1;

  // global offset (within the column) and column of element 0 of a full-round group
  auto group_origin = [&](uint32_t eb, uint32_t c0, uint64_t &off0, uint32_t &col) {
    uint32_t g;
    tile_elem<K, C>(eb, g, off0, tg.base_off, p.lb);
    col = c0 + g;
  };

  for (uint32_t c0 = tg.col_begin; c0 < tg.col_end; c0 += G) {
    if constexpr (!B2N && NF > 0) {
      __syncthreads(); // twiddles ready; previous column group's stores done
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
        if (p.load_scale) { // c^i for i = off0 + j * step: a running product
          const uint64_t c_step = coset_power(p.tabs, 0, (uint32_t)step, p.coset_kshift);
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
      net16<K, false>(x, tws, w, B);
      uint32_t a[16];
      slots16(eb, (uint32_t)C << B, a);
#pragma unroll
      for (int j = 0; j < 16; j++) tile[a[j]] = x[j];
      __syncthreads();
      full_rounds<K, C, false>(tile, tws, (int)B - 4, -4, NF - 1, tid);
      if constexpr (R > 0) rounds_from<K, C, false, false, NF>(tile, tws, tid, T);
    } else {
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const uint32_t e = 2 * (tid + T * j);
        uint32_t g;
        uint64_t off;
        tile_elem<K, C>(e, g, off, tg.base_off, p.lb);
        const uint32_t col = c0 + g;
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
          if (p.load_scale) {
            const uint32_t i0 = (uint32_t)off, i1 = (uint32_t)off + 1;
            const uint32_t n0 = B2N ? brev_bits(i0, p.log_n) : i0;
            const uint32_t n1 = B2N ? brev_bits(i1 & mask_n, p.log_n) : i1;
            v0 = gl::mul(v0, coset_power(p.tabs, 0, n0, p.coset_kshift));
            v1 = gl::mul(v1, coset_power(p.tabs, 0, n1, p.coset_kshift));
          }
        }
        tile[pad16(e)] = v0;
        tile[pad16(e) + 1] = v1;
      }
      __syncthreads();
      if constexpr (!B2N) {
        rounds_from<K, C, false, false, 0>(tile, tws, tid, T); // K < 4: one short round
      } else if constexpr (NF == 0) {
        rounds_from<K, C, true, true, 0>(tile, tws, tid, T);
      } else {
        if constexpr (R > 0) rounds_from<K, C, true, true, 0, 1>(tile, tws, tid, T);
        full_rounds<K, C, true>(tile, tws, R, 4, NF - 1, tid);
        // last full round (top 4 bits) stored straight from registers
        constexpr uint32_t B = K - 4;
        uint32_t w;
        const uint32_t eb = gbase16<K, C>(tid, B, w);
        uint32_t a[16];
        slots16(eb, (uint32_t)C << B, a);
        uint64_t x[16];
#pragma unroll
        for (int j = 0; j < 16; j++) x[j] = tile[a[j]];
        net16<K, true>(x, tws, w, B);
        uint64_t off0;
        uint32_t col;
        group_origin(eb, c0, off0, col);
        if (col < tg.col_end) {
          uint64_t *dst = out + (uint64_t)col * p.stride_out + off0;
          const uint64_t step = 1ull << (B + p.lb);
          if (p.store_scale) { // n^-1 c^-i for the natural index i = off0 + j * step: a running product
            uint64_t s = p.tabs.inv_pow2[p.log_n], s_step = 1;
            if (p.has_coset) {
              s = gl::mul(s, coset_power(p.tabs, 1, (uint32_t)off0, p.coset_kshift));
              s_step = coset_power(p.tabs, 1, (uint32_t)step, p.coset_kshift);
            }
#pragma unroll
            for (int j = 0; j < 16; j++) {
              x[j] = gl::mul(x[j], s);
              if (j + 1 < 16) s = gl::mul(s, s_step);
            }
          }
#pragma unroll
          for (int j = 0; j < 16; j++) __stcg(dst + j * step, p.canon_out ? gl::canon(x[j]) : x[j]);
        }
        __syncthreads();
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
__host__ __device__ constexpr uint32_t pass_smem_words(uint32_t tile, int K) {
  return tile + tile / 16 + (1u << K) + (1u << K) / 16;
}

template <int K, int C, bool B2N>
__global__ void __launch_bounds__(256, BC_PASS_MIN_BLOCKS) ntt_pass_kernel(const PassParams p) {
  extern __shared__ uint64_t smem[];
  pass_body<K, C, B2N>(p, blockIdx.x, blockIdx.y, smem);
}

} // namespace bc
