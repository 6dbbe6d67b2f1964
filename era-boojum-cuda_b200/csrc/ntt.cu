// ntt.cu -- per-device tables, pass plans, and the plain batched-NTT C ABI.
//
// C-ABI entry points mirror the reference's Rust surface in src/ntt.rs and
// src/context.rs (declared in include/bc_ntt.h with the line each replaces).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/bc_ntt.h"
#include "ntt_host.cuh"
#include "ntt_pass.cuh"

namespace bc {

// ---------------------------------------------------------------- host field
namespace hostf {
constexpr uint64_t P = 0xffffffff00000001ull;
typedef unsigned __int128 u128;
inline uint64_t mul(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a * b) % P); }
inline uint64_t pow(uint64_t b, uint64_t e) {
  uint64_t r = 1;
  b %= P;
  while (e) {
    if (e & 1) r = mul(r, b);
    b = mul(b, b);
    e >>= 1;
  }
  return r;
}
inline uint64_t inv(uint64_t a) { return pow(a, P - 2); }
inline uint64_t root(unsigned log_size) { return pow(pow(7, (P - 1) >> 32), 1ull << (32 - log_size)); }
inline uint32_t brev(uint32_t x, unsigned bits) {
  uint32_t r = 0;
  for (unsigned i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}
} // namespace hostf

// ---------------------------------------------------------------- context
namespace {
constexpr int MAX_DEVICES = 64;
struct DeviceCtx {
  bool live = false;
  uint64_t *block = nullptr;
  uint64_t *top_pw = nullptr; // precomputed top-window power tables
  uint64_t *top_pw_st = nullptr; // the same for the short-round-on-top partition
  DevTables tabs{};
  int sms = 0;
};
DeviceCtx g_ctx[MAX_DEVICES];
std::mutex g_ctx_mutex;

constexpr size_t N_TW_LO = 1u << TW_FINE, N_TW_HI = 1u << (TW_LOG - 1 - TW_FINE);
constexpr size_t N_G_LO = 1u << G_FINE, N_G_HI = 1u << (TW_LOG - G_FINE);
constexpr size_t N_W_LO = 1u << PW_FINE, N_W_HI = 1u << (PW_LOG - PW_FINE);
constexpr size_t TABLE_WORDS = 2 * (N_TW_LO + N_TW_HI + N_G_LO + N_G_HI + N_W_LO + N_W_HI);
constexpr int MAX_TOP_K = 12; // largest window of a pass

void build_host_tables(std::vector<uint64_t> &h, size_t off[12]) {
  using namespace hostf;
  h.assign(TABLE_WORDS, 0);
  size_t o = 0;
  auto seg = [&](int idx, size_t len) {
    off[idx] = o;
    o += len;
  };
  for (int inv_ = 0; inv_ < 2; inv_++) {
    seg(0 + inv_, N_TW_LO);
    seg(2 + inv_, N_TW_HI);
    seg(4 + inv_, N_G_LO);
    seg(6 + inv_, N_G_HI);
    seg(8 + inv_, N_W_LO);
    seg(10 + inv_, N_W_HI);
  }
  for (int inv_ = 0; inv_ < 2; inv_++) {
    const uint64_t w_lo_root = inv_ ? inv(root(TW_FINE + 1)) : root(TW_FINE + 1);
    const uint64_t w_hi_root = inv_ ? inv(root(TW_LOG)) : root(TW_LOG);
    for (uint32_t r = 0; r < N_TW_LO; r++) h[off[0 + inv_] + r] = pow(w_lo_root, brev(r, TW_FINE));
    for (uint32_t r = 0; r < N_TW_HI; r++) h[off[2 + inv_] + r] = pow(w_hi_root, brev(r, TW_LOG - 1 - TW_FINE));
    const uint64_t g = inv_ ? inv(7) : 7;
    uint64_t acc = 1;
    for (size_t i = 0; i < N_G_LO; i++, acc = mul(acc, g)) h[off[4 + inv_] + i] = acc;
    const uint64_t g_step = pow(g, N_G_LO);
    acc = 1;
    for (size_t i = 0; i < N_G_HI; i++, acc = mul(acc, g_step)) h[off[6 + inv_] + i] = acc;
    const uint64_t w = inv_ ? inv(root(PW_LOG)) : root(PW_LOG);
    acc = 1;
    for (size_t i = 0; i < N_W_LO; i++, acc = mul(acc, w)) h[off[8 + inv_] + i] = acc;
    const uint64_t w_step = pow(w, N_W_LO);
    acc = 1;
    for (size_t i = 0; i < N_W_HI; i++, acc = mul(acc, w_step)) h[off[10 + inv_] + i] = acc;
  }
}
} // namespace

int current_device() {
  int d = -1;
  if (cudaGetDevice(&d) != cudaSuccess) return -1;
  return d;
}

const DevTables *device_tables() {
  const int d = current_device();
  if (d < 0 || d >= MAX_DEVICES || !g_ctx[d].live) return nullptr;
  return &g_ctx[d].tabs;
}

int sm_count() {
  const int d = current_device();
  if (d >= 0 && d < MAX_DEVICES && g_ctx[d].sms) return g_ctx[d].sms;
  int n = 148;
  if (d >= 0) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d);
  return n;
}

// Layout of the top-window power tables: per K (1..12) the inverse table, then
// for b = 1 .. TOP_PW_LOG - K the 2^b forward tables, 2^K words each, i.e.
// 2^K (2^(TOP_PW_LOG + 1 - K) - 1) = 2^16 - 2^K words per K.  Table t of a K
// (t = 0 the inverse one, t = 2^b - 1 + k the forward one of coset k of b).
size_t top_pw_base(int K) { return (size_t)(K - 1) * (1u << (TOP_PW_LOG + 1)) - ((1u << K) - 2); }
size_t top_pw_words() { return top_pw_base(MAX_TOP_K + 1); }

// One block per table t of window size K, rounds of partition PART.
template <int K, int PART> __global__ void top_pw_fill_kernel(const DevTables tabs, uint64_t *base) {
  const uint32_t t = blockIdx.x;
  uint32_t inv = 1, H = 0;
  if (t > 0) {
    const uint32_t b = 31 - __clz(t + 1), k = t + 1 - (1u << b);
    inv = 0;
    H = brev_bits(k, b);
  }
  fill_powers<K, 0, PART>(base + (size_t)t * (1u << K), tabs, inv, H, threadIdx.x, blockDim.x);
}

template <int K, int PART> cudaError_t top_pw_fill(const DevTables &tabs, uint64_t *all) {
  const uint32_t tables = (1u << (TOP_PW_LOG + 1 - K)) - 1;
  top_pw_fill_kernel<K, PART><<<tables, 256>>>(tabs, all + top_pw_base(K));
  if constexpr (K < MAX_TOP_K) return top_pw_fill<K + 1, PART>(tabs, all);
  return cudaGetLastError();
}

cudaError_t context_create_current() {
  std::lock_guard<std::mutex> lock(g_ctx_mutex);
  const int d = current_device();
  if (d < 0 || d >= MAX_DEVICES) return cudaErrorInvalidDevice;
  DeviceCtx &c = g_ctx[d];
  if (c.live) return cudaSuccess;
  std::vector<uint64_t> h;
  size_t off[12];
  build_host_tables(h, off);
  // the pass kernels apply T[u], u < 8, as shifts by small_tw_exp
  for (int inv_ = 0; inv_ < 2; inv_++)
    for (int u = 0; u < 8; u++)
      if (h[off[0 + inv_] + u] != hostf::pow(2, (uint64_t)small_tw_exp(inv_ != 0, u))) return cudaErrorInvalidValue;
  cudaError_t e = cudaMalloc(&c.block, TABLE_WORDS * sizeof(uint64_t));
  if (e != cudaSuccess) return e;
  e = cudaMemcpy(c.block, h.data(), TABLE_WORDS * sizeof(uint64_t), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(c.block);
    c.block = nullptr;
    return e;
  }
  for (int inv_ = 0; inv_ < 2; inv_++) {
    c.tabs.tw_lo[inv_] = c.block + off[0 + inv_];
    c.tabs.tw_hi[inv_] = c.block + off[2 + inv_];
    c.tabs.g_lo[inv_] = c.block + off[4 + inv_];
    c.tabs.g_hi[inv_] = c.block + off[6 + inv_];
    c.tabs.w_lo[inv_] = c.block + off[8 + inv_];
    c.tabs.w_hi[inv_] = c.block + off[10 + inv_];
  }
  const uint64_t two_inv = hostf::inv(2);
  uint64_t acc = 1;
  for (int k = 0; k <= TW_LOG; k++, acc = hostf::mul(acc, two_inv)) c.tabs.inv_pow2[k] = acc;
  e = cudaMalloc(&c.top_pw, top_pw_words() * sizeof(uint64_t));
  if (e == cudaSuccess) e = cudaMalloc(&c.top_pw_st, top_pw_words() * sizeof(uint64_t));
  if (e == cudaSuccess) e = top_pw_fill<1, 0>(c.tabs, c.top_pw);
  if (e == cudaSuccess) e = top_pw_fill<1, 1>(c.tabs, c.top_pw_st);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    cudaFree(c.block);
    cudaFree(c.top_pw);
    cudaFree(c.top_pw_st);
    c.block = c.top_pw = c.top_pw_st = nullptr;
    return e;
  }
  cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, d);
  c.live = true;
  return cudaSuccess;
}

const uint64_t *top_power_tables(uint32_t K, uint32_t log_blowup, bool inverse, bool short_top) {
  const int d = current_device();
  if (d < 0 || d >= MAX_DEVICES || !g_ctx[d].live || K < 1 || K > (uint32_t)MAX_TOP_K) return nullptr;
  const uint64_t *base = (short_top ? g_ctx[d].top_pw_st : g_ctx[d].top_pw) + top_pw_base((int)K);
  if (inverse) return base;
  if (log_blowup < 1 || K + log_blowup > (uint32_t)TOP_PW_LOG) return nullptr;
  return base + ((size_t)(1u << log_blowup) - 1) * (1u << K);
}

cudaError_t context_destroy_current() {
  std::lock_guard<std::mutex> lock(g_ctx_mutex);
  const int d = current_device();
  if (d < 0 || d >= MAX_DEVICES) return cudaErrorInvalidDevice;
  DeviceCtx &c = g_ctx[d];
  if (!c.live) return cudaSuccess;
  c.live = false;
  cudaError_t e = cudaFree(c.block);
  const cudaError_t e2 = cudaFree(c.top_pw);
  const cudaError_t e3 = cudaFree(c.top_pw_st);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = e3;
  c.block = c.top_pw = c.top_pw_st = nullptr;
  return e;
}

// ---------------------------------------------------------------- plans
// Default pass plans.  The pass that owns bit 0 takes up to 12 bits (contiguous
// 32 KB tiles); the others use windows whose shared-memory rounds are free of
// bank conflicts: 4, 5, 8 or 9 bits with runs of 8 (64-byte rows), 10 bits with
// runs of 4, 11 bits with runs of 2.
Plan default_plan(uint32_t log_n) {
  Plan pl{};
  auto run_for = [](int K) -> uint8_t { return K <= 9 ? 8 : K == 10 ? 4 : 2; };
  // top window bits for 13..23 (index log_n - 13), then 12 bits at the bottom
  static const uint8_t top2[11] = {5, 5, 5, 8, 8, 9, 9, 9, 9, 10, 11};
  static const uint8_t low2[11] = {8, 9, 10, 8, 9, 9, 10, 11, 12, 12, 12};
  if (log_n <= 12) {
    pl.npasses = 1;
    pl.pass[0] = {(uint8_t)log_n, 1};
  } else if (log_n <= 23) {
    pl.npasses = 2;
    const int k1 = top2[log_n - 13], k2 = low2[log_n - 13];
    pl.pass[0] = {(uint8_t)k1, run_for(k1)};
    pl.pass[1] = {(uint8_t)k2, 1};
  } else {
    // 24..27: two upper windows from {4, 5, 8, 9, 10} over the bits above 12
    static const uint8_t a3[4] = {4, 5, 5, 5}, b3[4] = {8, 8, 9, 10};
    pl.npasses = 3;
    pl.pass[0] = {a3[log_n - 24], run_for(a3[log_n - 24])};
    pl.pass[1] = {b3[log_n - 24], run_for(b3[log_n - 24])};
    pl.pass[2] = {12, 1};
  }
  return pl;
}

static bool shape_supported(int K, int C) {
  if (C == 1) return K >= 1 && K <= 12;
  if (C == 8) return K >= 1 && K <= 9;
  if (C == 4) return K == 10;
  if (C == 2) return K == 11;
  return false;
}

bool plan_valid(const Plan &pl, uint32_t log_n) {
  if (pl.npasses < 1 || pl.npasses > 4) return false;
  uint32_t sum = 0;
  for (int i = 0; i < pl.npasses; i++) {
    const int K = pl.pass[i].K, C = pl.pass[i].C;
    if (!shape_supported(K, C)) return false;
    sum += K;
  }
  if (sum != log_n) return false;
  // window of pass i starts at lb = log_n - (K_0 + ... + K_i); C must fit below it
  uint32_t top = log_n;
  for (int i = 0; i < pl.npasses; i++) {
    const uint32_t lb = top - pl.pass[i].K;
    const int C = pl.pass[i].C;
    if (C == 1 && lb != 0) return false;
    if (C > 1 && (1u << lb) < (uint32_t)C) return false;
    top = lb;
  }
  return true;
}

// ---------------------------------------------------------------- kernels

template <int K, int C, bool B2N, bool INV> static PassKernel kptr() { return ntt_pass_kernel<K, C, B2N, INV>; }

template <bool B2N, bool INV> static PassKernel pick_c1(int K) {
  switch (K) {
  case 1: return kptr<1, 1, B2N, INV>();
  case 2: return kptr<2, 1, B2N, INV>();
  case 3: return kptr<3, 1, B2N, INV>();
  case 4: return kptr<4, 1, B2N, INV>();
  case 5: return kptr<5, 1, B2N, INV>();
  case 6: return kptr<6, 1, B2N, INV>();
  case 7: return kptr<7, 1, B2N, INV>();
  case 8: return kptr<8, 1, B2N, INV>();
  case 9: return kptr<9, 1, B2N, INV>();
  case 10: return kptr<10, 1, B2N, INV>();
  case 11: return kptr<11, 1, B2N, INV>();
  case 12: return kptr<12, 1, B2N, INV>();
  default: return nullptr;
  }
}

template <bool B2N, bool INV> static PassKernel pick_c8(int K) {
  switch (K) {
  case 1: return kptr<1, 8, B2N, INV>();
  case 2: return kptr<2, 8, B2N, INV>();
  case 3: return kptr<3, 8, B2N, INV>();
  case 4: return kptr<4, 8, B2N, INV>();
  case 5: return kptr<5, 8, B2N, INV>();
  case 6: return kptr<6, 8, B2N, INV>();
  case 7: return kptr<7, 8, B2N, INV>();
  case 8: return kptr<8, 8, B2N, INV>();
  case 9: return kptr<9, 8, B2N, INV>();
  default: return nullptr;
  }
}

template <bool B2N, bool INV> static PassKernel pick(int K, int C) {
  if (C == 1) return pick_c1<B2N, INV>(K);
  if (C == 8) return pick_c8<B2N, INV>(K);
  if (C == 4 && K == 10) return kptr<10, 4, B2N, INV>();
  if (C == 2 && K == 11) return kptr<11, 2, B2N, INV>();
  return nullptr;
}

// The other occupancy variant of the C = 1 passes of 9..12 bits: 3 CTAs per SM
// for natural->bit-reversed (default 2), 2 for bit-reversed->natural (default 3).
template <bool B2N, bool INV> static PassKernel pick_occ(int K) {
  constexpr int M = B2N ? BC_PASS_MIN_BLOCKS : BC_PASS_MIN_BLOCKS_B2N;
  switch (K) {
  case 9: return ntt_pass_kernel<9, 1, B2N, INV, M>;
  case 10: return ntt_pass_kernel<10, 1, B2N, INV, M>;
  case 11: return ntt_pass_kernel<11, 1, B2N, INV, M>;
  case 12: return ntt_pass_kernel<12, 1, B2N, INV, M>;
  default: return nullptr;
  }
}

PassKernel pick_pass_kernel(int K, int C, bool b2n, bool inverse, int occ) {
  const int dflt = (b2n && K >= 9) ? BC_PASS_MIN_BLOCKS_B2N : BC_PASS_MIN_BLOCKS;
  if (occ && occ != dflt && C == 1 && K >= 9 && K <= 12) {
    const int other = b2n ? BC_PASS_MIN_BLOCKS : BC_PASS_MIN_BLOCKS_B2N;
    if (occ != other) return nullptr;
    if (b2n) return inverse ? pick_occ<true, true>(K) : pick_occ<true, false>(K);
    return inverse ? pick_occ<false, true>(K) : pick_occ<false, false>(K);
  }
  if (b2n) return inverse ? pick<true, true>(K, C) : pick<true, false>(K, C);
  return inverse ? pick<false, true>(K, C) : pick<false, false>(K, C);
}

static uint32_t log2_ceil(uint64_t x) {
  uint32_t l = 0;
  while ((1ull << l) < x) l++;
  return l;
}

bool ntt_args_ok(uint32_t log_n, uint64_t stride_in, uint64_t stride_out, uint32_t log_ext, uint32_t coset_idx) {
  if (log_n < 1 || log_n > (uint32_t)MAX_LOG_N || log_n + log_ext > (uint32_t)PW_LOG) return false;
  const uint64_t n = 1ull << log_n;
  if (n > stride_in || n > stride_out) return false;
  if (coset_idx > 0 && (log_ext == 0 || coset_idx >= (1u << log_ext))) return false;
  return true;
}

uint32_t plan_lb(const Plan &pl, uint32_t log_n, int i) {
  uint32_t top = log_n;
  for (int j = 0; j <= i; j++) top -= pl.pass[j].K;
  return top;
}

uint32_t choose_log_g(uint32_t wc_log, uint32_t cols) {
  // tile of ~4096 elements, at least 512 (one warp of 16 values each), never
  // more columns per iteration than the batch holds
  uint32_t log_g = wc_log < 12 ? 12 - wc_log : 0;
  const uint32_t lg_cols = log2_ceil(cols);
  if (log_g > lg_cols) log_g = lg_cols;
  if (wc_log + log_g < 9) log_g = 9 - wc_log;
  return log_g;
}

bool build_pass(const PassLaunch &pl, int cols_factor_max, PassParams &p, dim3 &grid, uint32_t &threads,
                size_t &smem_bytes) {
  const DevTables *tabs = device_tables();
  if (!tabs) return false;
  const int K = pl.K, C = pl.C;
  p = PassParams{};
  p.in = pl.in;
  p.out = pl.out;
  p.stride_in = pl.stride_in;
  p.stride_out = pl.stride_out;
  p.group_stride_in = pl.group_stride_in;
  p.group_stride_out = pl.group_stride_out;
  p.group_cols = pl.cols;
  p.log_groups = pl.log_groups;
  p.log_n = pl.log_n;
  p.lb = pl.lb;
  const uint32_t wc_log = (uint32_t)K + log2_ceil((uint32_t)C);
  p.log_g = pl.full_tile ? (wc_log < 12 ? 12 - wc_log : 0) : choose_log_g(wc_log, pl.cols);
  const uint32_t G = 1u << p.log_g;
  const uint64_t tiles_per_col = (1ull << pl.log_n) >> wc_log;
  const uint64_t groups = 1ull << pl.log_groups;
  const uint64_t chunks = (pl.cols + G - 1) / G;
  uint64_t factor = (tiles_per_col * chunks * groups) / ((uint64_t)sm_count() * 8);
  if (factor < 1) factor = 1;
  if (factor > (uint64_t)cols_factor_max) factor = cols_factor_max;
  p.cols_per_cta = G * (uint32_t)factor;
  p.chunks_per_group = (pl.cols + p.cols_per_cta - 1) / p.cols_per_cta;
  p.inverse = pl.inverse;
  p.load_scale = pl.load_scale;
  p.store_scale = pl.store_scale;
  p.canon_out = pl.canon_out;
  p.has_coset = pl.has_coset;
  p.coset_kshift = pl.coset_kshift;
  p.vec_in = ((uintptr_t)p.in % 16 == 0 && p.stride_in % 2 == 0 && p.group_stride_in % 2 == 0) ? 1 : 0;
  p.vec_out = ((uintptr_t)p.out % 16 == 0 && p.stride_out % 2 == 0 && p.group_stride_out % 2 == 0) ? 1 : 0;
  p.tabs = *tabs;
  const uint32_t tile = G << wc_log;
  threads = tile / 16;
  smem_bytes = (size_t)pass_smem_words(tile, K) * sizeof(uint64_t);
  const uint64_t gy = groups * p.chunks_per_group;
  if (tiles_per_col > 0x7fffffffull || gy > 65535) return false;
  grid = dim3((uint32_t)tiles_per_col, (uint32_t)gy);
  return true;
}

cudaError_t launch_pass(const PassLaunch &pl, cudaStream_t stream) {
  if (!device_tables()) return cudaErrorInitializationError;
  if (pl.cols == 0) return cudaSuccess;
  PassParams p;
  dim3 grid;
  uint32_t threads;
  size_t smem;
  if (!build_pass(pl, pl.walk, p, grid, threads, smem)) return cudaErrorInvalidConfiguration;
  PassKernel kern = pick_pass_kernel(pl.K, pl.C, pl.b2n, pl.inverse, pl.occ);
  if (!kern) return cudaErrorInvalidValue;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  kern<<<grid, threads, smem, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_ntt(const Plan &pl, const uint64_t *in, uint64_t *out, uint32_t log_n, uint32_t num_ntts,
                       uint64_t stride_in, uint64_t stride_out, bool bitrev_inputs, bool inverse, uint32_t log_ext,
                       uint32_t coset_idx, cudaStream_t stream) {
  if (!device_tables()) return cudaErrorInitializationError;
  if (num_ntts == 0) return cudaSuccess;
  for (int s = 0; s < pl.npasses; s++) {
    const int i = bitrev_inputs ? pl.npasses - 1 - s : s; // b2n runs the passes bottom-up
    const bool first = s == 0, last = s == pl.npasses - 1;
    PassLaunch q;
    q.K = pl.pass[i].K;
    q.C = pl.pass[i].C;
    q.b2n = bitrev_inputs;
    q.in = first ? in : out;
    q.out = out;
    q.stride_in = first ? stride_in : stride_out;
    q.stride_out = stride_out;
    q.cols = num_ntts;
    q.log_n = log_n;
    q.lb = plan_lb(pl, log_n, i);
    q.inverse = inverse;
    q.load_scale = first && !inverse && log_ext > 0;
    q.store_scale = last && inverse;
    q.canon_out = last;
    q.has_coset = log_ext > 0 ? 1 : 0;
    q.coset_kshift = coset_idx ? coset_idx << (PW_LOG - log_n - log_ext) : 0;
    q.walk = plan_walk(pl);
    q.occ = pl.knobs.occ;
    cudaError_t e = launch_pass(q, stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

} // namespace bc

using namespace bc;

// ---------------------------------------------------------------- C ABI
extern "C" cudaError_t bc_ntt_context_create(uint32_t powers_of_w_coarse_log_count,
                                             uint32_t powers_of_g_coarse_log_count) {
  // The reference splits its tables by these counts (src/context.rs:171-176);
  // the split here is fixed, the arguments keep the reference's bounds check.
  if (powers_of_w_coarse_log_count > 24 || powers_of_g_coarse_log_count > 24) return cudaErrorInvalidValue;
  return context_create_current();
}

extern "C" cudaError_t bc_ntt_context_destroy(void) { return context_destroy_current(); }

extern "C" cudaError_t bc_batch_ntt_internal(const uint64_t *inputs, uint64_t *outputs, uint32_t log_n,
                                             uint32_t num_ntts, uint64_t stride_in, uint64_t stride_out,
                                             bool bitrev_inputs, bool inverse, uint32_t log_extension_degree,
                                             uint32_t coset_index, cudaStream_t stream) {
  if (!ntt_args_ok(log_n, stride_in, stride_out, log_extension_degree, coset_index)) return cudaErrorInvalidValue;
  if (num_ntts && (!inputs || !outputs)) return cudaErrorInvalidValue;
  return launch_ntt(tuned_plan(log_n, 0), inputs, outputs, log_n, num_ntts, stride_in, stride_out, bitrev_inputs,
                    inverse, log_extension_degree, coset_index, stream);
}

extern "C" cudaError_t bc_batch_ntt_out_of_place(const uint64_t *inputs_matrix, size_t inputs_len,
                                                 uint64_t *outputs_matrix, size_t outputs_len, uint32_t log_n,
                                                 uint32_t num_ntts, uint64_t inputs_offset, uint64_t outputs_offset,
                                                 uint64_t stride_in, uint64_t stride_out, bool bitrev_inputs,
                                                 bool inverse, uint32_t log_extension_degree, uint32_t coset_index,
                                                 cudaStream_t stream) {
  if (log_n < 1 || log_n > (uint32_t)MAX_LOG_N) return cudaErrorInvalidValue;
  const uint64_t n = 1ull << log_n;
  if (inputs_offset + n > stride_in || outputs_offset + n > stride_out) return cudaErrorInvalidValue;
  if (inputs_len < (uint64_t)num_ntts * stride_in || outputs_len < (uint64_t)num_ntts * stride_out)
    return cudaErrorInvalidValue;
  if (inputs_matrix == outputs_matrix) return cudaErrorInvalidValue;
  const uint64_t *in = inputs_matrix + inputs_offset;
  uint64_t *out = outputs_matrix + outputs_offset;
  if (in == out) return cudaErrorInvalidValue;
  return bc_batch_ntt_internal(in, out, log_n, num_ntts, stride_in, stride_out, bitrev_inputs, inverse,
                               log_extension_degree, coset_index, stream);
}

extern "C" cudaError_t bc_batch_ntt_in_place(uint64_t *inputs_matrix, size_t len, uint32_t log_n, uint32_t num_ntts,
                                             uint64_t inputs_offset, uint64_t stride, bool bitrev_inputs,
                                             bool inverse, uint32_t log_extension_degree, uint32_t coset_index,
                                             cudaStream_t stream) {
  if (log_n < 1 || log_n > (uint32_t)MAX_LOG_N) return cudaErrorInvalidValue;
  const uint64_t n = 1ull << log_n;
  if (inputs_offset + n > stride) return cudaErrorInvalidValue;
  if (len < (uint64_t)num_ntts * stride) return cudaErrorInvalidValue;
  uint64_t *p = inputs_matrix + inputs_offset;
  return bc_batch_ntt_internal(p, p, log_n, num_ntts, stride, stride, bitrev_inputs, inverse, log_extension_degree,
                               coset_index, stream);
}

extern "C" cudaError_t bc_batch_ntt_with_plan(const uint64_t *inputs, uint64_t *outputs, uint32_t log_n,
                                              uint32_t num_ntts, uint64_t stride_in, uint64_t stride_out,
                                              bool bitrev_inputs, bool inverse, uint32_t log_extension_degree,
                                              uint32_t coset_index, const uint8_t *pass_bits,
                                              const uint8_t *pass_runs, uint32_t npasses, cudaStream_t stream) {
  if (!ntt_args_ok(log_n, stride_in, stride_out, log_extension_degree, coset_index)) return cudaErrorInvalidValue;
  if (npasses < 1 || npasses > 4 || !pass_bits || !pass_runs) return cudaErrorInvalidValue;
  Plan pl{};
  pl.npasses = (int)npasses;
  for (uint32_t i = 0; i < npasses; i++) pl.pass[i] = {pass_bits[i], pass_runs[i]};
  if (!plan_valid(pl, log_n)) return cudaErrorInvalidValue;
  return launch_ntt(pl, inputs, outputs, log_n, num_ntts, stride_in, stride_out, bitrev_inputs, inverse,
                    log_extension_degree, coset_index, stream);
}
