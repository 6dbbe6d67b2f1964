// lde.cu -- coset low-degree extension: plain composition and fused kernels.
//
// The reference ships no LDE function; its callers compose one inverse
// transform with one forward transform per coset (src/ntt.rs:527-583 as used
// by benches/ntt.rs:114-116):
//     bit-reversed evaluations on H --iNTT b2n--> natural coefficients a_i
//     --for k < B: n2b with (log_ext = log2 B, coset k)--> bit-reversed
//     evaluations on c_k H, c_k = g * w_{nB}^k.
// bc_lde_plain runs exactly that composition through bc_batch_ntt_internal.
//
// bc_lde_fused computes the same outputs with three kernels per plan:
//   A  the inverse transform's passes below the top window (b2n, in -> T);
//   B  one kernel on the top window: the inverse stages, the scale
//      n^-1 * g^i, then for every coset the forward stages of that window;
//   C  the forward passes below the top window for all cosets at once.
// It rests on one identity: the B cosets together are the domain g * H_{Bn},
// so the B forward transforms are the size-Bn transform of the zero-padded
// sequence g^i a_i, and coset k is its output block brev(k).  Each coset's
// forward transform is therefore the plain size-n transform of g^i a_i with
// the index prefix brev(k) in its twiddles (column groups, ntt_pass.cuh):
// the per-coset factors w_{nB}^{k i} vanish into the twiddles and the scale is
// applied once per element instead of once per element and coset.  T is the
// output block of the last coset, so no scratch memory is used.
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <tuple>

#include "../../include/bc_ntt.h"
#include "lde.cuh"

namespace bc {

template <int K, int C>
__global__ void __launch_bounds__(256, BC_TOP_MIN_BLOCKS) lde_top_kernel(const LdeTopParams p) {
  extern __shared__ uint64_t smem[];
  top_body<K, C>(p, blockIdx.x, blockIdx.y, smem);
}

typedef void (*TopKernel)(const LdeTopParams);
typedef void (*PassKernelT)(const PassParams);

static TopKernel pick_top(int K, int C);

// resident CTAs per SM of lde_top_kernel<K, C> at this block size and dynamic
// shared memory (0 when the kernel or the query is unavailable); cached per
// device and shape, since every fused-LDE call that may pipeline asks
static int top_ctas_per_sm(int K, int C, uint32_t threads, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int, uint32_t, size_t>, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  const auto key = std::make_tuple(dev, K, C, threads, smem);
  {
    std::lock_guard<std::mutex> lock(mu);
    const auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  TopKernel kern = pick_top(K, C);
  if (!kern) return 0;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TOP_RESIDENT_SMEM_MAX) !=
          cudaSuccess)
    return 0;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, (int)threads, smem) != cudaSuccess) return 0;
  std::lock_guard<std::mutex> lock(mu);
  cache[key] = n;
  return n;
}

template <int K, int C> static TopKernel tk() { return lde_top_kernel<K, C>; }

static TopKernel pick_top(int K, int C) {
  if (C == 1) {
    switch (K) {
    case 1: return tk<1, 1>();
    case 2: return tk<2, 1>();
    case 3: return tk<3, 1>();
    case 4: return tk<4, 1>();
    case 5: return tk<5, 1>();
    case 6: return tk<6, 1>();
    case 7: return tk<7, 1>();
    case 8: return tk<8, 1>();
    case 9: return tk<9, 1>();
    case 10: return tk<10, 1>();
    case 11: return tk<11, 1>();
    case 12: return tk<12, 1>();
    default: return nullptr;
    }
  }
  if (C == 8) {
    switch (K) {
    case 1: return tk<1, 8>();
    case 2: return tk<2, 8>();
    case 3: return tk<3, 8>();
    case 4: return tk<4, 8>();
    case 5: return tk<5, 8>();
    case 6: return tk<6, 8>();
    case 7: return tk<7, 8>();
    case 8: return tk<8, 8>();
    case 9: return tk<9, 8>();
    default: return nullptr;
    }
  }
  if (C == 4 && K == 10) return tk<10, 4>();
  if (C == 2 && K == 11) return tk<11, 2>();
  return nullptr;
}

static uint32_t ilog2_ceil(uint64_t x) {
  uint32_t l = 0;
  while ((1ull << l) < x) l++;
  return l;
}

// Layout checks shared by both LDE paths: coset blocks and columns must be
// disjoint windows, either coset-major (block k = cols x stride_out) or
// column-major (each column holds its B cosets at coset_stride apart).
bool lde_args_ok(uint32_t log_n, uint32_t num_cols, uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride,
                 uint32_t log_blowup) {
  if (log_n < 1 || log_blowup < 1 || log_n + log_blowup > (uint32_t)TW_LOG) return false;
  const uint64_t n = 1ull << log_n, B = 1ull << log_blowup;
  if (stride_in < n || stride_out < n || coset_stride < n) return false;
  if (num_cols == 0) return true;
  const bool coset_major = coset_stride >= (uint64_t)(num_cols - 1) * stride_out + n;
  const bool column_major = stride_out >= (B - 1) * coset_stride + n;
  return coset_major || column_major;
}

bool build_lde_steps(const Plan &pl, const uint64_t *in, uint64_t *out, uint32_t log_n, uint32_t num_cols,
                     uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride, uint32_t log_blowup,
                     bool full_tile, int pass_walk, int top_walk, std::vector<LdeStep> &steps) {
  const DevTables *tabs = device_tables();
  if (!tabs) return false;
  steps.clear();
  if (num_cols == 0) return true;
  const uint32_t nb = 1u << log_blowup;
  uint64_t *T = out + (uint64_t)(nb - 1) * coset_stride;
  const int np = pl.npasses;
  // A: inverse passes below the top window, bottom-up: in -> T
  for (int s = 0; s < np - 1; s++) {
    const int i = np - 1 - s;
    PassLaunch q;
    q.K = pl.pass[i].K;
    q.C = pl.pass[i].C;
    q.b2n = true;
    q.in = s == 0 ? in : T;
    q.out = T;
    q.stride_in = s == 0 ? stride_in : stride_out;
    q.stride_out = stride_out;
    q.cols = num_cols;
    q.log_n = log_n;
    q.lb = plan_lb(pl, log_n, i);
    q.inverse = true;
    q.full_tile = full_tile;
    LdeStep st;
    st.K = q.K;
    st.C = q.C;
    st.b2n = true;
    st.occ = pl.knobs.occ;
    if (!build_pass(q, pass_walk, st.pass, st.grid, st.threads, st.smem)) return false;
    steps.push_back(st);
  }
  // B: top window
  {
    const int K = pl.pass[0].K, C = pl.pass[0].C;
    LdeStep st;
    st.top = true;
    st.K = K;
    st.C = C;
    LdeTopParams &p = st.topp;
    p.in = np == 1 ? in : T;
    p.out = out;
    p.stride_in = np == 1 ? stride_in : stride_out;
    p.stride_out = stride_out;
    p.coset_stride = coset_stride;
    p.num_cols = num_cols;
    p.log_n = log_n;
    p.lb = log_n - K;
    p.log_blowup = log_blowup;
    const uint32_t wc_log = (uint32_t)K + ilog2_ceil((uint32_t)C);
    p.log_g = full_tile ? (wc_log < 12 ? 12 - wc_log : 0) : choose_log_g(wc_log, num_cols);
    const uint32_t G = 1u << p.log_g;
    const uint64_t tiles = (1ull << log_n) >> wc_log;
    const uint64_t chunks = (num_cols + G - 1) / G;
    uint64_t factor = (tiles * chunks) / ((uint64_t)sm_count() * 8);
    if (factor < 1) factor = 1;
    if (factor > (uint64_t)top_walk) factor = top_walk;
    p.cols_per_cta = G * (uint32_t)factor;
    p.canon_out = np == 1;
    p.vec_in = ((uintptr_t)p.in % 16 == 0 && p.stride_in % 2 == 0) ? 1 : 0;
    p.vec_out = ((uintptr_t)out % 16 == 0 && stride_out % 2 == 0 && coset_stride % 2 == 0) ? 1 : 0;
    p.tabs = *tabs;
    const uint32_t tile = G << wc_log;
    st.threads = tile / 16;
    const uint32_t nb = 1u << log_blowup;
    // forward power tables: all resident if they fit with two CTAs per SM, else
    // two slots fed ahead by cp.async from the precomputed ones, else refilled
    const bool direct = top_direct(K, C); // top_body_direct: short-round-on-top tables, one tile
    p.fwd_tables = top_power_tables((uint32_t)K, log_blowup, false, direct);
    p.inv_table = top_power_tables((uint32_t)K, log_blowup, true, direct);
    auto fits = [&](uint32_t tables) {
      return (size_t)top_smem_words(tile, K, tables) * sizeof(uint64_t) <= TOP_RESIDENT_SMEM_MAX;
    };
    uint32_t slots = 1;
    const bool can_prefetch = p.fwd_tables && K >= 4 && fits(2);
    const uint8_t mode = pl.knobs.top_mode;
    if (mode == TOP_MODE_REFILL) {
      p.fwd_mode = TOP_TABLES_REFILL;
    } else if (mode == TOP_MODE_PREFETCH && can_prefetch) {
      p.fwd_mode = TOP_TABLES_PREFETCH;
      slots = 2;
    } else if (fits(nb)) {
      p.fwd_mode = TOP_TABLES_RESIDENT;
      slots = nb;
    } else if (can_prefetch) {
      p.fwd_mode = TOP_TABLES_PREFETCH;
      slots = 2;
    } else {
      p.fwd_mode = TOP_TABLES_REFILL;
    }
    // two tiles (the next column group copied during this one) in the 8-column
    // kernels with short transforms per tile (window bits x cosets <= 16: on
    // B200 2^16 x 4096 columns, blowup 2, gains 13 %; 2^19 x 512, blowup 4,
    // loses 2 %), when they fit and cost no resident CTA per SM
    const size_t smem1 = (size_t)top_smem_words(tile, K, slots, 1) * sizeof(uint64_t);
    const size_t smem2 = (size_t)top_smem_words(tile, K, slots, 2) * sizeof(uint64_t);
    p.dbuf = 0;
    const bool dbuf_allowed = !direct && C == 8 && p.fwd_mode != TOP_TABLES_PREFETCH && p.cols_per_cta > G &&
                              smem2 <= TOP_RESIDENT_SMEM_MAX;
    if (pl.knobs.top_dbuf == 2) {
      p.dbuf = dbuf_allowed ? 1 : 0;
    } else if (pl.knobs.top_dbuf == 0 && dbuf_allowed && (uint32_t)K * nb <= 16) {
      const int n2 = top_ctas_per_sm(K, C, st.threads, smem2);
      p.dbuf = (n2 > 0 && n2 >= top_ctas_per_sm(K, C, st.threads, smem1)) ? 1 : 0;
    }
    st.smem = p.dbuf ? smem2 : smem1;
    // the scale factors once per CTA in shared memory, when the CTA walks more
    // than one column group and the table costs no resident CTA per SM
    p.scale_off = 0;
    if (K >= 4 && p.cols_per_cta > G) {
      const size_t with = st.smem + (size_t)tile * sizeof(uint64_t);
      if (with <= TOP_RESIDENT_SMEM_MAX &&
          top_ctas_per_sm(K, C, st.threads, with) >= top_ctas_per_sm(K, C, st.threads, st.smem)) {
        p.scale_off = (uint32_t)(st.smem / sizeof(uint64_t));
        st.smem = with;
      }
    }
    const uint64_t gy = (num_cols + p.cols_per_cta - 1) / p.cols_per_cta;
    if (gy > 65535 || tiles > 0x7fffffffull) return false;
    st.grid = dim3((uint32_t)tiles, (uint32_t)gy);
    steps.push_back(st);
  }
  // C: forward passes below the top window for all cosets (column groups with prefix brev(k))
  for (int i = 1; i < np; i++) {
    PassLaunch q;
    q.K = pl.pass[i].K;
    q.C = pl.pass[i].C;
    q.b2n = false;
    q.in = out;
    q.out = out;
    q.stride_in = stride_out;
    q.stride_out = stride_out;
    q.group_stride_in = coset_stride;
    q.group_stride_out = coset_stride;
    q.cols = num_cols;
    q.log_groups = log_blowup;
    q.log_n = log_n;
    q.lb = plan_lb(pl, log_n, i);
    q.inverse = false;
    q.canon_out = i == np - 1;
    q.full_tile = full_tile;
    LdeStep st;
    st.K = q.K;
    st.C = q.C;
    st.occ = pl.knobs.occ;
    if (!build_pass(q, pass_walk, st.pass, st.grid, st.threads, st.smem)) return false;
    steps.push_back(st);
  }
  return true;
}

cudaError_t launch_lde_step(const LdeStep &st, cudaStream_t stream) {
  if (st.top) {
    TopKernel kern = pick_top(st.K, st.C);
    if (!kern) return cudaErrorInvalidValue;
    if (st.smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)st.smem);
      if (e != cudaSuccess) return e;
    }
    kern<<<st.grid, st.threads, st.smem, stream>>>(st.topp);
  } else {
    PassKernel kern = pick_pass_kernel(st.K, st.C, st.b2n, st.pass.inverse != 0, st.occ);
    if (!kern) return cudaErrorInvalidValue;
    if (st.smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)st.smem);
      if (e != cudaSuccess) return e;
    }
    kern<<<st.grid, st.threads, st.smem, stream>>>(st.pass);
  }
  return cudaGetLastError();
}

cudaError_t lde_fused(const Plan &pl, const uint64_t *in, uint64_t *out, uint32_t log_n, uint32_t num_cols,
                      uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride, uint32_t log_blowup,
                      cudaStream_t stream, cudaEvent_t *ev, uint32_t n_ev) {
  if (!device_tables()) return cudaErrorInitializationError;
  if (num_cols == 0) return cudaSuccess;
  std::vector<LdeStep> steps;
  if (!build_lde_steps(pl, in, out, log_n, num_cols, stride_in, stride_out, coset_stride, log_blowup, false,
                       plan_walk(pl), plan_top_walk(pl), steps))
    return cudaErrorInvalidConfiguration;
  uint32_t ev_used = 0;
  if (ev_used < n_ev) cudaEventRecord(ev[ev_used++], stream);
  for (const LdeStep &st : steps) {
    cudaError_t e = launch_lde_step(st, stream);
    if (e != cudaSuccess) return e;
    if (ev_used < n_ev) cudaEventRecord(ev[ev_used++], stream);
  }
  return cudaSuccess;
}

} // namespace bc

using namespace bc;

extern "C" cudaError_t bc_lde_plain(const uint64_t *evals_bitrev, uint64_t *out, uint32_t log_n, uint32_t num_cols,
                                    uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride,
                                    uint32_t log_blowup, cudaStream_t stream) {
  if (!lde_args_ok(log_n, num_cols, stride_in, stride_out, coset_stride, log_blowup)) return cudaErrorInvalidValue;
  if (num_cols && (!evals_bitrev || !out)) return cudaErrorInvalidValue;
  const uint32_t nb = 1u << log_blowup;
  uint64_t *coef = out + (uint64_t)(nb - 1) * coset_stride;
  cudaError_t e =
      bc_batch_ntt_internal(evals_bitrev, coef, log_n, num_cols, stride_in, stride_out, true, true, 0, 0, stream);
  for (uint32_t k = 0; e == cudaSuccess && k < nb; k++)
    e = bc_batch_ntt_internal(coef, out + (uint64_t)k * coset_stride, log_n, num_cols, stride_out, stride_out, false,
                              false, log_blowup, k, stream);
  return e;
}

extern "C" cudaError_t bc_lde_fused(const uint64_t *evals_bitrev, uint64_t *out, uint32_t log_n, uint32_t num_cols,
                                    uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride,
                                    uint32_t log_blowup, cudaStream_t stream) {
  if (!lde_args_ok(log_n, num_cols, stride_in, stride_out, coset_stride, log_blowup)) return cudaErrorInvalidValue;
  if (num_cols && (!evals_bitrev || !out)) return cudaErrorInvalidValue;
  return lde_fused(tuned_plan(log_n, log_blowup), evals_bitrev, out, log_n, num_cols, stride_in, stride_out, coset_stride,
                   log_blowup, stream);
}

extern "C" cudaError_t bc_lde_fused_profiled(const uint64_t *evals_bitrev, uint64_t *out, uint32_t log_n,
                                             uint32_t num_cols, uint64_t stride_in, uint64_t stride_out,
                                             uint64_t coset_stride, uint32_t log_blowup, cudaStream_t stream,
                                             cudaEvent_t *events, uint32_t num_events, uint32_t *num_kernels) {
  if (!lde_args_ok(log_n, num_cols, stride_in, stride_out, coset_stride, log_blowup)) return cudaErrorInvalidValue;
  if (num_cols && (!evals_bitrev || !out)) return cudaErrorInvalidValue;
  const Plan pl = tuned_plan(log_n, log_blowup);
  if (num_kernels) *num_kernels = (uint32_t)(2 * pl.npasses - 1);
  return lde_fused(pl, evals_bitrev, out, log_n, num_cols, stride_in, stride_out, coset_stride, log_blowup, stream,
                   events, num_events);
}
