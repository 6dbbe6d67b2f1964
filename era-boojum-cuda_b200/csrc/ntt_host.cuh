// ntt_host.cuh -- host-side pieces shared by the NTT, LDE and batch code.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "tables.cuh"

namespace bc {

// Column groups one standalone pass CTA walks at most (it fills its power
// table once per walk; the walk is shortened to keep >= 8 CTAs per SM).  On
// B200, 16 against 8: forward 12-bit passes 1.8 % faster, 32 no better.  The
// top-window kernel, which copies precomputed tables, walks at most
// BC_TOP_COLS_FACTOR_MAX (16 was 0.5-4 % slower there).
#ifndef BC_COLS_FACTOR_MAX
#define BC_COLS_FACTOR_MAX 16
#endif
#ifndef BC_TOP_COLS_FACTOR_MAX
#define BC_TOP_COLS_FACTOR_MAX 8
#endif

// A pass covers K index bits; C is the run of consecutive low positions a tile
// spans (C = 1 only when the window starts at bit 0, where the tile is one
// contiguous run of 2^K elements).
struct PassCfg {
  uint8_t K;
  uint8_t C;
};

// Launch-shape knobs of a plan, 0 = the built-in choice (autotuned per
// (log_n, log_blowup) by tune.cu):
//   walk      column groups one pass CTA walks at most (BC_COLS_FACTOR_MAX);
//   top_walk  the same for the fused LDE's top-window CTAs (BC_TOP_COLS_FACTOR_MAX);
//   top_mode  its forward power tables: TOP_MODE_RESIDENT / _PREFETCH / _REFILL
//             (see lde.cuh), used where it applies, else the built-in choice;
//   top_dbuf  its tile double-buffering: 1 off, 2 on where the kernel allows it;
//   occ       resident CTAs per SM the low-window passes (C = 1, 9..12 bits)
//             are compiled for: 2 or 3.
struct Knobs {
  uint8_t walk = 0, top_walk = 0, top_mode = 0, top_dbuf = 0, occ = 0;
};
enum : uint8_t { TOP_MODE_RESIDENT = 1, TOP_MODE_PREFETCH = 2, TOP_MODE_REFILL = 3 };

// Passes listed in natural->bit-reversed order: pass[0] owns the top bits,
// pass[npasses-1] owns bits [0, K).  Bit-reversed->natural runs them in the
// opposite order.
struct Plan {
  int npasses;
  PassCfg pass[4];
  Knobs knobs;
};

// Per-device tables; returns nullptr when the context was not created on the
// current device.
const DevTables *device_tables();

// Power tables (ntt_pass.cuh) of top windows, precomputed per device: for each
// K <= 12 the inverse table of H = 0, and for each log_blowup b with
// 2^(K + b) <= 2^TOP_PW_LOG the forward tables of the 2^b cosets
// (H = brev_b(k)), 2^K words each, for the rounds of the pass kernels'
// partition (short round at the bottom) or, short_top, of the top-window
// kernel's direct path (short round at the top).  nullptr when not
// precomputed.
constexpr int TOP_PW_LOG = 15;
const uint64_t *top_power_tables(uint32_t K, uint32_t log_blowup, bool inverse, bool short_top = false);
int current_device();
int sm_count();

Plan default_plan(uint32_t log_n);
// The autotuned plan of the current device for an LDE (log_blowup >= 1) or a
// plain NTT (log_blowup = 0), else default_plan (tune.cu).
Plan tuned_plan(uint32_t log_n, uint32_t log_blowup);
bool plan_valid(const Plan &pl, uint32_t log_n);

// One pass over columns that may come in 2^log_groups groups (see ntt_pass.cuh).
struct PassLaunch {
  int K = 0, C = 1;
  bool b2n = false;
  const uint64_t *in = nullptr;
  uint64_t *out = nullptr;
  uint64_t stride_in = 0, stride_out = 0;
  uint64_t group_stride_in = 0, group_stride_out = 0;
  uint32_t cols = 0; // per group
  uint32_t log_groups = 0;
  uint32_t log_n = 0, lb = 0;
  bool inverse = false, load_scale = false, store_scale = false, canon_out = false;
  uint32_t has_coset = 0, coset_kshift = 0;
  bool full_tile = false; // always 4096-element tiles (256 threads), as the batch kernel runs them
  int walk = BC_COLS_FACTOR_MAX, occ = 0; // column-group walk cap; occupancy variant (Knobs)
};
cudaError_t launch_pass(const PassLaunch &pl, cudaStream_t stream);

struct PassParams;
// Kernel parameters, grid, block size and shared memory of one pass (no launch).
// cols_factor_max bounds how many column groups one CTA walks.
bool build_pass(const PassLaunch &pl, int cols_factor_max, PassParams &p, dim3 &grid, uint32_t &threads,
                size_t &smem_bytes);

typedef void (*PassKernel)(const PassParams);
// The standalone pass kernel for a window shape and twiddle direction (nullptr
// when not instantiated); occ (Knobs::occ) selects the occupancy variant of the
// C = 1 kernels of 9..12 bits, 0 the default one.
PassKernel pick_pass_kernel(int K, int C, bool b2n, bool inverse, int occ = 0);
// Column-group walk caps of a plan's passes and top-window kernel.
inline int plan_walk(const Plan &pl) { return pl.knobs.walk ? pl.knobs.walk : BC_COLS_FACTOR_MAX; }
inline int plan_top_walk(const Plan &pl) { return pl.knobs.top_walk ? pl.knobs.top_walk : BC_TOP_COLS_FACTOR_MAX; }

// Window start (lowest bit) of pass i of a plan, passes listed top-down.
uint32_t plan_lb(const Plan &pl, uint32_t log_n, int i);

// Tile-size policy shared by the pass kernels: columns per tile iteration (log2).
uint32_t choose_log_g(uint32_t wc_log, uint32_t cols);

// Launches every pass of one batched transform; arguments already validated.
cudaError_t launch_ntt(const Plan &pl, const uint64_t *in, uint64_t *out, uint32_t log_n, uint32_t num_ntts,
                       uint64_t stride_in, uint64_t stride_out, bool bitrev_inputs, bool inverse, uint32_t log_ext,
                       uint32_t coset_idx, cudaStream_t stream);

// Argument checks of batch_ntt_internal (src/ntt.rs:192-200) with this
// library's wider limits (log_n <= 27, log_n + log_extension_degree <= 30).
bool ntt_args_ok(uint32_t log_n, uint64_t stride_in, uint64_t stride_out, uint32_t log_ext, uint32_t coset_idx);

} // namespace bc
