// tune.cu -- per-device plan table and the autotuner.
//
// The reference fixes its kernel plans in a table (PLANS, src/ntt.rs:74-169).
// Here plans are data: a per-device table maps (log_n, log_blowup) to a pass
// plan -- how the index bits split into windows (the radix split), which run
// of consecutive positions each window's tiles span (the tile shape), and so
// how many stages the fused LDE's top-window kernel carries (the stage fusion:
// its window is pass 0).  bc_autotune times every candidate on the current
// device and stores the fastest (near-ties go to the fewest passes, then the
// smallest top window), then tunes the plan's launch knobs (ntt_host.cuh
// Knobs: column walks, top-window table mode and double-buffering, pass
// occupancy) one at a time on that window split, keeping a value only when it
// is more than 1 % faster; LDE and NTT entry points consult the table and fall back to the built-in
// plan.  Candidates use only window shapes that
// every kernel (the persistent batch kernel included) can run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/bc_ntt.h"
#include "lde.cuh"

namespace bc {

namespace {
constexpr int TUNE_MAX_DEVICES = 64;
std::map<uint32_t, Plan> g_table[TUNE_MAX_DEVICES];
std::mutex g_table_mutex;

uint32_t key(uint32_t log_n, uint32_t log_blowup) { return (log_blowup << 8) | log_n; }

struct Shape {
  uint8_t K, C;
};
const Shape TOP_SHAPES[] = {{4, 8}, {5, 8}, {8, 8}, {9, 8}, {10, 4}, {11, 2}};
const Shape MID_SHAPES[] = {{8, 8}, {9, 8}, {10, 4}};

std::vector<Plan> candidates(uint32_t log_n) {
  std::vector<Plan> out;
  if (log_n <= 12) {
    Plan p{};
    p.npasses = 1;
    p.pass[0] = {(uint8_t)log_n, 1};
    out.push_back(p);
    return out;
  }
  for (const Shape &t : TOP_SHAPES) {
    const int low = (int)log_n - t.K;
    if (low >= 8 && low <= 12) {
      Plan p{};
      p.npasses = 2;
      p.pass[0] = {t.K, t.C};
      p.pass[1] = {(uint8_t)low, 1};
      if (plan_valid(p, log_n)) out.push_back(p);
    }
    for (const Shape &m : MID_SHAPES) {
      const int low3 = (int)log_n - t.K - m.K;
      if (low3 >= 8 && low3 <= 12) {
        Plan p{};
        p.npasses = 3;
        p.pass[0] = {t.K, t.C};
        p.pass[1] = {m.K, m.C};
        p.pass[2] = {(uint8_t)low3, 1};
        if (plan_valid(p, log_n)) out.push_back(p);
      }
    }
  }
  return out;
}

std::string plan_str(const Plan &p) {
  std::string s;
  for (int i = 0; i < p.npasses; i++) {
    char b[32];
    snprintf(b, sizeof b, "%s%d/%d", i ? "+" : "", p.pass[i].K, p.pass[i].C);
    s += b;
  }
  const Knobs &k = p.knobs;
  if (k.walk || k.top_walk || k.top_mode || k.top_dbuf || k.occ) {
    char b[64];
    snprintf(b, sizeof b, " [w%d t%d m%d d%d o%d]", k.walk, k.top_walk, k.top_mode, k.top_dbuf, k.occ);
    s += b;
  }
  return s;
}

bool has_occ_pass(const Plan &p) {
  for (int i = 0; i < p.npasses; i++)
    if (p.pass[i].C == 1 && p.pass[i].K >= 9) return true;
  return false;
}

// Knob values tried in stage 2 (0, the built-in choice, is stage 1's timing).
struct KnobAxis {
  uint8_t Knobs::*field;
  bool lde_only;
  uint8_t values[6];
  int n;
};
const KnobAxis KNOB_AXES[] = {
    {&Knobs::walk, false, {1, 2, 4, 8, 32, 64}, 6},
    {&Knobs::top_walk, true, {2, 4, 16}, 3},
    {&Knobs::top_mode, true, {TOP_MODE_PREFETCH, TOP_MODE_REFILL}, 2},
    {&Knobs::top_dbuf, true, {1, 2}, 2},
    {&Knobs::occ, false, {BC_PASS_MIN_BLOCKS, BC_PASS_MIN_BLOCKS_B2N}, 2},
};
} // namespace

// The plan of an LDE (log_blowup >= 1) or of a plain NTT (log_blowup = 0).
Plan tuned_plan(uint32_t log_n, uint32_t log_blowup) {
  const int d = current_device();
  if (d >= 0 && d < TUNE_MAX_DEVICES) {
    std::lock_guard<std::mutex> lock(g_table_mutex);
    auto it = g_table[d].find(key(log_n, log_blowup));
    if (it != g_table[d].end()) return it->second;
  }
  return default_plan(log_n);
}

} // namespace bc

using namespace bc;

extern "C" cudaError_t bc_autotune(uint32_t log_n, uint32_t log_blowup, uint32_t num_cols, uint32_t reps,
                                   char *report, size_t report_len) {
  if (log_n < 1 || log_n > (uint32_t)MAX_LOG_N || num_cols == 0 || reps == 0) return cudaErrorInvalidValue;
  if (log_blowup && !lde_args_ok(log_n, num_cols, 1ull << log_n, 1ull << log_n, (uint64_t)num_cols << log_n,
                                 log_blowup))
    return cudaErrorInvalidValue;
  if (!device_tables()) return cudaErrorInitializationError;
  const int dev = current_device();
  if (dev < 0 || dev >= TUNE_MAX_DEVICES) return cudaErrorInvalidDevice;
  const uint64_t n = 1ull << log_n, nb = 1ull << log_blowup;
  uint64_t *in = nullptr, *out = nullptr;
  cudaError_t e = cudaMalloc(&in, num_cols * n * 8);
  if (e != cudaSuccess) return e;
  e = cudaMalloc(&out, num_cols * n * nb * 8);
  if (e != cudaSuccess) {
    cudaFree(in);
    return e;
  }
  cudaStream_t s;
  cudaEvent_t a, b;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaMemsetAsync(in, 0x5A, num_cols * n * 8, s);
  std::string rep;
  float best_ms = 1e30f;
  Plan best = default_plan(log_n);
  std::vector<std::pair<Plan, float>> timed;
  // one warm-up, then `reps` timed runs; the mean ms, or a negative value on an error (kept in e)
  auto time_plan = [&](const Plan &pl) -> float {
    auto run = [&]() -> cudaError_t {
      if (log_blowup)
        return lde_fused(pl, in, out, log_n, num_cols, n, n, (uint64_t)num_cols * n, log_blowup, s);
      return launch_ntt(pl, in, out, log_n, num_cols, n, n, false, false, 0, 0, s);
    };
    if ((e = run()) != cudaSuccess) return -1.f;
    cudaEventRecord(a, s);
    for (uint32_t r = 0; r < reps && e == cudaSuccess; r++) e = run();
    cudaEventRecord(b, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    if (e != cudaSuccess) return -1.f;
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    ms /= (float)reps;
    char line[128];
    snprintf(line, sizeof line, "%s %.4f ms\n", plan_str(pl).c_str(), ms);
    rep += line;
    return ms;
  };
  // stage 1: window splits with the built-in launch shapes
  for (const Plan &pl : candidates(log_n)) {
    const float ms = time_plan(pl);
    if (ms < 0) break;
    timed.emplace_back(pl, ms);
    best_ms = std::min(best_ms, ms);
  }
  // Near-ties (within 1 %, below the run-to-run spread) go to the plan with
  // the fewest passes (one HBM round trip each, which the tuning shape's
  // column count may hide), then to the smallest top window: its top-window
  // kernel has more, shorter tiles, which shortens a job's critical path
  // inside the persistent batch kernel.
  float pick_ms = 1e30f;
  if (e == cudaSuccess) {
    int pick_np = 1 << 30, pick_k = 1 << 30;
    for (const auto &c : timed) {
      if (c.second > best_ms * 1.01f) continue;
      const int np = c.first.npasses, k0 = c.first.pass[0].K;
      if (np < pick_np || (np == pick_np && (k0 < pick_k || (k0 == pick_k && c.second < pick_ms)))) {
        pick_np = np;
        pick_k = k0;
        pick_ms = c.second;
        best = c.first;
      }
    }
  }
  // stage 2: the launch knobs of that split, one axis at a time
  for (const KnobAxis &ax : KNOB_AXES) {
    if (e != cudaSuccess) break;
    if (ax.lde_only && !log_blowup) continue;
    if (ax.field == &Knobs::occ && !has_occ_pass(best)) continue;
    Plan axis_best = best;
    float axis_ms = pick_ms;
    for (int v = 0; v < ax.n && e == cudaSuccess; v++) {
      Plan c = best;
      c.knobs.*ax.field = ax.values[v];
      const float ms = time_plan(c);
      if (ms < 0) break;
      if (ms < axis_ms) {
        axis_ms = ms;
        axis_best = c;
      }
    }
    if (axis_ms < pick_ms * 0.99f) {
      best = axis_best;
      pick_ms = axis_ms;
    }
  }
  cudaStreamSynchronize(s);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaStreamDestroy(s);
  cudaFree(in);
  cudaFree(out);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> lock(g_table_mutex);
    g_table[dev][key(log_n, log_blowup)] = best;
  }
  rep += "best " + plan_str(best) + "\n";
  if (report && report_len) {
    strncpy(report, rep.c_str(), report_len - 1);
    report[report_len - 1] = 0;
  }
  return cudaSuccess;
}

// Text form, one line per entry: "log_n log_blowup npasses K0 C0 [K1 C1 [K2 C2]]",
// then "k walk top_walk top_mode top_dbuf occ" when a knob is not the built-in one.
extern "C" cudaError_t bc_plan_table_export(char *buf, size_t len, size_t *needed) {
  const int dev = current_device();
  if (dev < 0 || dev >= TUNE_MAX_DEVICES) return cudaErrorInvalidDevice;
  std::string t;
  {
    std::lock_guard<std::mutex> lock(g_table_mutex);
    for (auto &kv : g_table[dev]) {
      char line[128];
      int w = snprintf(line, sizeof line, "%u %u %d", kv.first & 0xFF, kv.first >> 8, kv.second.npasses);
      for (int i = 0; i < kv.second.npasses; i++)
        w += snprintf(line + w, sizeof line - w, " %d %d", kv.second.pass[i].K, kv.second.pass[i].C);
      const Knobs &k = kv.second.knobs;
      if (k.walk || k.top_walk || k.top_mode || k.top_dbuf || k.occ)
        snprintf(line + w, sizeof line - w, " k %d %d %d %d %d", k.walk, k.top_walk, k.top_mode, k.top_dbuf, k.occ);
      t += line;
      t += "\n";
    }
  }
  if (needed) *needed = t.size() + 1;
  if (buf && len) {
    if (len < t.size() + 1) return cudaErrorInvalidValue;
    memcpy(buf, t.c_str(), t.size() + 1);
  }
  return cudaSuccess;
}

extern "C" cudaError_t bc_plan_table_import(const char *text) {
  if (!text) return cudaErrorInvalidValue;
  const int dev = current_device();
  if (dev < 0 || dev >= TUNE_MAX_DEVICES) return cudaErrorInvalidDevice;
  std::vector<std::pair<uint32_t, Plan>> parsed;
  const char *p = text;
  while (*p) {
    unsigned log_n, log_b;
    int np, used = 0;
    if (sscanf(p, "%u %u %d%n", &log_n, &log_b, &np, &used) != 3) break;
    p += used;
    Plan pl{};
    if (np < 1 || np > 4) return cudaErrorInvalidValue;
    pl.npasses = np;
    for (int i = 0; i < np; i++) {
      int K, C;
      if (sscanf(p, "%d %d%n", &K, &C, &used) != 2) return cudaErrorInvalidValue;
      p += used;
      pl.pass[i] = {(uint8_t)K, (uint8_t)C};
    }
    while (*p == ' ' || *p == '\t') p++;
    if (*p == 'k') {
      int kv[5];
      if (sscanf(p + 1, "%d %d %d %d %d%n", &kv[0], &kv[1], &kv[2], &kv[3], &kv[4], &used) != 5)
        return cudaErrorInvalidValue;
      p += 1 + used;
      if (kv[0] < 0 || kv[0] > 255 || kv[1] < 0 || kv[1] > 255 || kv[2] < 0 || kv[2] > TOP_MODE_REFILL || kv[3] < 0 ||
          kv[3] > 2 || (kv[4] != 0 && kv[4] != BC_PASS_MIN_BLOCKS && kv[4] != BC_PASS_MIN_BLOCKS_B2N))
        return cudaErrorInvalidValue;
      pl.knobs = Knobs{(uint8_t)kv[0], (uint8_t)kv[1], (uint8_t)kv[2], (uint8_t)kv[3], (uint8_t)kv[4]};
    }
    if (log_n < 1 || log_n > (unsigned)MAX_LOG_N || log_b > 8 || !plan_valid(pl, log_n)) return cudaErrorInvalidValue;
    parsed.push_back({key(log_n, log_b), pl});
    while (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t') p++;
  }
  std::lock_guard<std::mutex> lock(g_table_mutex);
  for (auto &kv : parsed) g_table[dev][kv.first] = kv.second;
  return cudaSuccess;
}

extern "C" cudaError_t bc_plan_table_clear(void) {
  const int dev = current_device();
  if (dev < 0 || dev >= TUNE_MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_table_mutex);
  g_table[dev].clear();
  return cudaSuccess;
}
