// lde_batch.cu -- uneven batches of coset LDE jobs in ONE persistent launch.
//
// The reference has no batch entry point: its callers issue one inverse and
// one forward batch_ntt per coset per job (src/ntt.rs:179-191), and for
// log_n < 16 every stage is its own launch (src/ntt.rs:201-241), so a batch of
// small, uneven jobs is dominated by launch latency and tail effects.
//
// Here a batch plan turns every job's fused LDE (lde.cu: inverse passes,
// top-window kernel, forward passes) into "records" -- one per kernel of the
// job, each holding exactly the parameters the standalone launch would get --
// and every record into work items, one per CTA of that launch.  Records are
// ordered by depth (first kernels of all jobs, then second kernels, ...) and
// items by record, so every item depends only on items earlier in the list.
// One persistent kernel (grid = resident CTAs) pulls items with an atomic
// counter; before an item of a job's k-th kernel it waits until all items of
// the job's (k-1)-th kernel are done.  Because items are taken in list order
// and every earlier item is held by a running CTA, the waits always end.  Each
// wait is still bounded in time: on expiry the kernel sets a status bit,
// skips the item and carries on, so a fault can never hang the GPU.
//
// The launch (counter reset + kernel) is captured once per plan in a CUDA
// graph and replayed by bc_lde_batch_run.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/bc_ntt.h"
#include "lde.cuh"

namespace bc {

// Dispatch id of a kernel body: (top << 7) | (b2n << 6) | (K << 2) | log2(C).
__host__ __device__ constexpr uint32_t shape_id(bool top, bool b2n, int K, int C) {
  return ((top ? 1u : 0u) << 7) | ((b2n ? 1u : 0u) << 6) | ((uint32_t)K << 2) |
         (C == 1 ? 0u : C == 2 ? 1u : C == 4 ? 2u : 3u);
}

struct BatchRecord {
  uint32_t shape;
  int32_t pred;     // record that must be complete before any item of this one, or -1
  uint32_t n_items; // CTAs of this kernel
  uint32_t pad;
  union {
    PassParams pass;
    LdeTopParams top;
  } u;
};

// item = record (16 bits) | column chunk by (20 bits) | tile position bx (28 bits)
__host__ __device__ constexpr uint64_t make_item(uint32_t rec, uint32_t by, uint32_t bx) {
  return ((uint64_t)rec << 48) | ((uint64_t)by << 28) | (uint64_t)bx;
}

constexpr uint32_t BATCH_THREADS = 256;
constexpr uint32_t BATCH_SMEM_BYTES = TOP_RESIDENT_SMEM_MAX; // largest body: top window of 12 bits, one forward table

// The bodies the persistent kernel can run: every window shape of the default
// plans (and of the tuner's candidates).
#define BC_BATCH_SHAPES(X)                                                                                           \
  X(true, false, 1, 1) X(true, false, 2, 1) X(true, false, 3, 1) X(true, false, 4, 1) X(true, false, 5, 1)        \
  X(true, false, 6, 1) X(true, false, 7, 1) X(true, false, 8, 1) X(true, false, 9, 1) X(true, false, 10, 1)       \
  X(true, false, 11, 1) X(true, false, 12, 1) X(true, false, 4, 8) X(true, false, 5, 8) X(true, false, 8, 8)      \
  X(true, false, 9, 8) X(true, false, 10, 4) X(true, false, 11, 2)                                                 \
  X(false, true, 8, 1) X(false, true, 9, 1) X(false, true, 10, 1) X(false, true, 11, 1) X(false, true, 12, 1)     \
  X(false, false, 8, 1) X(false, false, 9, 1) X(false, false, 10, 1) X(false, false, 11, 1)                         \
  X(false, false, 12, 1) X(false, true, 8, 8) X(false, true, 9, 8) X(false, true, 10, 4) X(false, false, 8, 8)    \
  X(false, false, 9, 8) X(false, false, 10, 4)

bool batch_shape_supported(uint32_t id) {
#define BC_CASE(TOP, B2N, K, C)                                                                                      \
  if (id == shape_id(TOP, B2N, K, C)) return true;
  BC_BATCH_SHAPES(BC_CASE)
#undef BC_CASE
  return false;
}

template <bool TOP, bool B2N, int K, int C>
__device__ __noinline__ void run_shape(const BatchRecord &rec, uint32_t bx, uint32_t by, uint64_t *smem) {
  if constexpr (TOP)
    top_body<K, C>(rec.u.top, bx, by, smem);
  else
    pass_body<K, C, B2N, B2N>(rec.u.pass, bx, by, smem); // LDE passes: b2n ones are the inverse transform
}

__device__ __forceinline__ void run_body(const BatchRecord &rec, uint32_t bx, uint32_t by, uint64_t *smem) {
  switch (rec.shape) {
#define BC_CASE(TOP, B2N, K, C)                                                                                      \
  case shape_id(TOP, B2N, K, C):                                                                                     \
    run_shape<TOP, B2N, K, C>(rec, bx, by, smem);                                                                    \
    break;
    BC_BATCH_SHAPES(BC_CASE)
#undef BC_CASE
  default:
    break;
  }
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// status bit 0: a dependency wait expired (the batch's results are invalid).
// wait_limit: SM clock cycles one dependency wait may take (read once per CTA).
__global__ void __launch_bounds__(BATCH_THREADS, 2)
    lde_batch_kernel(const BatchRecord *__restrict__ recs, const uint64_t *__restrict__ items, uint32_t n_items,
                     uint32_t *done, uint32_t *next, uint32_t *status, const long long *wait_limit) {
  extern __shared__ uint64_t smem[];
  __shared__ uint32_t s_idx, s_ok;
  __shared__ BatchRecord s_rec; // the item's kernel parameters, read by the body from shared memory
  const long long timeout_cycles = threadIdx.x == 0 ? *wait_limit : 0;
  for (;;) {
    if (threadIdx.x == 0) s_idx = atomicAdd(next, 1u);
    __syncthreads();
    const uint32_t idx = s_idx;
    if (idx >= n_items) return;
    const uint64_t it = items[idx];
    const uint32_t r = (uint32_t)(it >> 48), by = (uint32_t)(it >> 28) & 0xFFFFFu, bx = (uint32_t)it & 0xFFFFFFFu;
    const BatchRecord &rec = recs[r];
    static_assert(sizeof(BatchRecord) % 4 == 0, "record copy by words");
    for (uint32_t w = threadIdx.x; w < sizeof(BatchRecord) / 4; w += blockDim.x)
      reinterpret_cast<uint32_t *>(&s_rec)[w] = reinterpret_cast<const uint32_t *>(&rec)[w];
    if (threadIdx.x == 0) {
      uint32_t ok = 1;
      if (rec.pred >= 0) {
        const uint32_t need = recs[rec.pred].n_items;
        const long long t0 = clock64();
        while (ld_acquire(done + rec.pred) < need) {
          if (clock64() - t0 > timeout_cycles) {
            ok = 0;
            atomicOr(status, 1u);
            break;
          }
          __nanosleep(128);
        }
      }
      s_ok = ok;
    }
    __syncthreads();
    if (s_ok) run_body(s_rec, bx, by, smem);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(done + r, 1u);
    }
  }
}

} // namespace bc

using namespace bc;

struct bc_lde_batch_plan {
  int device = -1;
  uint32_t n_records = 0, n_items = 0, grid = 0;
  BatchRecord *d_records = nullptr;
  uint64_t *d_items = nullptr;
  uint32_t *d_counters = nullptr; // done[n_records], next, status, then the 64-bit wait limit (8-byte aligned)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long timeout_cycles = 0;
};

namespace {
// Words of a counters block for n_records records: done[], next, status, padding to 8 bytes, the wait limit.
uint32_t counter_words(uint32_t n_records) { return ((n_records + 2 + 1) & ~1u) + 2; }
long long *wait_limit_slot(uint32_t *counters, uint32_t n_records) {
  return reinterpret_cast<long long *>(counters + counter_words(n_records) - 2);
}
// About 4 s of SM clock per dependency wait.  The clock-rate query costs
// around a millisecond on some drivers, so it is made once per device.
long long default_wait_limit(int device) {
  static std::atomic<long long> cache[64];
  if (device >= 0 && device < 64) {
    const long long c = cache[device].load(std::memory_order_relaxed);
    if (c) return c;
  }
  int clock_khz = 0;
  cudaDeviceGetAttribute(&clock_khz, cudaDevAttrClockRate, device);
  const long long v = (long long)std::max(clock_khz, 1000000) * 1000ll * 4;
  if (device >= 0 && device < 64) cache[device].store(v, std::memory_order_relaxed);
  return v;
}
} // namespace

namespace {

cudaError_t free_plan(bc_lde_batch_plan *p) {
  if (!p) return cudaSuccess;
  cudaError_t e = cudaSuccess, e2;
  if (p->exec && (e2 = cudaGraphExecDestroy(p->exec)) != cudaSuccess) e = e2;
  if (p->graph && (e2 = cudaGraphDestroy(p->graph)) != cudaSuccess) e = e2;
  if (p->d_records && (e2 = cudaFree(p->d_records)) != cudaSuccess) e = e2;
  if (p->d_items && (e2 = cudaFree(p->d_items)) != cudaSuccess) e = e2;
  if (p->d_counters && (e2 = cudaFree(p->d_counters)) != cudaSuccess) e = e2;
  delete p;
  return e;
}

uint64_t job_work(const bc_lde_job &j) { return ((uint64_t)j.num_cols << j.log_n) << j.log_blowup; }

size_t round256(size_t x) { return (x + 255) & ~(size_t)255; }

// Device bytes of a schedule laid out as counters (done[n_records], next,
// status) | records | items, each part 256-byte aligned.
size_t schedule_bytes(size_t n_records, size_t n_items) {
  return round256((((n_records + 3) & ~(size_t)1) + 2) * sizeof(uint32_t)) +
         round256(n_records * sizeof(BatchRecord)) + n_items * sizeof(uint64_t);
}

// Records and items of a batch, in dependency order (host side).
// standalone_min_ctas > 0: a job whose every kernel, launched on its own, has
// at least that many CTAs goes to `standalone` (its fused-LDE steps in order)
// instead of the persistent kernel's schedule.
// max_bytes > 0: a schedule needing more device bytes (schedule_bytes) returns
// cudaErrorInvalidValue before any record or item is built.
cudaError_t schedule(const bc_lde_job *jobs, uint32_t n_jobs, std::vector<BatchRecord> &recs,
                     std::vector<uint64_t> &items, uint32_t standalone_min_ctas = 0,
                     std::vector<LdeStep> *standalone = nullptr, size_t max_bytes = 0) {
  std::vector<std::vector<LdeStep>> steps(n_jobs);
  size_t max_depth = 0;
  for (uint32_t j = 0; j < n_jobs; j++) {
    const bc_lde_job &jb = jobs[j];
    if (!lde_args_ok(jb.log_n, jb.num_cols, jb.stride_in, jb.stride_out, jb.coset_stride, jb.log_blowup))
      return cudaErrorInvalidValue;
    if (jb.num_cols && (!jb.evals_bitrev || !jb.out)) return cudaErrorInvalidValue;
    if (standalone_min_ctas && standalone && jb.num_cols) {
      std::vector<LdeStep> own;
      if (!build_lde_steps(tuned_plan(jb.log_n, jb.log_blowup), jb.evals_bitrev, jb.out, jb.log_n, jb.num_cols,
                           jb.stride_in, jb.stride_out, jb.coset_stride, jb.log_blowup, false, 8, 8, own))
        return cudaErrorInvalidConfiguration;
      uint64_t min_ctas = ~0ull;
      for (const LdeStep &st : own) min_ctas = std::min<uint64_t>(min_ctas, (uint64_t)st.grid.x * st.grid.y);
      if (min_ctas >= standalone_min_ctas) {
        standalone->insert(standalone->end(), own.begin(), own.end());
        continue; // steps[j] stays empty: no records for this job
      }
    }
    // the tuned plan, or the built-in one when the tuned plan uses a window shape this kernel does not carry
    auto build = [&](const Plan &pl) {
      if (!build_lde_steps(pl, jb.evals_bitrev, jb.out, jb.log_n, jb.num_cols, jb.stride_in, jb.stride_out,
                           jb.coset_stride, jb.log_blowup, true, 16, 16, steps[j]))
        return false;
      for (const LdeStep &st : steps[j])
        if (!batch_shape_supported(shape_id(st.top, st.b2n, st.K, st.C)) || st.threads != BATCH_THREADS ||
            st.smem > BATCH_SMEM_BYTES || st.grid.x >= (1u << 28) || st.grid.y >= (1u << 20) ||
            (!st.top && st.pass.inverse != (uint32_t)st.b2n)) // the kernel carries LDE passes only
          return false;
      return true;
    };
    if (!build(tuned_plan(jb.log_n, jb.log_blowup)) && !build(default_plan(jb.log_n)))
      return cudaErrorInvalidConfiguration;
    max_depth = std::max(max_depth, steps[j].size());
  }
  if (max_bytes) {
    uint64_t n_recs = 0, n_items = 0;
    for (uint32_t j = 0; j < n_jobs; j++)
      for (const LdeStep &st : steps[j]) {
        n_recs++;
        n_items += (uint64_t)st.grid.x * st.grid.y;
      }
    if (n_items > max_bytes / sizeof(uint64_t) || schedule_bytes(n_recs, n_items) > max_bytes)
      return cudaErrorInvalidValue;
  }
  // big jobs first within every depth
  std::vector<uint32_t> order(n_jobs);
  for (uint32_t j = 0; j < n_jobs; j++) order[j] = j;
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return job_work(jobs[a]) > job_work(jobs[b]); });
  std::vector<int32_t> last(n_jobs, -1);
  recs.clear();
  items.clear();
  for (size_t d = 0; d < max_depth; d++) {
    for (uint32_t j : order) {
      if (d >= steps[j].size()) continue;
      const LdeStep &st = steps[j][d];
      BatchRecord r;
      std::memset(&r, 0, sizeof(r));
      r.shape = shape_id(st.top, st.b2n, st.K, st.C);
      r.pred = last[j];
      r.n_items = st.grid.x * st.grid.y;
      if (st.top)
        r.u.top = st.topp;
      else
        r.u.pass = st.pass;
      const uint32_t rid = (uint32_t)recs.size();
      if (rid >= (1u << 16)) return cudaErrorInvalidConfiguration;
      recs.push_back(r);
      last[j] = (int32_t)rid;
      for (uint32_t by = 0; by < st.grid.y; by++)
        for (uint32_t bx = 0; bx < st.grid.x; bx++) items.push_back(make_item(rid, by, bx));
    }
  }
  if (items.size() >= (1ull << 32)) return cudaErrorInvalidConfiguration;
  return cudaSuccess;
}

} // namespace

extern "C" cudaError_t bc_lde_batch_plan_create_ex(const bc_lde_job *jobs, uint32_t n_jobs,
                                                   uint32_t standalone_min_ctas, bc_lde_batch_plan **plan) {
  if (!plan || (n_jobs && !jobs)) return cudaErrorInvalidValue;
  *plan = nullptr;
  if (!device_tables()) return cudaErrorInitializationError;
  std::vector<BatchRecord> recs;
  std::vector<uint64_t> items;
  std::vector<LdeStep> standalone;
  cudaError_t e = schedule(jobs, n_jobs, recs, items, standalone_min_ctas, &standalone);
  if (e != cudaSuccess) return e;
  bc_lde_batch_plan *p = new (std::nothrow) bc_lde_batch_plan();
  if (!p) return cudaErrorMemoryAllocation;
  p->device = current_device();
  p->n_records = (uint32_t)recs.size();
  p->n_items = (uint32_t)items.size();
  p->timeout_cycles = default_wait_limit(p->device);
#define CK(x)                                                                                                          \
  if ((e = (x)) != cudaSuccess) {                                                                                      \
    free_plan(p);                                                                                                      \
    return e;                                                                                                          \
  }
  CK(cudaFuncSetAttribute(lde_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BATCH_SMEM_BYTES));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lde_batch_kernel, BATCH_THREADS, BATCH_SMEM_BYTES));
  if (per_sm < 1) {
    free_plan(p);
    return cudaErrorInvalidConfiguration;
  }
  p->grid = (uint32_t)(per_sm * sm_count());
  if (p->n_records) {
    CK(cudaMalloc(&p->d_records, recs.size() * sizeof(BatchRecord)));
    CK(cudaMemcpy(p->d_records, recs.data(), recs.size() * sizeof(BatchRecord), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&p->d_items, items.size() * sizeof(uint64_t)));
    CK(cudaMemcpy(p->d_items, items.data(), items.size() * sizeof(uint64_t), cudaMemcpyHostToDevice));
  }
  CK(cudaMalloc(&p->d_counters, counter_words(p->n_records) * sizeof(uint32_t)));
  CK(cudaMemset(p->d_counters, 0, (p->n_records + 2) * sizeof(uint32_t)));
  CK(cudaMemcpy(wait_limit_slot(p->d_counters, p->n_records), &p->timeout_cycles, sizeof(long long),
                cudaMemcpyHostToDevice));
  // capture: reset the counters, run the persistent kernel; the standalone jobs'
  // kernels run on a forked branch of the same graph, concurrently with it
  cudaStream_t cs, cs2;
  cudaEvent_t fork, join;
  CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&cs2, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
  e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
  if (e == cudaSuccess) {
    cudaError_t ec = cudaMemsetAsync(p->d_counters, 0, (p->n_records + 2) * sizeof(uint32_t), cs);
    if (ec == cudaSuccess && !standalone.empty()) {
      ec = cudaEventRecord(fork, cs);
      if (ec == cudaSuccess) ec = cudaStreamWaitEvent(cs2, fork, 0);
      for (size_t i = 0; ec == cudaSuccess && i < standalone.size(); i++) ec = launch_lde_step(standalone[i], cs2);
      if (ec == cudaSuccess) ec = cudaEventRecord(join, cs2);
    }
    if (ec == cudaSuccess && p->n_items) {
      lde_batch_kernel<<<p->grid, BATCH_THREADS, BATCH_SMEM_BYTES, cs>>>(
          p->d_records, p->d_items, p->n_items, p->d_counters, p->d_counters + p->n_records,
          p->d_counters + p->n_records + 1, wait_limit_slot(p->d_counters, p->n_records));
      ec = cudaGetLastError();
    }
    if (ec == cudaSuccess && !standalone.empty()) ec = cudaStreamWaitEvent(cs, join, 0);
    e = cudaStreamEndCapture(cs, &p->graph);
    if (e == cudaSuccess) e = ec;
  }
  cudaEventDestroy(fork);
  cudaEventDestroy(join);
  cudaStreamDestroy(cs2);
  cudaStreamDestroy(cs);
  if (e != cudaSuccess) {
    free_plan(p);
    return e;
  }
  CK(cudaGraphInstantiate(&p->exec, p->graph, 0));
#undef CK
  *plan = p;
  return cudaSuccess;
}

extern "C" cudaError_t bc_lde_batch_plan_create(const bc_lde_job *jobs, uint32_t n_jobs, bc_lde_batch_plan **plan) {
  return bc_lde_batch_plan_create_ex(jobs, n_jobs, 0, plan);
}

extern "C" cudaError_t bc_lde_batch_run(bc_lde_batch_plan *plan, cudaStream_t stream) {
  if (!plan) return cudaErrorInvalidValue;
  if (current_device() != plan->device) return cudaErrorInvalidDevice;
  return cudaGraphLaunch(plan->exec, stream);
}

extern "C" cudaError_t bc_lde_batch_status(bc_lde_batch_plan *plan, cudaStream_t stream, uint32_t *status) {
  if (!plan || !status) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemcpyAsync(status, plan->d_counters + plan->n_records + 1, sizeof(uint32_t),
                                  cudaMemcpyDeviceToHost, stream);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(stream);
}

extern "C" cudaError_t bc_lde_batch_plan_set_wait_limit(bc_lde_batch_plan *plan, uint64_t cycles) {
  if (!plan || cycles > (uint64_t)LLONG_MAX) return cudaErrorInvalidValue;
  if (current_device() != plan->device) return cudaErrorInvalidDevice;
  const long long v = cycles ? (long long)cycles : default_wait_limit(plan->device);
  // runs already enqueued (on any stream) finish with the old limit; later ones read the new one
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(wait_limit_slot(plan->d_counters, plan->n_records), &v, sizeof(v), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) plan->timeout_cycles = v;
  return e;
}

extern "C" cudaError_t bc_lde_batch_plan_info(const bc_lde_batch_plan *plan, uint32_t *n_records, uint32_t *n_items,
                                              uint32_t *grid) {
  if (!plan) return cudaErrorInvalidValue;
  if (n_records) *n_records = plan->n_records;
  if (n_items) *n_items = plan->n_items;
  if (grid) *grid = plan->grid;
  return cudaSuccess;
}

extern "C" cudaError_t bc_lde_batch_plan_destroy(bc_lde_batch_plan *plan) { return free_plan(plan); }

// ---------------------------------------------------------------------------
// Batch entry point that allocates nothing.
//
// Some callers cannot call cudaMalloc: a prover that reserves nearly all of
// HBM for its own memory pool at start-up and sub-allocates from it (a
// cudaMalloc then fails or fragments the pool), or a latency-critical
// submission path where the implicit device-wide synchronisation of
// cudaMalloc/cudaFree would stall work on other streams.  For them the
// batch schedule (records, work items, counters) lives in the fixed array
// below instead of plan-owned allocations.  The array is part of this
// library's device image, so every GPU that loads the library holds its
// 16 MiB until the process exits.
namespace bc {
constexpr size_t NOALLOC_SCRATCH_BYTES = 16u << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
void *g_noalloc_base[NOALLOC_MAX_DEVICES] = {};
int g_noalloc_grid[NOALLOC_MAX_DEVICES] = {};
std::mutex g_noalloc_mutex;

// First call on a device: device address of the scratch array and the
// persistent grid size.  Host code cannot use g_noalloc_scratch directly --
// in host code that name is only a stand-in for the device symbol.
cudaError_t noalloc_setup(int dev, void **base, int *grid) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_base[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(lde_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BATCH_SMEM_BYTES);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lde_batch_kernel, BATCH_THREADS, BATCH_SMEM_BYTES);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    g_noalloc_grid[dev] = per_sm * sm_count();
    g_noalloc_base[dev] = p;
  }
  *base = g_noalloc_base[dev];
  *grid = g_noalloc_grid[dev];
  return cudaSuccess;
}
} // namespace
} // namespace bc

namespace bc {
// Enqueues a batch on `stream` with its schedule in device scratch the caller
// owns (used by the serving loop): the counters, records and items are
// written into host_staging (pinned, at least scratch_bytes) and copied to
// dev_scratch with one copy, then the persistent kernel runs.  The caller
// must not reuse host_staging until that copy has completed, nor dev_scratch
// until the kernel has.  A batch whose schedule exceeds scratch_bytes returns
// cudaErrorInvalidValue before anything is enqueued.
cudaError_t batch_enqueue_into(const bc_lde_job *jobs, uint32_t n_jobs, void *dev_scratch, void *host_staging,
                               size_t scratch_bytes, cudaStream_t stream) {
  if (n_jobs && !jobs) return cudaErrorInvalidValue;
  if (!dev_scratch || !host_staging || (uintptr_t)dev_scratch % 256 || (uintptr_t)host_staging % 256)
    return cudaErrorInvalidValue;
  std::vector<BatchRecord> recs;
  std::vector<uint64_t> items;
  cudaError_t e = schedule(jobs, n_jobs, recs, items, 0, nullptr, scratch_bytes);
  if (e != cudaSuccess) return e;
  if (items.empty()) return cudaSuccess;
  const uint32_t n_rec = (uint32_t)recs.size();
  const size_t counters_bytes = round256(counter_words(n_rec) * sizeof(uint32_t));
  const size_t recs_bytes = round256(recs.size() * sizeof(BatchRecord));
  const size_t items_bytes = items.size() * sizeof(uint64_t);
  const size_t total = counters_bytes + recs_bytes + items_bytes;
  if (total > scratch_bytes) return cudaErrorInvalidValue;
  unsigned char *h = static_cast<unsigned char *>(host_staging);
  std::memset(h, 0, counters_bytes);
  const long long limit = default_wait_limit(current_device());
  std::memcpy(wait_limit_slot(reinterpret_cast<uint32_t *>(h), n_rec), &limit, sizeof(limit));
  std::memcpy(h + counters_bytes, recs.data(), recs.size() * sizeof(BatchRecord));
  std::memcpy(h + counters_bytes + recs_bytes, items.data(), items_bytes);
  e = cudaMemcpyAsync(dev_scratch, host_staging, total, cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return e;
  static std::atomic<int> grid_cache[64];
  const int dev = current_device();
  int grid = (dev >= 0 && dev < 64) ? grid_cache[dev].load(std::memory_order_relaxed) : 0;
  if (!grid) {
    e = cudaFuncSetAttribute(lde_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BATCH_SMEM_BYTES);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lde_batch_kernel, BATCH_THREADS, BATCH_SMEM_BYTES);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    grid = per_sm * sm_count();
    if (dev >= 0 && dev < 64) grid_cache[dev].store(grid, std::memory_order_relaxed);
  }
  unsigned char *d = static_cast<unsigned char *>(dev_scratch);
  uint32_t *counters = reinterpret_cast<uint32_t *>(d);
  lde_batch_kernel<<<grid, BATCH_THREADS, BATCH_SMEM_BYTES, stream>>>(
      reinterpret_cast<const BatchRecord *>(d + counters_bytes),
      reinterpret_cast<const uint64_t *>(d + counters_bytes + recs_bytes), (uint32_t)items.size(), counters,
      counters + n_rec, counters + n_rec + 1, wait_limit_slot(counters, n_rec));
  return cudaGetLastError();
}
} // namespace bc

extern "C" cudaError_t bc_lde_batch_noalloc(const bc_lde_job *jobs, uint32_t n_jobs, cudaStream_t stream,
                                            uint32_t *status) {
  if (n_jobs && !jobs) return cudaErrorInvalidValue;
  // The schedule is copied from host vectors that this call frees on return,
  // and `status` synchronises the stream: neither can be recorded into a graph.
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(stream, &capture);
  if (e != cudaSuccess) return e;
  if (capture != cudaStreamCaptureStatusNone) return cudaErrorStreamCaptureUnsupported;
  if (!device_tables()) return cudaErrorInitializationError;
  const int dev = current_device();
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
  void *base = nullptr;
  int grid = 0;
  e = noalloc_setup(dev, &base, &grid);
  if (e != cudaSuccess) return e;
  std::vector<BatchRecord> recs;
  std::vector<uint64_t> items;
  e = schedule(jobs, n_jobs, recs, items, 0, nullptr, NOALLOC_SCRATCH_BYTES);
  if (e != cudaSuccess) return e;
  // layout: counters (done[n_records], next, status, wait limit) | records | items
  const size_t counters_bytes = round256(counter_words((uint32_t)recs.size()) * sizeof(uint32_t));
  const size_t recs_bytes = round256(recs.size() * sizeof(BatchRecord));
  const size_t items_bytes = items.size() * sizeof(uint64_t);
  if (schedule_bytes(recs.size(), items.size()) > NOALLOC_SCRATCH_BYTES) return cudaErrorInvalidValue;
  unsigned char *b = static_cast<unsigned char *>(base);
  uint32_t *counters = reinterpret_cast<uint32_t *>(b);
  BatchRecord *d_recs = reinterpret_cast<BatchRecord *>(b + counters_bytes);
  uint64_t *d_items = reinterpret_cast<uint64_t *>(b + counters_bytes + recs_bytes);
  // the previous call's contents stay in the array: the counters must start at zero
  e = cudaMemsetAsync(counters, 0, (recs.size() + 2) * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  if (!items.empty()) {
    // pageable sources: each copy has consumed its host buffer when it returns
    e = cudaMemcpyAsync(d_recs, recs.data(), recs.size() * sizeof(BatchRecord), cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(d_items, items.data(), items_bytes, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return e;
    const uint32_t n_rec = (uint32_t)recs.size();
    const long long limit = default_wait_limit(dev);
    e = cudaMemcpyAsync(wait_limit_slot(counters, n_rec), &limit, sizeof(limit), cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return e;
    lde_batch_kernel<<<grid, BATCH_THREADS, BATCH_SMEM_BYTES, stream>>>(d_recs, d_items, (uint32_t)items.size(),
                                                                         counters, counters + n_rec,
                                                                         counters + n_rec + 1,
                                                                         wait_limit_slot(counters, n_rec));
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (status) {
    *status = 0;
    e = cudaMemcpyAsync(status, counters + recs.size() + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(stream);
  }
  return e;
}
