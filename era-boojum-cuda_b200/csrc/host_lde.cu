// host_lde.cu -- coset LDE from host memory to host memory, with the copies
// overlapped with the computation.
//
// The reference's callers move columns to the device, run the NTTs, and move
// the cosets back, one step after the other.  Here the columns are split into
// chunks that cycle through a few device buffers on three streams: while chunk
// i is transformed, chunk i+1 is being copied in and chunk i-1 copied out, so
// the time approaches that of the slower copy direction (PCIe is full duplex)
// instead of the sum of all three steps.  Host buffers should be pinned
// (cudaHostAlloc / cudaHostRegister) for the copies to overlap; pageable
// buffers still give correct results, without the overlap.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "../../include/bc_ntt.h"
#include "host_lde.cuh"

namespace bc {

namespace {
constexpr int HOST_MAX_DEVICES = 64;
HostPipe g_pipes[HOST_MAX_DEVICES];
std::mutex g_pipe_mutex[HOST_MAX_DEVICES];
} // namespace

cudaError_t host_pipe_init(HostPipe &hp) {
  if (hp.live) return cudaSuccess;
  cudaError_t e = cudaSuccess;
  auto fail = [&]() {
    host_pipe_destroy(hp); // what was created so far
    return e;
  };
  if ((e = cudaStreamCreateWithFlags(&hp.s_in, cudaStreamNonBlocking)) != cudaSuccess) return fail();
  if ((e = cudaStreamCreateWithFlags(&hp.s_comp, cudaStreamNonBlocking)) != cudaSuccess) return fail();
  if ((e = cudaStreamCreateWithFlags(&hp.s_out, cudaStreamNonBlocking)) != cudaSuccess) return fail();
  for (auto &x : hp.ev)
    if ((e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming)) != cudaSuccess) return fail();
  if ((e = cudaEventCreateWithFlags(&hp.entry, cudaEventDisableTiming)) != cudaSuccess) return fail();
  if ((e = cudaEventCreateWithFlags(&hp.done_in, cudaEventDisableTiming)) != cudaSuccess) return fail();
  if ((e = cudaEventCreateWithFlags(&hp.done_out, cudaEventDisableTiming)) != cudaSuccess) return fail();
  hp.live = true;
  return cudaSuccess;
}

// Destroys every stream and event of the pipe that exists (a partly
// initialised pipe included) and resets it.
void host_pipe_destroy(HostPipe &hp) {
  for (cudaStream_t s : {hp.s_in, hp.s_comp, hp.s_out})
    if (s) cudaStreamDestroy(s);
  for (auto &x : hp.ev)
    if (x) cudaEventDestroy(x);
  for (cudaEvent_t x : {hp.entry, hp.done_in, hp.done_out})
    if (x) cudaEventDestroy(x);
  hp = HostPipe{};
}

// Columns per chunk so that HOST_NBUF chunk buffers (input + all cosets) fit the workspace.
uint32_t host_chunk_cols(uint32_t log_n, uint32_t num_cols, uint32_t log_blowup, size_t workspace_bytes,
                         uint32_t max_chunk_cols) {
  const uint64_t per_col = 8ull * ((1ull << log_n) + ((1ull << log_n) << log_blowup));
  uint64_t c = workspace_bytes / (per_col * HOST_NBUF);
  if (max_chunk_cols) c = std::min<uint64_t>(c, max_chunk_cols);
  return (uint32_t)std::min<uint64_t>(c, num_cols);
}

cudaError_t host_lde_enqueue(HostPipe &hp, const uint64_t *host_in, uint64_t *host_out, uint32_t log_n,
                             uint32_t num_cols, uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride,
                             uint32_t log_blowup, uint64_t *workspace, uint32_t chunk, bool caller_ordered,
                             cudaStream_t caller) {
  const uint64_t n = 1ull << log_n, nb = 1ull << log_blowup;
  const uint64_t in_words = (uint64_t)chunk * n, out_words = in_words * nb;
  const Plan pl = tuned_plan(log_n, log_blowup);
  cudaError_t e;
#define CK(x)                                                                                                          \
  if ((e = (x)) != cudaSuccess) return e;
  if (caller_ordered) { // everything below starts after the work already queued on the caller's stream
    CK(cudaEventRecord(hp.entry, caller));
    CK(cudaStreamWaitEvent(hp.s_in, hp.entry, 0));
    CK(cudaStreamWaitEvent(hp.s_comp, hp.entry, 0));
    CK(cudaStreamWaitEvent(hp.s_out, hp.entry, 0));
  }
  cudaEvent_t *ev_in = hp.ev, *ev_comp = hp.ev + HOST_NBUF, *ev_free = hp.ev + 2 * HOST_NBUF;
  const uint32_t n_chunks = (num_cols + chunk - 1) / chunk;
  for (uint32_t c = 0; c < n_chunks; c++) {
    const int b = (int)(c % HOST_NBUF);
    const uint32_t j0 = c * chunk, cols = std::min(chunk, num_cols - j0);
    uint64_t *d_in = workspace + (uint64_t)b * (in_words + out_words);
    uint64_t *d_out = d_in + in_words;
    // copy in (the buffer must have been drained by the copy-out of chunk c - HOST_NBUF)
    if (c >= (uint32_t)HOST_NBUF) CK(cudaStreamWaitEvent(hp.s_in, ev_free[b], 0));
    CK(cudaMemcpy2DAsync(d_in, n * 8, host_in + (uint64_t)j0 * stride_in, stride_in * 8, n * 8, cols,
                         cudaMemcpyHostToDevice, hp.s_in));
    CK(cudaEventRecord(ev_in[b], hp.s_in));
    // transform (dense coset-major layout inside the chunk buffer)
    CK(cudaStreamWaitEvent(hp.s_comp, ev_in[b], 0));
    CK(lde_fused(pl, d_in, d_out, log_n, cols, n, n, (uint64_t)cols * n, log_blowup, hp.s_comp));
    CK(cudaEventRecord(ev_comp[b], hp.s_comp));
    // copy out every coset block of the chunk
    CK(cudaStreamWaitEvent(hp.s_out, ev_comp[b], 0));
    for (uint64_t k = 0; k < nb; k++)
      CK(cudaMemcpy2DAsync(host_out + k * coset_stride + (uint64_t)j0 * stride_out, stride_out * 8,
                           d_out + k * (uint64_t)cols * n, n * 8, n * 8, cols, cudaMemcpyDeviceToHost, hp.s_out));
    CK(cudaEventRecord(ev_free[b], hp.s_out));
  }
  // the caller's stream (or s_out itself) continues once every step is done
  CK(cudaEventRecord(hp.done_in, hp.s_comp));
  if (caller_ordered) {
    CK(cudaEventRecord(hp.done_out, hp.s_out));
    CK(cudaStreamWaitEvent(caller, hp.done_in, 0));
    CK(cudaStreamWaitEvent(caller, hp.done_out, 0));
  } else {
    CK(cudaStreamWaitEvent(hp.s_out, hp.done_in, 0));
  }
#undef CK
  return cudaSuccess;
}

} // namespace bc

using namespace bc;

extern "C" cudaError_t bc_lde_host(const uint64_t *host_evals_bitrev, uint64_t *host_out, uint32_t log_n,
                                   uint32_t num_cols, uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride,
                                   uint32_t log_blowup, uint64_t *workspace, size_t workspace_bytes,
                                   uint32_t max_chunk_cols, cudaStream_t stream) {
  if (!lde_args_ok(log_n, num_cols, stride_in, stride_out, coset_stride, log_blowup)) return cudaErrorInvalidValue;
  if (num_cols == 0) return cudaSuccess;
  if (!host_evals_bitrev || !host_out || !workspace) return cudaErrorInvalidValue;
  if (!device_tables()) return cudaErrorInitializationError;
  const uint32_t chunk = host_chunk_cols(log_n, num_cols, log_blowup, workspace_bytes, max_chunk_cols);
  if (chunk == 0) return cudaErrorInvalidValue; // workspace smaller than NBUF single-column buffers
  const int dev = current_device();
  if (dev < 0 || dev >= HOST_MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_pipe_mutex[dev]);
  cudaError_t e = host_pipe_init(g_pipes[dev]);
  if (e != cudaSuccess) return e;
  return host_lde_enqueue(g_pipes[dev], host_evals_bitrev, host_out, log_n, num_cols, stride_in, stride_out,
                          coset_stride, log_blowup, workspace, chunk, true, stream);
}
