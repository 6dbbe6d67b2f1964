// host_lde.cuh -- the chunked host->device->host LDE pipeline (host_lde.cu),
// shared by bc_lde_host and the serving loop (server.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "lde.cuh"

namespace bc {

constexpr int HOST_NBUF = 3; // device buffers cycling through copy-in / compute / copy-out

// Three streams (copy-in, transform, copy-out) and the events that order them.
struct HostPipe {
  bool live = false;
  cudaStream_t s_in = nullptr, s_comp = nullptr, s_out = nullptr;
  cudaEvent_t ev[3 * HOST_NBUF] = {};
  cudaEvent_t entry = nullptr, done_in = nullptr, done_out = nullptr;
};

cudaError_t host_pipe_init(HostPipe &hp);
void host_pipe_destroy(HostPipe &hp);

// Columns per chunk so that HOST_NBUF chunk buffers fit workspace_bytes (0: none fit).
uint32_t host_chunk_cols(uint32_t log_n, uint32_t num_cols, uint32_t log_blowup, size_t workspace_bytes,
                         uint32_t max_chunk_cols);

// Enqueues a whole host LDE on the pipe's streams.  With `caller_ordered`,
// the work starts after what is already queued on `caller` and `caller` waits
// for its end (stream 0, the legacy default stream, is a valid caller);
// without it, the end is the pipe's copy-out stream.
cudaError_t host_lde_enqueue(HostPipe &hp, const uint64_t *host_in, uint64_t *host_out, uint32_t log_n,
                             uint32_t num_cols, uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride,
                             uint32_t log_blowup, uint64_t *workspace, uint32_t chunk, bool caller_ordered,
                             cudaStream_t caller);

} // namespace bc
