/*
 * bc_ntt.h -- C ABI of the B200 batched Goldilocks NTT / coset LDE library
 * (era-boojum-cuda_b200/libbc_ntt.so).
 *
 * Field: Goldilocks, p = 2^64 - 2^32 + 1.  Elements are u64 words; inputs may
 * be any u64 (non-canonical words are read mod p), outputs are canonical.
 * Matrices are column-major: column j of a matrix starts at ptr + j * stride
 * (u64 elements), exactly the layout of the reference's DeviceSlice matrices.
 * Transform calls are asynchronous on the given stream and return a
 * cudaError_t: argument violations that the reference rejects with
 * assert!/panic (src/ntt.rs:192-200, 309-320, 351-352) return
 * cudaErrorInvalidValue instead; launch failures return the CUDA error.
 *
 * Roots of unity are the generator-7 roots: w_{2^32} = 7^((p-1)/2^32) and
 * w_{2^k} = w_{2^32}^{2^(32-k)}.  Limits: 1 <= log_n <= 27 and
 * log_n + log_extension_degree <= 30 (the reference stops at 24,
 * src/context.rs:12).
 */
#ifndef BC_NTT_H
#define BC_NTT_H

#include <cuda_runtime_api.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces Context::create (src/context.rs:171-282).  Builds this library's
 * twiddle and power tables on the CURRENT device (about 1.7 MB); every other
 * call on that device requires it and returns cudaErrorInitializationError
 * without it.  The two counts keep the reference's bounds check (<= 24); the
 * table split itself is fixed.  Idempotent; thread-safe. */
cudaError_t bc_ntt_context_create(uint32_t powers_of_w_coarse_log_count, uint32_t powers_of_g_coarse_log_count);

/* Replaces Context::destroy (src/context.rs:284-296) for the current device. */
cudaError_t bc_ntt_context_destroy(void);

/* Replaces batch_ntt_internal (src/ntt.rs:179-191).
 * num_ntts columns of n = 2^log_n elements.
 *   bitrev_inputs = false: natural-order input, bit-reversed output
 *   bitrev_inputs = true : bit-reversed input, natural-order output
 *   inverse: inverse transform including the 1/n factor
 *   log_extension_degree e, coset_index k: coset c = 7 * w_{n*2^e}^k (c = 1 when
 *     e = 0); forward multiplies input i by c^i, inverse multiplies output i by
 *     c^-i, i being the natural index.
 * inputs == outputs (same strides) runs in place. */
cudaError_t bc_batch_ntt_internal(const uint64_t *inputs, uint64_t *outputs, uint32_t log_n, uint32_t num_ntts,
                                  uint64_t stride_between_input_arrays, uint64_t stride_between_output_arrays,
                                  bool bitrev_inputs, bool inverse, uint32_t log_extension_degree,
                                  uint32_t coset_index, cudaStream_t stream);

/* Replaces batch_ntt_out_of_place (src/ntt.rs:294-335).  The *_len arguments
 * are the element counts of the two device slices; the checks of
 * src/ntt.rs:309-320 apply (offset + n <= stride, len >= num_ntts * stride,
 * distinct buffers). */
cudaError_t bc_batch_ntt_out_of_place(const uint64_t *inputs_matrix, size_t inputs_len, uint64_t *outputs_matrix,
                                      size_t outputs_len, uint32_t log_n, uint32_t num_ntts, uint64_t inputs_offset,
                                      uint64_t outputs_offset, uint64_t stride_between_input_arrays,
                                      uint64_t stride_between_output_arrays, bool bitrev_inputs, bool inverse,
                                      uint32_t log_extension_degree, uint32_t coset_index, cudaStream_t stream);

/* Replaces batch_ntt_in_place (src/ntt.rs:338-369). */
cudaError_t bc_batch_ntt_in_place(uint64_t *inputs_matrix, size_t len, uint32_t log_n, uint32_t num_ntts,
                                  uint64_t inputs_offset, uint64_t stride_between_arrays, bool bitrev_inputs,
                                  bool inverse, uint32_t log_extension_degree, uint32_t coset_index,
                                  cudaStream_t stream);

/* batch_ntt_internal with an explicit pass plan instead of the built-in one
 * (the role of the reference's fixed PLANS table, src/ntt.rs:74-169, here
 * chosen by the autotuner).  Pass i covers pass_bits[i] index bits, listed
 * from the top bits down; pass_runs[i] is the run of consecutive low
 * positions a tile spans (1 for the pass that owns bit 0; 8 for windows of
 * <= 9 bits, 4 for 10, 2 for 11).  The bits must sum to log_n. */
cudaError_t bc_batch_ntt_with_plan(const uint64_t *inputs, uint64_t *outputs, uint32_t log_n, uint32_t num_ntts,
                                   uint64_t stride_in, uint64_t stride_out, bool bitrev_inputs, bool inverse,
                                   uint32_t log_extension_degree, uint32_t coset_index, const uint8_t *pass_bits,
                                   const uint8_t *pass_runs, uint32_t npasses, cudaStream_t stream);

/* ---- plans and the autotuner ------------------------------------------------
 * Replace the reference's fixed PLANS table (src/ntt.rs:74-169).  A plan says
 * how log_n index bits split into passes (the radix split), which run of
 * consecutive positions each pass's tiles span (the tile shape), and -- for
 * the fused LDE -- how many stages its middle kernel fuses (the top window).
 * Each device keeps a table keyed by (log_n, log_blowup), log_blowup = 0 for
 * the plain NTT; every entry point here uses the table's plan when present and
 * the built-in one otherwise.  bc_autotune times every candidate plan on the
 * current device (num_cols columns, reps timed runs after one warm-up; it
 * allocates and frees its own scratch and synchronises), then the launch knobs
 * of the fastest window split one at a time (column-group walk of the pass and
 * top-window CTAs, top-window table mode and tile double-buffering, CTAs per
 * SM of the low-window passes), and stores the fastest; report (optional)
 * receives one line per timed candidate. */
cudaError_t bc_autotune(uint32_t log_n, uint32_t log_blowup, uint32_t num_cols, uint32_t reps, char *report,
                        size_t report_len);
/* Text form of the current device's table, one entry per line:
 * "log_n log_blowup npasses K0 C0 [K1 C1 [K2 C2]]" (passes from the top bits),
 * followed by "k walk top_walk top_mode top_dbuf occ" when a launch knob is not
 * the built-in choice (0 = built-in; top_mode 1 resident, 2 prefetched,
 * 3 recomputed tables; top_dbuf 1 off, 2 on; occ 2 or 3 CTAs per SM). */
cudaError_t bc_plan_table_export(char *buf, size_t len, size_t *needed);
cudaError_t bc_plan_table_import(const char *text);
cudaError_t bc_plan_table_clear(void);

/* ---- coset low-degree extension ------------------------------------------
 * Input: num_cols columns of n = 2^log_n bit-reversed evaluations on the
 * subgroup H (column j at evals_bitrev + j * stride_in).  Output: for every
 * coset k < B = 2^log_blowup the bit-reversed evaluations of the same
 * polynomials on c_k H, c_k = 7 * w_{nB}^k, column j of coset k at
 * out + k * coset_stride + j * stride_out.  Blocks and columns must be
 * disjoint windows: coset-major (coset_stride >= (num_cols - 1) * stride_out
 * + n) or column-major (stride_out >= (B - 1) * coset_stride + n).
 * 1 <= log_blowup, log_n + log_blowup <= 27.  The input is not modified and
 * must not overlap the output.  No memory is allocated: the output block of
 * the last coset holds the intermediate values.
 *
 * The reference has no LDE function; these replace what its callers compose
 * from batch_ntt_internal (src/ntt.rs:179-191): one inverse b2n call, then
 * one forward n2b call per coset with (log_extension_degree = log_blowup,
 * coset_index = k), as benches/ntt.rs:110-116 does. */

/* The composition itself, one bc_batch_ntt_internal call per step. */
cudaError_t bc_lde_plain(const uint64_t *evals_bitrev, uint64_t *out, uint32_t log_n, uint32_t num_cols,
                         uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride, uint32_t log_blowup,
                         cudaStream_t stream);

/* Same result from fused kernels: inverse passes, one kernel that ends the
 * inverse transform, scales, and starts every coset's forward transform, then
 * the remaining forward passes of all cosets together. */
cudaError_t bc_lde_fused(const uint64_t *evals_bitrev, uint64_t *out, uint32_t log_n, uint32_t num_cols,
                         uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride, uint32_t log_blowup,
                         cudaStream_t stream);

/* bc_lde_fused that also records events[0] before its first kernel and
 * events[j + 1] after kernel j (up to num_events events), for per-kernel
 * timing; *num_kernels receives the number of kernels it launches. */
cudaError_t bc_lde_fused_profiled(const uint64_t *evals_bitrev, uint64_t *out, uint32_t log_n, uint32_t num_cols,
                                  uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride,
                                  uint32_t log_blowup, cudaStream_t stream, cudaEvent_t *events, uint32_t num_events,
                                  uint32_t *num_kernels);

/* Coset LDE from HOST memory to HOST memory (same layouts and meaning as
 * bc_lde_fused, host pointers).  No counterpart in the reference, whose
 * callers copy in, transform and copy out one step after the other.  Columns
 * are processed in chunks cycling through three device buffers carved from
 * the caller's `workspace` (device memory, workspace_bytes long; nothing is
 * allocated), so copy-in, transform and copy-out of consecutive chunks
 * overlap.  A chunk holds min(max_chunk_cols (0 = no limit), what fits)
 * columns; the workspace must hold at least 3 x 8 x n x (1 + 2^log_blowup)
 * bytes.  Host buffers should be pinned for the overlap.  Asynchronous:
 * `stream` waits for the whole operation; the host output is complete once
 * the stream has reached this point.  Calls sharing a workspace must not be
 * in flight at the same time. */
cudaError_t bc_lde_host(const uint64_t *host_evals_bitrev, uint64_t *host_out, uint32_t log_n, uint32_t num_cols,
                        uint64_t stride_in, uint64_t stride_out, uint64_t coset_stride, uint32_t log_blowup,
                        uint64_t *workspace, size_t workspace_bytes, uint32_t max_chunk_cols, cudaStream_t stream);

/* ---- uneven batches of LDE jobs in one persistent launch ------------------
 * No counterpart in the reference, whose callers issue 1 + B batch_ntt calls
 * per job (src/ntt.rs:179-191), each of 2-3 kernels, or log_n kernels for
 * log_n < 16 (src/ntt.rs:201-241).  Each job is an LDE with the meaning of
 * bc_lde_fused.  A plan schedules every job's kernels as work items of ONE
 * persistent kernel and captures the launch in a CUDA graph; run it as often
 * as needed (the job buffers are bound at plan time).  Plan creation
 * allocates the schedule on the current device (records, items, counters:
 * about 8 bytes per CTA-sized work item) and synchronises; bc_lde_batch_run
 * is asynchronous on the stream.  The kernel's dependency waits are bounded
 * (about 4 s each); bc_lde_batch_status returns status bit 0 if one expired,
 * in which case that run's outputs are invalid. */
typedef struct bc_lde_job {
  const uint64_t *evals_bitrev;
  uint64_t *out;
  uint64_t stride_in, stride_out, coset_stride;
  uint32_t log_n, num_cols, log_blowup, reserved;
} bc_lde_job;

typedef struct bc_lde_batch_plan bc_lde_batch_plan;

cudaError_t bc_lde_batch_plan_create(const bc_lde_job *jobs, uint32_t n_jobs, bc_lde_batch_plan **plan);
/* Same, except that a job whose every fused-LDE kernel would launch at least
 * standalone_min_ctas CTAs on its own is run as those kernels, on a branch of
 * the plan's graph forked beside the persistent kernel that runs all other
 * jobs (0: every job in the persistent kernel, as bc_lde_batch_plan_create).
 * Big jobs gain nothing from sharing a launch; small ones do. */
cudaError_t bc_lde_batch_plan_create_ex(const bc_lde_job *jobs, uint32_t n_jobs, uint32_t standalone_min_ctas,
                                        bc_lde_batch_plan **plan);
cudaError_t bc_lde_batch_run(bc_lde_batch_plan *plan, cudaStream_t stream);
/* Waits for the stream, then returns the status word of the plan's last run. */
cudaError_t bc_lde_batch_status(bc_lde_batch_plan *plan, cudaStream_t stream, uint32_t *status);
/* Sets how long one dependency wait of the plan's persistent kernel may take,
 * in SM clock cycles (0: the default, about 4 s).  A wait that runs out sets
 * status bit 0, skips its work item and lets the kernel finish, so a stalled
 * dependency ends as an error status instead of a hung GPU.  Waits for the
 * device first; later runs use the new limit. */
cudaError_t bc_lde_batch_plan_set_wait_limit(bc_lde_batch_plan *plan, uint64_t cycles);
cudaError_t bc_lde_batch_plan_info(const bc_lde_batch_plan *plan, uint32_t *n_records, uint32_t *n_items,
                                   uint32_t *grid);
cudaError_t bc_lde_batch_plan_destroy(bc_lde_batch_plan *plan);

/* No counterpart in the reference.  The same batch as a plan, run once, for
 * callers that cannot allocate device memory -- for example a prover that has
 * reserved nearly all of HBM for its own pool at start-up, or a
 * latency-critical submission path that cannot afford the device-wide
 * synchronisation of cudaMalloc/cudaFree.  It calls no cudaMalloc or
 * cudaFree: the schedule goes into a fixed 16 MiB array inside this library,
 * which every GPU that loads the library holds until the process exits.  A
 * batch whose schedule does not fit (about two million 4096-element work
 * items) returns cudaErrorInvalidValue before its work items are built.  The
 * first call on a device looks up the array's device address and the kernel's
 * occupancy and keeps them for the life of the process: they do not survive
 * cudaDeviceReset (or any other replacement of the device's primary context).
 * The schedule is copied from host memory the call frees on return, so a call
 * on a stream that is capturing returns cudaErrorStreamCaptureUnsupported and
 * enqueues nothing.  All calls on a device share the array: calls
 * whose work overlaps on the GPU (different streams, not ordered by events)
 * race and corrupt each other; calls ordered on one stream are safe.
 * status (optional): if non-null, the call waits for the stream and stores
 * the batch status word (bit 0: a bounded dependency wait expired and the
 * outputs are invalid). */
cudaError_t bc_lde_batch_noalloc(const bc_lde_job *jobs, uint32_t n_jobs, cudaStream_t stream, uint32_t *status);

/* ---- the integer ceiling of the transform arithmetic ------------------------
 * No counterpart in the reference.  Runs the transform kernels' radix-16 round
 * arithmetic (a DIT round of 15 general multiplications plus the shift
 * network, then a DIF round) on register-resident values in every resident
 * thread slot of the device, `iters` times, with no memory traffic: its
 * butterflies per second are the 32-bit integer issue roofline of the NTT
 * kernels.  bc_butterfly_peak_words gives the size of `out` (the final values,
 * written so that no arithmetic is dead); *butterflies receives the count the
 * launch performs.  Asynchronous on `stream`; time it with events. */
cudaError_t bc_butterfly_peak_words(size_t *out_words);
cudaError_t bc_butterfly_peak(uint64_t *out, size_t out_words, uint32_t iters, cudaStream_t stream,
                              uint64_t *butterflies);

/* ---- continuous-batching LDE server ---------------------------------------
 * No counterpart in the reference.  One server per device: it creates the
 * context, allocates a device arena of memory_budget_bytes ONCE, and runs
 * `slots` pipelines.  Requests (host buffers, pinned for overlap; dense
 * layouts: column j at j * n, coset k of column j at (k * num_cols + j) * n)
 * are admitted in arrival order whenever a slot is free and the arena has
 * room for their workspace -- requests arriving while others run join as
 * slots and memory free up, and their copies and kernels overlap on the GPU.
 * A request bigger than its arena share (budget / slots) is streamed through
 * in column chunks.  Submit never blocks on the GPU. */
typedef struct bc_lde_server_config {
  size_t memory_budget_bytes; /* device memory the server holds for requests */
  uint32_t slots;             /* requests on the GPU at once (1..64) */
  uint32_t max_chunk_cols;    /* 0: chunks as large as a slot's share allows */
} bc_lde_server_config;

typedef struct bc_lde_server_stats {
  uint64_t completed, pending, running;
  double p50_ms, p99_ms;         /* latency = completion - submit, last 65536 completed requests */
  double max_ms;                 /* worst latency of all completed requests */
  double span_s;                 /* first submit to last completion */
  double out_melem_per_s;        /* output elements of completed requests / span */
  size_t arena_largest_free;
} bc_lde_server_stats;

typedef struct bc_lde_server bc_lde_server;

cudaError_t bc_lde_server_create(const bc_lde_server_config *cfg, bc_lde_server **server);
cudaError_t bc_lde_server_submit(bc_lde_server *server, const uint64_t *host_evals_bitrev, uint64_t *host_out,
                                 uint32_t log_n, uint32_t num_cols, uint32_t log_blowup, uint64_t *request_id);
/* A request whose columns and output are already in device memory (dense
 * layouts as above), e.g. produced by earlier GPU work: no copies, no arena.
 * Device requests pending at the same moment whose output has at most
 * max_batch_elems elements (bc_lde_server_set_device_batching; default 2^22)
 * run together as ONE persistent batch launch (the batch kernel of
 * bc_lde_batch_*), larger ones as their own fused LDE, all on the server's
 * device stream with at most two launches in flight, so arrivals during a
 * launch join the next one.  The buffers must stay valid until the request is
 * done. */
cudaError_t bc_lde_server_submit_device(bc_lde_server *server, const uint64_t *dev_evals_bitrev, uint64_t *dev_out,
                                        uint32_t log_n, uint32_t num_cols, uint32_t log_blowup, uint64_t *request_id);
/* 0: no coalescing, every device request runs as its own fused LDE. */
cudaError_t bc_lde_server_set_device_batching(bc_lde_server *server, uint64_t max_batch_elems);
/* Batch launches made for device requests, the requests they carried, and the
 * device requests run as their own fused LDE. */
cudaError_t bc_lde_server_get_device_stats(bc_lde_server *server, uint64_t *batches, uint64_t *batched_requests,
                                           uint64_t *single_requests);
/* *state: 0 pending, 1 running, 2 done, 3 cancelled, 4 failed (the call returns the error). */
cudaError_t bc_lde_server_poll(bc_lde_server *server, uint64_t request_id, int *state, double *latency_ms);
/* Waits up to timeout_ms: cudaErrorTimeout if still unfinished, cudaErrorNotReady if cancelled. */
cudaError_t bc_lde_server_wait(bc_lde_server *server, uint64_t request_id, uint32_t timeout_ms, double *latency_ms);
/* Cancels a request not yet admitted (cudaErrorNotReady once it runs or ran). */
cudaError_t bc_lde_server_cancel(bc_lde_server *server, uint64_t request_id);
/* Forgets a done, cancelled or failed request: its id is unknown afterwards
 * (poll/wait return cudaErrorInvalidValue); cudaErrorNotReady while it is
 * pending or running.  A long-running caller releases what it has collected;
 * unreleased records are freed by destroy. */
cudaError_t bc_lde_server_release(bc_lde_server *server, uint64_t request_id);
cudaError_t bc_lde_server_get_stats(bc_lde_server *server, bc_lde_server_stats *stats);
/* Cancels pending requests, waits for running ones, frees everything. */
cudaError_t bc_lde_server_destroy(bc_lde_server *server);

#ifdef __cplusplus
}
#endif

#endif /* BC_NTT_H */
