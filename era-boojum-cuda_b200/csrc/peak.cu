// peak.cu -- the 32-bit integer ceiling of the NTT arithmetic, measured.
//
// The transform kernels are bound by 32-bit integer issue (the 64x64 -> 128
// multiplies, their reductions and the carry chains of the modular adds), not
// by HBM.  This kernel runs exactly their radix-16 round arithmetic -- the
// same dit_prepare / cnet / mul_powers of ntt_pass.cuh: a DIT round (15 general
// multiplications by the powers s^j, then the network of shift
// multiplications) followed by a DIF round (the inverse network, then 15
// multiplications) -- on values held in registers, with no loads, stores,
// shared-memory exchanges or barriers.  Butterflies per second of this loop
// is the roofline the transform kernels' butterfly rate is judged against.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/bc_ntt.h"
#include "ntt_pass.cuh"

namespace bc {

constexpr uint32_t PEAK_THREADS = 256;

__device__ __forceinline__ uint64_t splitmix(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// 64 butterflies per thread per iteration (one DIT and one DIF radix-16 round).
// The powers are arbitrary canonical field elements of the thread; `out`
// receives the 16 values so that no arithmetic is dead.
__global__ void __launch_bounds__(PEAK_THREADS, 2) butterfly_peak_kernel(uint64_t *out, uint32_t iters) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t x[16], pd[15], pi[15];
#pragma unroll
  for (int j = 0; j < 16; j++) x[j] = splitmix(((uint64_t)t << 6) + j);
#pragma unroll
  for (int j = 0; j < 15; j++) {
    pd[j] = gl::canon(splitmix(((uint64_t)t << 6) + 16 + j));
    pi[j] = gl::canon(splitmix(((uint64_t)t << 6) + 32 + j));
  }
#pragma unroll 1
  for (uint32_t it = 0; it < iters; it++) {
    dit_prepare<4, 0>(x, pd, true);
    cnet<false, false, 4, 0>(x);
    cnet<true, true, 4, 0>(x);
    mul_powers<4, 0>(x, pi);
  }
#pragma unroll
  for (int j = 0; j < 16; j++) out[(size_t)t * 16 + j] = x[j];
}

} // namespace bc

using namespace bc;

extern "C" cudaError_t bc_butterfly_peak(uint64_t *out, size_t out_words, uint32_t iters, cudaStream_t stream,
                                         uint64_t *butterflies) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, butterfly_peak_kernel, PEAK_THREADS, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  // every resident slot filled once: the loop's own issue rate, no tail
  const uint64_t grid = (uint64_t)per_sm * sms;
  const uint64_t need = grid * PEAK_THREADS * 16;
  if (butterflies) *butterflies = grid * PEAK_THREADS * 64ull * iters;
  if (!out) return out_words ? cudaErrorInvalidValue : cudaSuccess; // size query: *butterflies only
  if (out_words < need || iters == 0) return cudaErrorInvalidValue;
  butterfly_peak_kernel<<<(uint32_t)grid, PEAK_THREADS, 0, stream>>>(out, iters);
  return cudaGetLastError();
}

extern "C" cudaError_t bc_butterfly_peak_words(size_t *out_words) {
  if (!out_words) return cudaErrorInvalidValue;
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, butterfly_peak_kernel, PEAK_THREADS, 0);
  if (e != cudaSuccess) return e;
  *out_words = (size_t)per_sm * sms * PEAK_THREADS * 16;
  return cudaSuccess;
}
