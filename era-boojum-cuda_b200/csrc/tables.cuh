// tables.cuh -- compact on-device twiddle and power tables (the "context").
//
// Replaces the reference's Context (src/context.rs:157-297) and its
// __constant__ powers_data structs (native/context.cuh:11-48).  Instead of
// process-global __constant__ symbols, every kernel receives a DevTables
// struct by value, built once per device by bc_ntt_context_create.
//
// Roots of unity: w_{2^32} = 7^((p-1)/2^32), w_{2^k} = w_{2^32}^{2^(32-k)}.
//
// Twiddles.  A stage that pairs index bits at position a uses, for the pair
// whose index has upper part r = idx >> (a + 1), the twiddle
//     T[r] = w_{2^TW_LOG}^{brev_{TW_LOG-1}(r)}
// (the reference's bit-reversed twiddle convention, native/ntt.cu:23-35:
// T[r] does not depend on the stage or on log_n).  It is split in two levels,
// r = rh * 2^TW_FINE + rl:
//     T[r] = tw_lo[rl] * tw_hi[rh],
//     tw_lo[rl] = w_{2^(TW_FINE+1)}^{brev_TW_FINE(rl)},
//     tw_hi[rh] = w_{2^TW_LOG}^{brev_{TW_LOG-1-TW_FINE}(rh)}.
// The inverse tables hold the same with w^-1.
//
// Powers for coset scaling: g = 7 and w_{2^PW_LOG}, two levels each:
//     g^i   = g_lo[i & (2^G_FINE-1)] * g_hi[i >> G_FINE]      (i < 2^TW_LOG)
//     w^e   = w_lo[e & (2^PW_FINE-1)] * w_hi[e >> PW_FINE]     (e < 2^PW_LOG)
// with inverse variants for g^-i and w^-e.
#pragma once
#include <cstdint>

namespace bc {

constexpr int TW_LOG = 27;   // transform sizes up to 2^27 (regions r < 2^26)
constexpr int TW_FINE = 13;  // tw_lo: 2^13 entries, tw_hi: 2^13 entries
constexpr int G_FINE = 14;   // g_lo: 2^14, g_hi: 2^13  (i < 2^27)
constexpr int PW_LOG = 30;   // LDE domains up to 2^30 (log_n + log_blowup <= 30)
constexpr int PW_FINE = 15;  // w_lo: 2^15, w_hi: 2^15
constexpr int MAX_LOG_N = TW_LOG;

// The first eight twiddles are signed powers of two.  T[u] = w_16^{brev_3(u)}
// for u < 8, and w_16 = w_{2^32}^{2^28} = 2^156 (mod p), so T[u] = 2^e with e
// below (mod 192; 2^96 = -1, so e >= 96 is -2^(e-96)).  Inverse: 2^(192 - e).
// The context checks these against its tables when it is created.
__host__ __device__ constexpr int small_tw_exp(bool inv, int u) {
  constexpr int fwd[8] = {0, 48, 120, 168, 156, 12, 84, 132};
  return inv ? (192 - fwd[u]) % 192 : fwd[u];
}

// Twiddle of the Cooley-Tukey form of a DIF round's network: the stage that
// pairs round bit qq multiplies by w_{2^(qq+1)}^j (inverse: w^-j), j = the
// round bits below qq; w_{2^(qq+1)} = w_16^(2^(3-qq)) = 2^(156 * 2^(3-qq)).
__host__ __device__ constexpr int ct_tw_exp(bool inv, int qq, int j) {
  const int e = (156 * (j << (3 - qq))) % 192;
  return inv ? (192 - e) % 192 : e;
}

struct DevTables {
  const uint64_t *tw_lo[2]; // [0] forward, [1] inverse
  const uint64_t *tw_hi[2];
  const uint64_t *g_lo[2];  // [0] g^i, [1] g^-i
  const uint64_t *g_hi[2];
  const uint64_t *w_lo[2];  // [0] w^e, [1] w^-e  with w = w_{2^PW_LOG}
  const uint64_t *w_hi[2];
  uint64_t inv_pow2[TW_LOG + 1]; // 2^-k
};

} // namespace bc
