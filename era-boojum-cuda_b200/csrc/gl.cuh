// gl.cuh -- Goldilocks field arithmetic for the NTT kernels (sm_100a).
//
// p = 2^64 - 2^32 + 1, EPS = 2^64 - p = 2^32 - 1.  Values are carried as raw
// u64 words in [0, 2^64) -- possibly non-canonical, exactly like the
// reference's base_field (native/goldilocks.cuh:90-183, whose add/sub/mul never
// reduce to [0, p)) -- and are made canonical only where a kernel stores a
// final result.  Every routine accepts any u64 operand.
//
// The 64x64 -> 128 multiply is written with mul.lo/mul.hi on u64 (the
// compiler emits 32-bit IMAD.WIDE chains); the 128 -> 64 reduction uses
// 2^64 = EPS and 2^96 = -1 (mod p) with explicit carry chains.  A carry is
// read back with addc after an add chain and a borrow with subc after a sub
// chain, so each flag is consumed by an instruction of its own kind.
#pragma once
#include <cstdint>

namespace gl {

constexpr uint64_t P = 0xffffffff00000001ull;
constexpr uint64_t EPS = 0xffffffffull;

__device__ __forceinline__ uint32_t lo32(uint64_t x) { return (uint32_t)x; }
__device__ __forceinline__ uint32_t hi32(uint64_t x) { return (uint32_t)(x >> 32); }

// a + b (mod p).  A carry out of 2^64 is worth EPS; a second carry can only
// happen when both operands are >= p and is absorbed by a second EPS.
__device__ __forceinline__ uint64_t add(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("{\n\t"
      ".reg .u32 a0, a1, b0, b1, r0, r1, c;\n\t"
      "mov.b64 {a0, a1}, %1;\n\t"
      "mov.b64 {b0, b1}, %2;\n\t"
      "add.cc.u32 r0, a0, b0;\n\t"
      "addc.cc.u32 r1, a1, b1;\n\t"
      "addc.u32 c, 0, 0;\n\t" // c = carry (0 or 1), read with addc after an add chain
      "neg.s32 c, c;\n\t"     // c = carry ? 0xffffffff : 0 = EPS or 0
      "add.cc.u32 r0, r0, c;\n\t"
      "addc.cc.u32 r1, r1, 0;\n\t"
      "addc.u32 c, 0, 0;\n\t"
      "neg.s32 c, c;\n\t"
      "add.cc.u32 r0, r0, c;\n\t"
      "addc.u32 r1, r1, 0;\n\t"
      "mov.b64 %0, {r0, r1};\n\t"
      "}"
      : "=l"(r)
      : "l"(a), "l"(b));
  return r;
}

// a - b (mod p).  A borrow is worth -EPS; a second borrow (only when b >= p)
// is absorbed the same way.
__device__ __forceinline__ uint64_t sub(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("{\n\t"
      ".reg .u32 a0, a1, b0, b1, r0, r1, c;\n\t"
      "mov.b64 {a0, a1}, %1;\n\t"
      "mov.b64 {b0, b1}, %2;\n\t"
      "sub.cc.u32 r0, a0, b0;\n\t"
      "subc.cc.u32 r1, a1, b1;\n\t"
      "subc.u32 c, 0, 0;\n\t" // c = borrow ? 0xffffffff : 0
      "sub.cc.u32 r0, r0, c;\n\t"
      "subc.cc.u32 r1, r1, 0;\n\t"
      "subc.u32 c, 0, 0;\n\t"
      "sub.cc.u32 r0, r0, c;\n\t"
      "subc.u32 r1, r1, 0;\n\t"
      "mov.b64 %0, {r0, r1};\n\t"
      "}"
      : "=l"(r)
      : "l"(a), "l"(b));
  return r;
}

// Reduce x = hi * 2^64 + lo (mod p) to [0, 2^64):
//   x = lo + hl * 2^64 + hh * 2^96 = lo - hh + hl * EPS.
// t0 = lo - hh borrows at most once (then -EPS, which cannot borrow again);
// t1 = hl * EPS = (hl << 32) - hl < 2^64; t0 + t1 carries at most once
// (then +EPS, which cannot carry again).
__device__ __forceinline__ uint64_t reduce128(uint64_t lo, uint64_t hi) {
  uint64_t r;
  asm("{\n\t"
      ".reg .u32 l0, l1, hl, hh, t0, t1, u0, u1, c;\n\t"
      "mov.b64 {l0, l1}, %1;\n\t"
      "mov.b64 {hl, hh}, %2;\n\t"
      "sub.cc.u32 t0, l0, hh;\n\t"
      "subc.cc.u32 t1, l1, 0;\n\t"
      "subc.u32 c, 0, 0;\n\t"
      "sub.cc.u32 t0, t0, c;\n\t"
      "subc.u32 t1, t1, 0;\n\t"
      // u = hl * EPS = (hl << 32) - hl : low word -hl, high word hl - (hl != 0)
      "sub.cc.u32 u0, 0, hl;\n\t"
      "subc.u32 u1, hl, 0;\n\t"
      "add.cc.u32 t0, t0, u0;\n\t"
      "addc.cc.u32 t1, t1, u1;\n\t"
      "addc.u32 c, 0, 0;\n\t"
      "neg.s32 c, c;\n\t"
      "add.cc.u32 t0, t0, c;\n\t"
      "addc.u32 t1, t1, 0;\n\t"
      "mov.b64 %0, {t0, t1};\n\t"
      "}"
      : "=l"(r)
      : "l"(lo), "l"(hi));
  return r;
}

// Canonical representative in [0, p).
__device__ __forceinline__ uint64_t canon(uint64_t x) { return x >= P ? x - P : x; }

__device__ __forceinline__ uint64_t mul(uint64_t a, uint64_t b) { return reduce128(a * b, __umul64hi(a, b)); }

// reduce128 with a canonical result: t0 = lo - hh is formed as there; for
// s = t0 + hl * EPS, a carry out of 2^64 leaves s - 2^64 + EPS < p, and
// without one s >= p exactly when s + EPS carries (then s + EPS - 2^64 = s - p).
// hl * EPS goes in with one multiply-add pair (mad.lo.cc / madc.hi.cc).
__device__ __forceinline__ uint64_t reduce128_canon(uint64_t lo, uint64_t hi) {
  uint64_t r;
  asm("{\n\t"
      ".reg .u32 l0, l1, hl, hh, t0, t1, v0, v1, c;\n\t"
      ".reg .pred q;\n\t"
      "mov.b64 {l0, l1}, %1;\n\t"
      "mov.b64 {hl, hh}, %2;\n\t"
      "sub.cc.u32 t0, l0, hh;\n\t"
      "subc.cc.u32 t1, l1, 0;\n\t"
      "subc.u32 c, 0, 0;\n\t"
      "sub.cc.u32 t0, t0, c;\n\t"
      "subc.u32 t1, t1, 0;\n\t"
      "mad.lo.cc.u32 t0, hl, 0xffffffff, t0;\n\t"
      "madc.hi.cc.u32 t1, hl, 0xffffffff, t1;\n\t"
      "addc.u32 c, 0, 0;\n\t"
      "add.cc.u32 v0, t0, 0xffffffff;\n\t"
      "addc.cc.u32 v1, t1, 0;\n\t"
      "addc.u32 c, c, 0;\n\t"
      "setp.ne.u32 q, c, 0;\n\t"
      "selp.b32 t0, v0, t0, q;\n\t"
      "selp.b32 t1, v1, t1, q;\n\t"
      "mov.b64 %0, {t0, t1};\n\t"
      "}"
      : "=l"(r)
      : "l"(lo), "l"(hi));
  return r;
}

// a * b reduced to [0, p).
__device__ __forceinline__ uint64_t mul_canon(uint64_t a, uint64_t b) {
  return reduce128_canon(a * b, __umul64hi(a, b));
}

// The same products for the round multiplications by powers (s^j), where many
// independent multiplications are in flight: the 128-bit product as a
// schoolbook chain of 32-bit multiply-adds with carries, and the reduction's
// hl * EPS term and final carry fix as multiply-adds, which moves work from
// the ALU pipe (the transform kernels' bound) to the multiplier pipe.  Their
// carry chains are longer, so dependent multiplications (running products)
// keep mul above.  Measured on B200 in the fused LDE (128 x 2^22, blowup 2):
// 31.35 -> 30.73 ms; used everywhere, including the running products, the
// kernels were no faster (the issue rate fell as much as the instructions).
__device__ __forceinline__ void mul128_chain(uint64_t a, uint64_t b, uint64_t &lo, uint64_t &hi) {
  asm("{\n\t"
      ".reg .u32 a0, a1, b0, b1, r0, r1, r2, r3;\n\t"
      "mov.b64 {a0, a1}, %2;\n\t"
      "mov.b64 {b0, b1}, %3;\n\t"
      "mul.lo.u32 r0, a0, b0;\n\t"
      "mul.hi.u32 r1, a0, b0;\n\t"
      "mad.lo.cc.u32 r1, a0, b1, r1;\n\t"
      "madc.hi.u32 r2, a0, b1, 0;\n\t"
      "mad.lo.cc.u32 r1, a1, b0, r1;\n\t"
      "madc.hi.cc.u32 r2, a1, b0, r2;\n\t"
      "madc.hi.u32 r3, a1, b1, 0;\n\t"
      "mad.lo.cc.u32 r2, a1, b1, r2;\n\t"
      "addc.u32 r3, r3, 0;\n\t"
      "mov.b64 %0, {r0, r1};\n\t"
      "mov.b64 %1, {r2, r3};\n\t"
      "}"
      : "=l"(lo), "=l"(hi)
      : "l"(a), "l"(b));
}

// reduce128 with hl * EPS added by a multiply-add chain (hl * EPS < 2^64, one
// carry at most); after a carry the low 64 bits are below 2^64 - 2^33 + 1, so
// the carry's EPS goes in with one wide multiply-add that cannot overflow.
__device__ __forceinline__ uint64_t reduce128_chain(uint64_t lo, uint64_t hi) {
  uint64_t r;
  asm("{\n\t"
      ".reg .u32 l0, l1, hl, hh, t0, t1, c;\n\t"
      ".reg .u64 t;\n\t"
      "mov.b64 {l0, l1}, %1;\n\t"
      "mov.b64 {hl, hh}, %2;\n\t"
      "sub.cc.u32 t0, l0, hh;\n\t"
      "subc.cc.u32 t1, l1, 0;\n\t"
      "subc.u32 c, 0, 0;\n\t"
      "sub.cc.u32 t0, t0, c;\n\t"
      "subc.u32 t1, t1, 0;\n\t"
      "mad.lo.cc.u32 t0, hl, 0xffffffff, t0;\n\t"
      "madc.hi.cc.u32 t1, hl, 0xffffffff, t1;\n\t"
      "addc.u32 c, 0, 0;\n\t"
      "mov.b64 t, {t0, t1};\n\t"
      "mad.wide.u32 t, c, 0xffffffff, t;\n\t"
      "mov.b64 %0, t;\n\t"
      "}"
      : "=l"(r)
      : "l"(lo), "l"(hi));
  return r;
}

__device__ __forceinline__ uint64_t mul_chain(uint64_t a, uint64_t b) {
  uint64_t lo, hi;
  mul128_chain(a, b, lo, hi);
  return reduce128_chain(lo, hi);
}

__device__ __forceinline__ uint64_t mul_chain_canon(uint64_t a, uint64_t b) {
  uint64_t lo, hi;
  mul128_chain(a, b, lo, hi);
  return reduce128_canon(lo, hi);
}

// a + b (mod p) for b < p: a + b < 2^64 + p, so one carry correction suffices.
__device__ __forceinline__ uint64_t add_bc(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("{\n\t"
      ".reg .u32 a0, a1, b0, b1, r0, r1, c;\n\t"
      "mov.b64 {a0, a1}, %1;\n\t"
      "mov.b64 {b0, b1}, %2;\n\t"
      "add.cc.u32 r0, a0, b0;\n\t"
      "addc.cc.u32 r1, a1, b1;\n\t"
      "addc.u32 c, 0, 0;\n\t"
      "neg.s32 c, c;\n\t"
      "add.cc.u32 r0, r0, c;\n\t"
      "addc.u32 r1, r1, 0;\n\t"
      "mov.b64 %0, {r0, r1};\n\t"
      "}"
      : "=l"(r)
      : "l"(a), "l"(b));
  return r;
}

// a - b (mod p) for b < p: a - b > -p, so one borrow correction suffices.
__device__ __forceinline__ uint64_t sub_bc(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("{\n\t"
      ".reg .u32 a0, a1, b0, b1, r0, r1, c;\n\t"
      "mov.b64 {a0, a1}, %1;\n\t"
      "mov.b64 {b0, b1}, %2;\n\t"
      "sub.cc.u32 r0, a0, b0;\n\t"
      "subc.cc.u32 r1, a1, b1;\n\t"
      "subc.u32 c, 0, 0;\n\t"
      "sub.cc.u32 r0, r0, c;\n\t"
      "subc.u32 r1, r1, 0;\n\t"
      "mov.b64 %0, {r0, r1};\n\t"
      "}"
      : "=l"(r)
      : "l"(a), "l"(b));
  return r;
}

// lo + h * EPS (mod p) for h < 2^32 (h < 2^32 - 1 for CANON).  h * EPS =
// (h << 32) - h <= 2^64 - 2^33 + 1 needs no reduction, and s = lo + h * EPS
// carries at most once; without CANON the carry is folded back as EPS and the
// result is only < 2^64.  CANON forms s' = lo + (h + 1) * EPS = s + EPS < 2^65
// instead: s' carries exactly when s >= p, and then s' - 2^64 = s - p;
// without a carry the result is s' - EPS = s < p.  Either way lo + h * EPS is
// one multiply-add pair (mad.lo.cc / madc.hi.cc by 0xffffffff), which runs on
// the multiplier pipe and leaves the integer ALU, the transforms' bound, to
// the carries.
template <bool CANON>
__device__ __forceinline__ uint64_t add_h_eps(uint64_t lo, uint32_t h) {
  uint64_t r;
  if constexpr (CANON) {
    asm("{\n\t"
        ".reg .u32 l0, l1, h1, m;\n\t"
        "mov.b64 {l0, l1}, %1;\n\t"
        "add.u32 h1, %2, 1;\n\t"
        "mad.lo.cc.u32 l0, h1, 0xffffffff, l0;\n\t"
        "madc.hi.cc.u32 l1, h1, 0xffffffff, l1;\n\t"
        "addc.u32 m, 0xffffffff, 0;\n\t"
        "sub.cc.u32 l0, l0, m;\n\t"
        "subc.u32 l1, l1, 0;\n\t"
        "mov.b64 %0, {l0, l1};\n\t"
        "}"
        : "=l"(r)
        : "l"(lo), "r"(h));
  } else {
    asm("{\n\t"
        ".reg .u32 l0, l1, c;\n\t"
        "mov.b64 {l0, l1}, %1;\n\t"
        "mad.lo.cc.u32 l0, %2, 0xffffffff, l0;\n\t"
        "madc.hi.cc.u32 l1, %2, 0xffffffff, l1;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "neg.s32 c, c;\n\t"
        "add.cc.u32 l0, l0, c;\n\t"
        "addc.u32 l1, l1, 0;\n\t"
        "mov.b64 %0, {l0, l1};\n\t"
        "}"
        : "=l"(r)
        : "l"(lo), "r"(h));
  }
  return r;
}

// x * 2^E (mod p) for a compile-time 0 < E < 96 and any u64 x, without a
// multiply.  x << E spans at most 160 bits, words v0..v4 (32 bits each), and
//   v = v0 + v1 2^32 + v2 2^64 + v3 2^96 + v4 2^128
//     = v0 - v2 - v3 + (v1 + v2 - v4) 2^32        (2^64 = 2^32 - 1, 2^96 = -1)
// of which at most three words are non-zero for a given E.
//   E < 32:       v = lo + h EPS, lo = x << E (64 bits), h = x >> (64 - E);
//   32 <= E < 64: v1 2^32 + v2 EPS - v3, s = E - 32;
//   64 <= E < 96: v2 EPS - (v3 + v4 2^32), s = E - 64.
// Each product by EPS is a 32-bit multiply(-add) on the multiplier pipe.
// CANON: the result is reduced to [0, p); for E >= 32 it always is (bounds at
// each case), so only E < 32 pays for it.
template <int E, bool CANON = false>
__device__ __forceinline__ uint64_t mul_pow2(uint64_t x) {
  static_assert(E > 0 && E < 96, "mul_pow2: 0 < E < 96");
  if constexpr (E < 32) {
    return add_h_eps<CANON>(x << E, (uint32_t)(x >> (64 - E)));
  } else if constexpr (E < 64) {
    constexpr int s = E - 32;
    const uint64_t xs = x << s;
    const uint32_t v1 = (uint32_t)xs, v2 = (uint32_t)(xs >> 32), v3 = s ? (uint32_t)(x >> (64 - s)) : 0u;
    uint64_t r;
    // T = v2 EPS + (v1 2^32 + EPS - v3) (carry c), v = T - EPS: subtract
    // (1 - c) EPS, then EPS once more on a borrow (only when v1 = v2 = 0).
    // Canonical: T < 2^65 - 2^33, so with c = 1 the result T - 2^64 < p; with
    // c = 0, T - EPS <= p - 1, and after a borrow T - EPS + p is in [p - EPS, p).
    asm("{\n\t"
        ".reg .u32 z, r0, r1, m, b;\n\t"
        "not.b32 z, %3;\n\t"
        "mad.lo.cc.u32 r0, %2, 0xffffffff, z;\n\t"
        "madc.hi.cc.u32 r1, %2, 0xffffffff, %1;\n\t"
        "addc.u32 m, 0xffffffff, 0;\n\t"
        "sub.cc.u32 r0, r0, m;\n\t"
        "subc.cc.u32 r1, r1, 0;\n\t"
        "subc.u32 b, 0, 0;\n\t"
        "sub.cc.u32 r0, r0, b;\n\t"
        "subc.u32 r1, r1, 0;\n\t"
        "mov.b64 %0, {r0, r1};\n\t"
        "}"
        : "=l"(r)
        : "r"(v1), "r"(v2), "r"(v3));
    return r;
  } else {
    constexpr int s = E - 64;
    // v = y0 EPS - Y with y0 = (x << s) mod 2^32 and Y = x >> (32 - s); a borrow
    // leaves 2^64 + v >= 2^63 and is folded back by subtracting EPS.
    // Canonical: y0 EPS <= p - 2^32, so without a borrow v < p, and after one
    // v + p is in (p - 2^63, p).
    const uint32_t y0 = (uint32_t)x << s;
    const uint64_t t = (uint64_t)y0 * 0xffffffffull, Y = x >> (32 - s);
    uint64_t r;
    asm("{\n\t"
        ".reg .u32 t0, t1, y0, y1, r0, r1, b;\n\t"
        "mov.b64 {t0, t1}, %1;\n\t"
        "mov.b64 {y0, y1}, %2;\n\t"
        "sub.cc.u32 r0, t0, y0;\n\t"
        "subc.cc.u32 r1, t1, y1;\n\t"
        "subc.u32 b, 0, 0;\n\t"
        "sub.cc.u32 r0, r0, b;\n\t"
        "subc.u32 r1, r1, 0;\n\t"
        "mov.b64 %0, {r0, r1};\n\t"
        "}"
        : "=l"(r)
        : "l"(t), "l"(Y));
    return r;
  }
}

__device__ __forceinline__ uint64_t sqr(uint64_t a) { return mul(a, a); }

__device__ __forceinline__ uint64_t pow(uint64_t b, uint32_t e) {
  uint64_t r = 1;
  while (e) {
    if (e & 1) r = mul(r, b);
    b = mul(b, b);
    e >>= 1;
  }
  return r;
}

} // namespace gl
