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

__device__ __forceinline__ uint64_t mul(uint64_t a, uint64_t b) { return reduce128(a * b, __umul64hi(a, b)); }

__device__ __forceinline__ uint64_t sqr(uint64_t a) { return mul(a, a); }

// Canonical representative in [0, p).
__device__ __forceinline__ uint64_t canon(uint64_t x) { return x >= P ? x - P : x; }

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
