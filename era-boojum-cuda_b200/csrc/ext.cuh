// ext.cuh -- the quadratic extension F_p[x] / (x^2 - 7) of the Goldilocks field
// (the reference's native/goldilocks_extension.cuh:8-80: non-residue 7), and
// base-field inversion.  Values are raw u64 words like gl.cuh's.
#pragma once
#include "gl.cuh"

namespace bc {

struct Ext {
  uint64_t c0, c1; // c0 + c1 x
};

// 7 x = 8 x - x.
__device__ __forceinline__ uint64_t mul7(uint64_t x) { return gl::sub(gl::mul_pow2<3>(x), x); }

__device__ __forceinline__ Ext ext_add(const Ext &a, const Ext &b) { return {gl::add(a.c0, b.c0), gl::add(a.c1, b.c1)}; }

// (a0 + a1 x)(b0 + b1 x) = a0 b0 + 7 a1 b1 + ((a0 + a1)(b0 + b1) - a0 b0 - a1 b1) x
__device__ __forceinline__ Ext ext_mul(const Ext &a, const Ext &b) {
  const uint64_t a0b0 = gl::mul(a.c0, b.c0), a1b1 = gl::mul(a.c1, b.c1);
  const uint64_t cross = gl::mul(gl::add(a.c0, a.c1), gl::add(b.c0, b.c1));
  return {gl::add(a0b0, mul7(a1b1)), gl::sub(gl::sub(cross, a0b0), a1b1)};
}

__device__ __forceinline__ Ext ext_mul_base(const Ext &a, uint64_t b) { return {gl::mul(a.c0, b), gl::mul(a.c1, b)}; }

// a^(p-2): the inverse of a != 0 and 0 for a = 0 (square-and-multiply over
// the bits of p - 2 = 0xfffffffeffffffff).
__device__ __forceinline__ uint64_t inv(uint64_t a) {
  uint64_t r = 1, b = a;
  uint64_t e = gl::P - 2;
#pragma unroll 1
  while (e) {
    if (e & 1) r = gl::mul(r, b);
    e >>= 1;
    if (e) b = gl::sqr(b);
  }
  return r;
}

// Norm c0^2 - 7 c1^2 (non-zero for a non-zero element: x^2 - 7 is irreducible).
__device__ __forceinline__ uint64_t ext_norm(const Ext &a) { return gl::sub(gl::sqr(a.c0), mul7(gl::sqr(a.c1))); }

} // namespace bc
