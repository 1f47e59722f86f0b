// Shared device/host helpers for the parparpar_b200 CUDA kernels (sm_100a).
//
// Fields:
//   GF(2^16): x^16 + x^12 + x^3 + x + 1 (0x1100B), the PAR2 field
//             (reference gf16/gfmat_coeff.c:28).
//   GF(2^64): x^64 + x^4 + x^3 + x + 1 (low word 0x1B), the PAR3 field
//             (reference gf64/gf64_global.h:8, gf64/gf64_single.c:6-53).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#define PP_HD __host__ __device__ __forceinline__
#define PP_D __device__ __forceinline__

namespace pp {

constexpr uint32_t kGf16Poly = 0x1100B;
constexpr uint64_t kGf64Low = 0x1BULL;

// ---------------------------------------------------------------- GF(2^16)
// multiply by x
PP_HD uint32_t gf16_dbl(uint32_t v) {
  v <<= 1;
  return (v & 0x10000u) ? (v ^ kGf16Poly) : v;
}
// general product by shift-and-add (used only for table construction and
// the scalar pivot work of the inversion kernels, never in the region loops)
PP_HD uint16_t gf16_mul(uint32_t a, uint32_t b) {
  uint32_t r = 0;
#pragma unroll
  for (int i = 0; i < 16; i++) {
    if (b & (1u << i)) r ^= a;
    a = gf16_dbl(a);
  }
  return (uint16_t)r;
}
PP_HD int gf16_deg(uint32_t v) {  // degree of a nonzero polynomial
#ifdef __CUDA_ARCH__
  return 31 - __clz(v);
#else
  return 31 - __builtin_clz(v);
#endif
}
// inverse by the extended Euclidean algorithm over GF(2)[x] (binary-field
// inversion, Hankerson, Menezes and Vanstone, "Guide to Elliptic Curve
// Cryptography", Algorithm 2.48): at most 32 short steps, about a third of
// the dependent work of a^(2^16 - 2).  inverse(0) = 0.
PP_HD uint16_t gf16_inv_euclid(uint16_t a) {
  if (!a) return 0;
  uint32_t u = a, v = kGf16Poly, g1 = 1, g2 = 0;
  for (int it = 0; it < 40 && u != 1; it++) {  // terminates within 32 steps for a != 0
    int j = gf16_deg(u) - gf16_deg(v);
    if (j < 0) {
      const uint32_t t = u, tg = g1;
      u = v, v = t, g1 = g2, g2 = tg, j = -j;
    }
    u ^= v << j;
    g1 ^= g2 << j;
  }
  return (uint16_t)g1;
}
// inverse = a^(2^16 - 2); inverse(0) = 0
PP_HD uint16_t gf16_inv(uint16_t a) {
  uint32_t r = 1, s = a;
#pragma unroll 1
  for (int i = 1; i < 16; i++) {
    s = gf16_mul(s, s);
    r = gf16_mul(r, s);
  }
  return (uint16_t)(a ? r : 0);
}

// ---------------------------------------------------------------- GF(2^64)
PP_HD uint64_t gf64_dbl(uint64_t v) {
  return (v << 1) ^ ((uint64_t)((int64_t)v >> 63) & kGf64Low);
}
// Reduce a 128-bit carry-less product hi:lo modulo x^64+x^4+x^3+x+1.
PP_HD uint64_t gf64_reduce(uint64_t hi, uint64_t lo) {
  uint64_t t = hi ^ (hi >> 60) ^ (hi >> 61) ^ (hi >> 63);
  return lo ^ t ^ (t << 1) ^ (t << 3) ^ (t << 4);
}
// 32x32 -> 64 carry-less product from four integer multiplies per term pair
// with every 4th bit kept ("holes" of 3 zero bits absorb the carries: each
// partial sum has at most 8 terms, which fits in 4 bits).
PP_HD uint64_t clmul32(uint32_t a, uint32_t b) {
  const uint32_t m0 = 0x11111111u, m1 = 0x22222222u, m2 = 0x44444444u, m3 = 0x88888888u;
  uint64_t a0 = a & m0, a1 = a & m1, a2 = a & m2, a3 = a & m3;
  uint64_t b0 = b & m0, b1 = b & m1, b2 = b & m2, b3 = b & m3;
  const uint64_t M0 = 0x1111111111111111ull, M1 = 0x2222222222222222ull,
                 M2 = 0x4444444444444444ull, M3 = 0x8888888888888888ull;
  uint64_t z0 = (a0 * b0) ^ (a1 * b3) ^ (a2 * b2) ^ (a3 * b1);
  uint64_t z1 = (a0 * b1) ^ (a1 * b0) ^ (a2 * b3) ^ (a3 * b2);
  uint64_t z2 = (a0 * b2) ^ (a1 * b1) ^ (a2 * b0) ^ (a3 * b3);
  uint64_t z3 = (a0 * b3) ^ (a1 * b2) ^ (a2 * b1) ^ (a3 * b0);
  return (z0 & M0) | (z1 & M1) | (z2 & M2) | (z3 & M3);
}
// General GF(2^64) product (Karatsuba over 32-bit halves); used for scalar
// work (inverses, pivots, table seeds), not in the region loops.
PP_HD uint64_t gf64_mul(uint64_t a, uint64_t b) {
  uint32_t al = (uint32_t)a, ah = (uint32_t)(a >> 32);
  uint32_t bl = (uint32_t)b, bh = (uint32_t)(b >> 32);
  uint64_t lo = clmul32(al, bl);
  uint64_t hi = clmul32(ah, bh);
  uint64_t mid = clmul32(al ^ ah, bl ^ bh) ^ lo ^ hi;
  return gf64_reduce(hi ^ (mid >> 32), lo ^ (mid << 32));
}
// Squaring is GF(2)-linear: interleave zeros between the bits, then reduce.
PP_HD uint64_t spread32(uint32_t v) {
  uint64_t x = v;
  x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
  x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
  x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return x;
}
PP_HD uint64_t gf64_sqr(uint64_t a) {
  return gf64_reduce(spread32((uint32_t)(a >> 32)), spread32((uint32_t)a));
}
// Inverse by Itoh-Tsujii: a^-1 = (a^(2^63 - 1))^2, with a^(2^k - 1) built by
// the addition chain 1,2,3,6,12,15,30,31,62,63 (k doubling steps use
// squarings). inverse(0) = 0.
PP_HD uint64_t gf64_pow2k_mul(uint64_t x, int k, uint64_t y) {
#pragma unroll 1
  for (int i = 0; i < k; i++) x = gf64_sqr(x);
  return gf64_mul(x, y);
}
PP_HD uint64_t gf64_inv(uint64_t a) {
  // e_k := a^(2^k - 1)
  uint64_t e1 = a;
  uint64_t e2 = gf64_pow2k_mul(e1, 1, e1);
  uint64_t e3 = gf64_pow2k_mul(e2, 1, e1);
  uint64_t e6 = gf64_pow2k_mul(e3, 3, e3);
  uint64_t e12 = gf64_pow2k_mul(e6, 6, e6);
  uint64_t e15 = gf64_pow2k_mul(e12, 3, e3);
  uint64_t e30 = gf64_pow2k_mul(e15, 15, e15);
  uint64_t e31 = gf64_pow2k_mul(e30, 1, e1);
  uint64_t e62 = gf64_pow2k_mul(e31, 31, e31);
  uint64_t e63 = gf64_pow2k_mul(e62, 1, e1);
  return gf64_sqr(e63);
}

// ---------------------------------------------------------------- misc
PP_HD size_t ceil_div(size_t a, size_t b) { return (a + b - 1) / b; }

}  // namespace pp
