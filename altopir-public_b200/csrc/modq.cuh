// modq.cuh -- exact arithmetic modulo Q = 4294955009 = 2^32 - 12287 on 32-bit residues, shared by host and device.
//
// All inputs are residues in [0, Q) unless stated.  Q > 2^31, so sums overflow 32 bits; the helpers use the wrap of
// unsigned arithmetic, which subtracts 2^32 = Q + 12287, to stay in 32-bit registers.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define ALTO_HD __host__ __device__ __forceinline__
#else
#define ALTO_HD inline
#endif

namespace alto {

constexpr uint32_t kQ32 = 4294955009u;
constexpr uint32_t kFold = 12287u;  // 2^32 mod Q

ALTO_HD uint32_t umin_u32(uint32_t a, uint32_t b) { return a < b ? a : b; }

// (a + b) mod Q.  d = s - Q (mod 2^32).  On a carry the true sum a + b = s + 2^32 >= Q, and d = s + 12287 is that
// sum minus Q.  Without a carry, d < s exactly when s >= Q (below Q the subtraction wraps to s + 12287 > s), so the
// smaller of s and d is the residue.
ALTO_HD uint32_t add_q(uint32_t a, uint32_t b) {
  const uint32_t s = a + b, d = s - kQ32;
  return s < a ? d : umin_u32(s, d);
}

// (a - b) mod Q.
ALTO_HD uint32_t sub_q(uint32_t a, uint32_t b) {
  const uint32_t d = a - b;
  return a < b ? d + kQ32 : d;
}

// x mod Q for any 64-bit x: x = h 2^32 + l = 12287 h + l (mod Q); two folds leave x < 2^32 + 2^28, whose high word
// h is 0 or 1.  With h = 1, x - Q = l + 12287 < Q (l < 2^28); with h = 0 the smaller of l and l - Q (mod 2^32) is the
// residue, as in add_q.
ALTO_HD uint32_t red_q64(uint64_t x) {
  x = (x >> 32) * kFold + (x & 0xffffffffull);
  x = (x >> 32) * kFold + (x & 0xffffffffull);
  const uint32_t t = (uint32_t)x + (uint32_t)(x >> 32) * kFold;
  return umin_u32(t, t - kQ32);
}

// One fold of a 64-bit x: h 2^32 + l -> 12287 h + l, congruent to x mod Q and below 2^46 (not reduced).
ALTO_HD uint64_t fold_q64(uint64_t x) { return (x >> 32) * kFold + (x & 0xffffffffull); }

// (a * b) mod Q for any 32-bit a, b.
ALTO_HD uint32_t mul_q(uint32_t a, uint32_t b) { return red_q64((uint64_t)a * b); }

// 2^-l mod Q: (Q + 1) / 2 is the inverse of 2.
ALTO_HD uint32_t inv_pow2_q(int l) {
  uint32_t r = 1;
  for (int i = 0; i < l; ++i) r = mul_q(r, (kQ32 + 1u) / 2u);
  return r;
}

// floor(u / Q) for u < 2^53.  u / 2^32 <= u / Q, so q0 = u >> 32 undershoots; the remainder u - q0 Q =
// (u mod 2^32) + 12287 q0 < 2^32 + 2^35 leaves at most a few more multiples of Q, found the same way.
ALTO_HD uint64_t div_q(uint64_t u) {
  const uint64_t q0 = u >> 32;
  uint64_t r = (u & 0xffffffffull) + q0 * kFold;
  const uint64_t q1 = r >> 32;
  r = (r & 0xffffffffull) + q1 * kFold;
  return q0 + q1 + (r >= kQ32 ? 1u : 0u);
}

// Centred rescale of v in [0, Q) from Q to q1 (q1 < 2^21), rounding half away from zero, result in [0, q1):
// c = v or v - Q (centred), t = trunc((c q1 +- floor(Q/2)) / Q), t + q1 when negative, t - q1 when t = q1
// (src/amx_kernels.cpp:522-529; the reference divides in double precision, which rounds to the same integer).
ALTO_HD uint32_t rescale_q(uint32_t v, uint32_t q1) {
  constexpr uint64_t half = kQ32 / 2u;
  const bool neg = v >= (uint32_t)half;
  const uint32_t mag = neg ? kQ32 - v : v;  // |c| <= ceil(Q / 2)
  // |trunc(x / Q)| = floor((|c| q1 + floor(Q/2)) / Q) <= (q1 + 1) / 2 + 1: below q1 for every q1 >= 2, so a negative
  // c maps to q1 - t (0 for t = 0) and a non-negative one to t
  const uint32_t t = (uint32_t)div_q((uint64_t)mag * q1 + half);
  return neg ? (t ? q1 - t : 0u) : (t >= q1 ? t - q1 : t);
}

}  // namespace alto
