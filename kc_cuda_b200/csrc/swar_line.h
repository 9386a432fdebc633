// One TSV line decoded eight bytes at a time (SIMD within a register): the
// fast path of the device parser (parse.cu), also compiled for the host so
// that tests can check it against the byte-at-a-time grammar.
//
// Grammar (the reference parser's, src/kc_gpu.cpp:243-306): a byte is a
// digit when, read as a signed char, it is >= '0' (0x30..0x7f) and adds
// byte - '0'; a line's first two digit runs are x and y, the rest of the
// line is ignored, and a line without digits is blank.
//
// The fast path takes a 24-byte window that starts at the line and handles
// the common form: the runs are '0'..'9' only, at most 8 digits each, and y
// ends inside the window.  Anything else (a longer number, a grammar digit
// that is not '0'..'9', a run that reaches the window's end, a line with one
// number) returns false and the caller decodes the line a byte at a time.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define KT_HD __host__ __device__ __forceinline__
#else
#define KT_HD inline
#endif

namespace kt {
namespace swar {

constexpr uint64_t kHigh = 0x8080808080808080ull;
constexpr uint64_t kLow7 = 0x7f7f7f7f7f7f7f7full;

// Byte j of x with its high bit set -> bit j of the result (j = 0..7).  The
// multiplier moves high bit 8j+7 to bit 56+j; no two products overlap.
KT_HD uint32_t gather_high(uint64_t x) { return (uint32_t)(((x & kHigh) * 0x0002040810204081ull) >> 56); }

// High bit set in each byte equal to 0 (exact: no carries between bytes).
KT_HD uint64_t zero_bytes(uint64_t x) { return ~(((x & kLow7) + kLow7) | x) & kHigh; }

// '0'..'9'.
KT_HD uint64_t true_digits(uint64_t x) {
  const uint64_t t = x ^ 0x3030303030303030ull;  // digits -> 0..9
  return ~(((t & kLow7) + 0x7676767676767676ull) | t) & kHigh;
}

// 0x30..0x7f (a digit of the grammar).
KT_HD uint64_t grammar_digits(uint64_t x) { return ~x & ((x & kLow7) + 0x5050505050505050ull) & kHigh; }

KT_HD uint32_t ctz32(uint32_t x) {
#if defined(__CUDA_ARCH__)
  return (uint32_t)(__ffs((int)x) - 1);
#else
  return (uint32_t)__builtin_ctz(x);
#endif
}

// Value of the n (1..8) decimal digits at bytes [s, s+n) of the window w[3]
// (byte 0 of w[0] first).  The digits are right-aligned into one word with
// the most significant first, then combined pairwise: bytes into two-digit
// 16-bit lanes, those into four-digit 32-bit lanes, those into the value.
KT_HD uint32_t digits_value(const uint64_t* w, uint32_t s, uint32_t n) {
  const uint32_t q = s >> 3, r = (s & 7) * 8;
  // Selects rather than w[q]: the window stays in registers.
  const uint64_t lo = q == 0 ? w[0] : q == 1 ? w[1] : w[2];
  const uint64_t hi = q == 0 ? w[1] : q == 1 ? w[2] : 0ull;
  uint64_t d = lo >> r;
  if (r) d |= hi << (64 - r);
  d ^= 0x3030303030303030ull;
  d &= n == 8 ? ~0ull : ((1ull << (8 * n)) - 1);
  d <<= 8 * (8 - n);
  d = (d * 10 + (d >> 8)) & 0x00ff00ff00ff00ffull;
  d = (d * 100 + (d >> 16)) & 0x0000ffff0000ffffull;
  d = (d * 10000 + (d >> 32)) & 0xffffffffull;
  return (uint32_t)d;
}

// The line whose first 24 bytes are w[0..2]: true with *x, *y set (or
// *blank for a line without digits), false when the byte-at-a-time decoder
// must take it.
KT_HD bool decode_line(const uint64_t* w, uint32_t* x, uint32_t* y, bool* blank) {
  uint32_t G = 0, T = 0, N = 0;
  for (int i = 0; i < 3; ++i) {
    G |= gather_high(grammar_digits(w[i])) << (8 * i);
    T |= gather_high(true_digits(w[i])) << (8 * i);
    N |= gather_high(zero_bytes(w[i] ^ 0x0a0a0a0a0a0a0a0aull)) << (8 * i);
  }
  const uint32_t nl = N ? ctz32(N) : 24;
  const uint32_t before_nl = (1u << nl) - 1;
  *blank = false;
  if (!(G & before_nl)) {
    if (nl == 24) return false;  // no newline in sight: the line may go on
    *blank = true;
    return true;
  }
  const uint32_t xs = ctz32(G);
  const uint32_t xe = ctz32(~G & ~((1u << xs) - 1));  // bits 24.. of ~G are set: xe <= 24
  if (xe >= 24 || xe - xs > 8) return false;
  const uint32_t xm = ((1u << xe) - 1) & ~((1u << xs) - 1);
  if ((G ^ T) & xm) return false;
  const uint32_t rest = G & ~((1u << xe) - 1) & before_nl;
  if (!rest) return false;  // one number on the line (an error), or the line goes on
  const uint32_t ys = ctz32(rest);
  const uint32_t ye = ctz32(~G & ~((1u << ys) - 1));
  if (ye >= 24 || ye - ys > 8) return false;
  const uint32_t ym = ((1u << ye) - 1) & ~((1u << ys) - 1);
  if ((G ^ T) & ym) return false;
  *x = digits_value(w, xs, xe - xs);
  *y = digits_value(w, ys, ye - ys);
  return true;
}

}  // namespace swar
}  // namespace kt
