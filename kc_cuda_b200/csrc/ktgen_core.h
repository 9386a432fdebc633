// Seeded synthetic graph generators: the integer core shared by the CPU
// generator (ktgen.cpp) and the device generator (gen.cu).
//
// Every random quantity is a pure function of (seed, stream, counter), so the
// same graph comes out on any thread count, on the host or on the GPU.
//
// Conventions (they fix the expected answers, so they are part of the format):
//   * Random words: the SplitMix64 output finaliser (Steele, Lea, Flood,
//     "Fast splittable pseudorandom number generators", OOPSLA 2014) applied
//     to seed-, stream- and counter-dependent inputs.
//   * R-MAT (Chakrabarti, Zhan, Faloutsos, SDM 2004): draw i at scale S takes
//     S quadrant decisions, most significant bit first.  Decision l uses the
//     32-bit word (l even: low half, l odd: high half) of
//     word(seed, RMAT, i*ceil(S/2) + l/2).  Quadrant 0 (a) sets no bit,
//     1 (b) sets the column bit, 2 (c) sets the row bit, 3 (d) sets both.
//     Thresholds are a, a+b, a+b+c scaled by 2^32 and truncated.
//   * Uniform integer in [0, r): high 64 bits of word * r (no rejection).
//   * A draw (x, y) is the undirected edge {x, y}; self-loops and repeated
//     edges are dropped after all draws are made.
//   * Planted cliques: vertices chosen by Floyd's sampling algorithm
//     (Bentley, "Programming Pearls", CACM 30(9), 1987) on stream CLIQUE + j.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define KTG_HD __host__ __device__ __forceinline__
#else
#define KTG_HD static inline
#endif

enum {
  KTG_STREAM_RMAT = 1,
  KTG_STREAM_ER = 2,
  KTG_STREAM_CL_WEIGHT = 3,
  KTG_STREAM_CL_EDGE = 4,
  KTG_STREAM_BLOCK = 5,
  KTG_STREAM_MIX = 6,
  KTG_STREAM_CLIQUE = 64,
};

KTG_HD uint64_t ktg_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// One random 64-bit word for (seed, stream, counter).
KTG_HD uint64_t ktg_word(uint64_t seed, uint64_t stream, uint64_t ctr) {
  uint64_t s = ktg_mix64(seed * 0x9e3779b97f4a7c15ULL + stream * 0xd1b54a32d192ed03ULL + 0x632be59bd9b4e019ULL);
  return ktg_mix64(s + ctr * 0x9e3779b97f4a7c15ULL);
}

KTG_HD uint64_t ktg_mulhi64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return (uint64_t)(((__uint128_t)a * (__uint128_t)b) >> 64);
#endif
}

// Uniform integer in [0, r) from one word.
KTG_HD uint64_t ktg_below(uint64_t w, uint64_t r) { return ktg_mulhi64(w, r); }

// Quadrant thresholds of an R-MAT generator, scaled by 2^32.
typedef struct {
  uint64_t t0, t1, t2;
} ktg_rmat_t;

// a, b, c in parts per million (d = 1e6 - a - b - c).
KTG_HD ktg_rmat_t ktg_rmat_thresholds(uint32_t a_ppm, uint32_t b_ppm, uint32_t c_ppm) {
  ktg_rmat_t t;
  t.t0 = ((uint64_t)a_ppm << 32) / 1000000ULL;
  t.t1 = ((uint64_t)(a_ppm + b_ppm) << 32) / 1000000ULL;
  t.t2 = ((uint64_t)(a_ppm + b_ppm + c_ppm) << 32) / 1000000ULL;
  return t;
}

// Draw i of an R-MAT generator at the given scale: returns (row, col) packed
// as row << 32 | col.
KTG_HD uint64_t ktg_rmat_draw(uint64_t seed, ktg_rmat_t t, uint32_t scale, uint64_t i) {
  const uint64_t words = (scale + 1) / 2;
  uint32_t row = 0, col = 0;
  uint64_t w = 0;
  for (uint32_t l = 0; l < scale; ++l) {
    if ((l & 1) == 0) w = ktg_word(seed, KTG_STREAM_RMAT, i * words + l / 2);
    const uint64_t r = (l & 1) ? (w >> 32) : (w & 0xffffffffULL);
    const uint32_t rb = (r >= t.t1) ? 1u : 0u;                 // quadrants c, d
    const uint32_t cb = ((r >= t.t0 && r < t.t1) || r >= t.t2) ? 1u : 0u;  // b, d
    row = (row << 1) | rb;
    col = (col << 1) | cb;
  }
  return ((uint64_t)row << 32) | col;
}

// Draw i of a uniform (Erdos-Renyi G(n, M)) generator over n vertices.
KTG_HD uint64_t ktg_er_draw(uint64_t seed, uint64_t n, uint64_t i) {
  const uint64_t w0 = ktg_word(seed, KTG_STREAM_ER, 2 * i);
  const uint64_t w1 = ktg_word(seed, KTG_STREAM_ER, 2 * i + 1);
  return (ktg_below(w0, n) << 32) | ktg_below(w1, n);
}

// Canonical undirected key of a draw: min << 32 | max, or ~0 for a self-loop
// or an endpoint outside [0, n).
KTG_HD uint64_t ktg_canon(uint64_t xy, uint64_t n) {
  const uint32_t x = (uint32_t)(xy >> 32), y = (uint32_t)xy;
  if (x == y || x >= n || y >= n) return ~0ULL;
  return x < y ? (((uint64_t)x << 32) | y) : (((uint64_t)y << 32) | x);
}
