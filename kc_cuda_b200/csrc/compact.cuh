// Order-preserving stream compaction of an index range by a predicate:
// count per 2048-index tile, scan the tile counts, then write each kept
// item's value at tile offset + block-scan rank.  No n-sized temporaries.
#pragma once
#include "kt_device.cuh"
#include "kt_internal.h"
#include "stages.h"

namespace kt {

constexpr unsigned kCompactThreads = 256;
constexpr unsigned kCompactItems = 8;
constexpr unsigned kCompactTile = kCompactThreads * kCompactItems;

template <class F>
__global__ void __launch_bounds__(kCompactThreads) k_compact_count(uint64_t n, F f, uint64_t* __restrict__ counts) {
  __shared__ uint64_t tmp[33];
  const uint64_t base = (uint64_t)blockIdx.x * kCompactTile;
  uint64_t s = 0;
#pragma unroll
  for (unsigned i = 0; i < kCompactItems; ++i) {
    const uint64_t j = base + i * kCompactThreads + threadIdx.x;
    if (j < n && f.keep(j)) ++s;
  }
  s = block_sum<uint64_t>(s, tmp);
  if (threadIdx.x == 0) counts[blockIdx.x] = s;
}

template <class F, typename T>
__global__ void __launch_bounds__(kCompactThreads) k_compact_write(uint64_t n, F f,
                                                                   const uint64_t* __restrict__ offs,
                                                                   T* __restrict__ out) {
  __shared__ uint64_t tmp[33];
  const uint64_t base = (uint64_t)blockIdx.x * kCompactTile;
  uint32_t flags = 0;
#pragma unroll
  for (unsigned i = 0; i < kCompactItems; ++i) {
    const uint64_t j = base + threadIdx.x * kCompactItems + i;
    if (j < n && f.keep(j)) flags |= 1u << i;
  }
  uint64_t total;
  uint64_t pos = offs[blockIdx.x] + block_excl_scan<uint64_t>((uint64_t)__popc(flags), tmp, &total);
#pragma unroll
  for (unsigned i = 0; i < kCompactItems; ++i)
    if (flags & (1u << i)) out[pos++] = f.value(base + threadIdx.x * kCompactItems + i);
}

// Returns the number of kept items; out receives f.value(i) for each kept i
// in increasing i.
template <class F, typename T>
uint64_t compact(Ctx* c, uint64_t n, const F& f, T* out) {
  if (n == 0) return 0;
  const uint64_t tiles = (n + kCompactTile - 1) / kCompactTile;
  DBuf counts(c, (tiles + 1) * sizeof(uint64_t));
  k_compact_count<F><<<(unsigned)tiles, kCompactThreads, 0, c->stream>>>(n, f, counts.as<uint64_t>());
  KT_LAUNCHED(c);
  zero(c, counts.as<uint64_t>() + tiles, sizeof(uint64_t));
  scan_u64(c, counts.as<uint64_t>(), counts.as<uint64_t>(), tiles + 1);
  k_compact_write<F, T><<<(unsigned)tiles, kCompactThreads, 0, c->stream>>>(n, f, counts.as<uint64_t>(), out);
  KT_LAUNCHED(c);
  return read_word<uint64_t>(c, counts.as<uint64_t>() + tiles);
}

}  // namespace kt
