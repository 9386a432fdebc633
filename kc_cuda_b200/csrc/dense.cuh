// Dense mode: the working graph's alive adjacency as bitsets (row u = W
// 32-bit words), so |N(u) n N(v)| is a popcount of W word-ANDs.
//
// A warp takes 32 consecutive edges of a list.  Each lane fetches one edge's
// ends, then the warp walks the 32 edges: row u is cached in registers (R
// words per lane, W <= 32 R) and reused while consecutive edges share u (the
// edge lists are sorted by u), row v streams from L2.  Lane j keeps the
// count of the j-th edge, so results are written or pushed once per group.
#pragma once
#include "kt_device.cuh"

namespace kt {

template <int R>
__device__ __forceinline__ void dense_load_row(const uint32_t* __restrict__ bits, uint32_t W, uint32_t u,
                                               uint32_t (&w)[R]) {
  const uint32_t* p = bits + (uint64_t)u * W;
  const unsigned l = lane_id();
#pragma unroll
  for (int k = 0; k < R; ++k) {
    const uint32_t idx = k * 32 + l;
    w[k] = idx < W ? p[idx] : 0u;
  }
}

template <int R>
__device__ __forceinline__ uint32_t dense_and_popc(const uint32_t* __restrict__ bits, uint32_t W,
                                                   const uint32_t (&w)[R], uint32_t v) {
  const uint32_t* p = bits + (uint64_t)v * W;
  const unsigned l = lane_id();
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < R; ++k) {
    const uint32_t idx = k * 32 + l;
    if (idx < W) s += __popc(w[k] & p[idx]);
  }
  return warp_sum(s);
}

// One group of up to 32 list entries [base, min(base+32, cnt)).  Entries
// whose state is not kAlive (when state != nullptr) are skipped.  On return
// lane j holds (my_e, my_s) of the group's j-th entry, my_ok = counted.
template <int R>
__device__ __forceinline__ void dense_group(const uint32_t* __restrict__ list, uint64_t base, uint64_t cnt,
                                            const uint64_t* __restrict__ ends, const uint32_t* __restrict__ bits,
                                            uint32_t W, const uint32_t* __restrict__ state, uint32_t& my_e,
                                            uint32_t& my_s, bool& my_ok) {
  const unsigned l = lane_id();
  const uint64_t idx = base + l;
  uint32_t e = 0, u = 0, v = 0;
  bool ok = false;
  if (idx < cnt) {
    e = list ? list[idx] : (uint32_t)idx;
    ok = state == nullptr || state[e] == kAlive;
    if (ok) {
      const uint64_t k = ends[e];
      u = (uint32_t)(k >> 32);
      v = (uint32_t)k;
    }
  }
  my_e = e;
  my_ok = ok;
  my_s = 0;
  unsigned todo = __ballot_sync(kFull, ok);
  uint32_t w[R];
  uint32_t cu = 0xffffffffu;
  while (todo) {
    const int j = __ffs(todo) - 1;
    todo &= todo - 1;
    const uint32_t uj = __shfl_sync(kFull, u, j), vj = __shfl_sync(kFull, v, j);
    if (uj != cu) {
      dense_load_row<R>(bits, W, uj, w);
      cu = uj;
    }
    const uint32_t s = dense_and_popc<R>(bits, W, w, vj);
    if (l == (unsigned)j) my_s = s;
  }
}

// As dense_group, but an edge whose count can no longer reach `thr` is
// abandoned: the row is ANDed in four segments, and after each one the count
// so far plus the set bits left in row u bounds the result.  An abandoned
// edge reports a count below thr (not its support).
template <int R>
__device__ __forceinline__ void dense_group_capped(const uint32_t* __restrict__ list, uint64_t base, uint64_t cnt,
                                                   const uint64_t* __restrict__ ends,
                                                   const uint32_t* __restrict__ bits, uint32_t W, uint32_t thr,
                                                   uint32_t& my_e, uint32_t& my_s, bool& my_ok) {
  constexpr int Q = R / 4;
  const unsigned l = lane_id();
  const uint64_t idx = base + l;
  uint32_t e = 0, u = 0, v = 0;
  bool ok = false;
  if (idx < cnt) {
    e = list ? list[idx] : (uint32_t)idx;
    const uint64_t k = ends[e];
    u = (uint32_t)(k >> 32);
    v = (uint32_t)k;
    ok = true;
  }
  my_e = e;
  my_ok = ok;
  my_s = 0;
  unsigned todo = __ballot_sync(kFull, ok);
  uint32_t w[R];
  uint32_t seg[4] = {0, 0, 0, 0};
  uint32_t cu = 0xffffffffu;
  while (todo) {
    const int j = __ffs(todo) - 1;
    todo &= todo - 1;
    const uint32_t uj = __shfl_sync(kFull, u, j), vj = __shfl_sync(kFull, v, j);
    if (uj != cu) {
      dense_load_row<R>(bits, W, uj, w);
      cu = uj;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint32_t c = 0;
#pragma unroll
        for (int k = q * Q; k < (q + 1) * Q; ++k) c += __popc(w[k]);
        seg[q] = warp_sum(c);
      }
    }
    const uint32_t* p = bits + (uint64_t)vj * W;
    uint32_t found = 0, left = seg[0] + seg[1] + seg[2] + seg[3];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t c = 0;
#pragma unroll
      for (int k = q * Q; k < (q + 1) * Q; ++k) {
        const uint32_t wi = k * 32 + l;
        if (wi < W) c += __popc(w[k] & p[wi]);
      }
      found += warp_sum(c);
      left -= seg[q];
      if (found + left < thr) break;  // uniform: every lane holds the same sums
    }
    if (l == (unsigned)j) my_s = found;
  }
}

// Row-cache size (words per lane) for W words per row: 8, 16, 32 or 64.
inline int dense_regs(uint32_t W) { return W <= 256 ? 8 : W <= 512 ? 16 : W <= 1024 ? 32 : 64; }

}  // namespace kt
