// Dense mode: the working graph's alive adjacency as bitsets (row u = W
// 32-bit words), so |N(u) n N(v)| is a popcount of W word-ANDs.
//
// A batched union of graphs keeps one block of bitsets per graph (block
// diagonal): row u has the words of its own graph's size, starts at word
// roff[u], and bit j of it is vertex cbase[u] + j.  Two ends of an edge are
// in the same graph, so their rows have the same length.
//
// A warp takes 32 consecutive edges of a list.  Each lane fetches one edge's
// ends, then the warp walks the 32 edges: row u is copied into the warp's
// slice of shared memory (W words) and reused while consecutive edges share
// u (the lists are tile-ordered by (u block, v block, u, v)); for exact
// counts up to four edges that share row u are counted together, each lane
// reading a vector of row u from shared memory once and ANDing it with the
// same vector of each row v, which stream from L2 with every lane on
// consecutive vectors; capped counts run two edges that share row u side by
// side, one per half of the warp.
// Keeping row u in shared memory rather than registers leaves the kernels at
// few registers, so many warps hide the L2 latency.  Lane j keeps the count
// of the j-th edge, so results are written or pushed once per group.
#pragma once
#include "kt_device.cuh"
#include "subgraph.h"

namespace kt {

// Row addressing of the bitsets: uniform rows of W words (roff == nullptr),
// or per-graph rows (roff, rw, cbase per vertex; W = the longest row).
struct DenseRows {
  uint32_t* bits;
  uint32_t W;
  const uint64_t* roff;
  const uint32_t* rw;
  const uint32_t* cbase;
  const uint32_t* sbits;  // rows as built (may be null)
  const uint32_t* spre;   // set bits of the built row before each word
  // Position of neighbour column `col` in row u's sorted adjacency.
  __device__ __forceinline__ uint32_t rank(uint32_t u, uint32_t col) const {
    const uint64_t w = off(u) + (col >> 5);
    return spre[w] + __popc(sbits[w] & ((1u << (col & 31)) - 1u));
  }
  __device__ __forceinline__ uint64_t off(uint32_t u) const { return roff ? roff[u] : (uint64_t)u * W; }
  __device__ __forceinline__ uint32_t words(uint32_t u) const { return roff ? rw[u] : W; }
  // Bit position of neighbour v in row u.
  __device__ __forceinline__ uint32_t col(uint32_t u, uint32_t v) const { return roff ? v - cbase[u] : v; }
};

inline DenseRows dense_rows(const Sub& s) {
  const bool grouped = s.roff.get() != nullptr;
  return DenseRows{const_cast<uint32_t*>(s.bits.as<uint32_t>()), s.W,
                   grouped ? s.roff.as<uint64_t>() : nullptr, grouped ? s.rw.as<uint32_t>() : nullptr,
                   grouped ? s.vbase.as<uint32_t>() : nullptr, s.sbits.as<uint32_t>(), s.spre.as<uint32_t>()};
}

// Rows are whole 16-byte vectors (W a multiple of 4, rows 16-byte aligned;
// the padding words stay zero).

// Shared memory a block of `threads` needs for rows of W words.
inline size_t dense_smem_bytes(uint32_t W, unsigned threads) { return (size_t)(threads / 32) * W * 4; }

__device__ __forceinline__ void dense_load_row(const uint32_t* __restrict__ p, uint32_t W, uint32_t* su) {
  const uint4* p4 = reinterpret_cast<const uint4*>(p);
  uint4* s4 = reinterpret_cast<uint4*>(su);
  for (uint32_t i = lane_id(); i < W / 4; i += 32) s4[i] = p4[i];
  __syncwarp();
}

__device__ __forceinline__ uint32_t popc_and4(uint4 a, uint4 b) {
  return __popc(a.x & b.x) + __popc(a.y & b.y) + __popc(a.z & b.z) + __popc(a.w & b.w);
}

// popcount(row u & row v) over words [w0, w1) (multiples of 4) by one half
// of the warp (16 lanes, 16-byte vectors); `active` false contributes 0.
// Every lane of the warp must call it; each lane gets its half's total.
__device__ __forceinline__ uint32_t half_and_popc(const uint32_t* __restrict__ p, const uint32_t* su, uint32_t w0,
                                                  uint32_t w1, bool active) {
  uint32_t s = 0;
  if (active) {
    const uint4* p4 = reinterpret_cast<const uint4*>(p);
    const uint4* s4 = reinterpret_cast<const uint4*>(su);
    uint32_t i = w0 / 4 + (lane_id() & 15);
    const uint32_t e = w1 / 4;
    for (; i + 3 * 16 < e; i += 4 * 16) {
      uint4 a[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) a[k] = __ldcg(p4 + i + 16 * k);
#pragma unroll
      for (int k = 0; k < 4; ++k) s += popc_and4(s4[i + 16 * k], a[k]);
    }
    for (; i < e; i += 16) s += popc_and4(s4[i], __ldcg(p4 + i));
  }
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
  return s;
}

// popcount(row u & row v_q) over the 16-byte vectors [i0, i1) of up to NQ
// rows v_q at once (row q taking part when act[q]; the loads of the others
// are predicated off): each lane reads a vector of row u from shared memory
// once and ANDs it with the same vector of every row v_q (two vectors per row
// in flight per lane), so edges that share row u share its shared-memory
// reads.  Every lane of the warp must call it; out[q] gets row q's warp total
// (0 when it takes no part).
template <int NQ>
__device__ __forceinline__ void rows_and_popc(const DenseRows& R, const uint32_t* vq, const bool* act,
                                              const uint32_t* su, uint32_t i0, uint32_t i1, uint32_t* out) {
  const uint4* pv[NQ];
  uint32_t c[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    pv[q] = reinterpret_cast<const uint4*>(R.bits + R.off(act[q] ? vq[q] : vq[0]));
    c[q] = 0;
  }
  const uint4* s4 = reinterpret_cast<const uint4*>(su);
  const uint4 z = make_uint4(0u, 0u, 0u, 0u);
  uint32_t i = i0 + lane_id();
  for (; i + 32 < i1; i += 64) {
    const uint4 a0 = s4[i], a1 = s4[i + 32];
    uint4 b0[NQ], b1[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      b0[q] = act[q] ? __ldcg(pv[q] + i) : z;
      b1[q] = act[q] ? __ldcg(pv[q] + i + 32) : z;
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) c[q] += popc_and4(a0, b0[q]) + popc_and4(a1, b1[q]);
  }
  if (i < i1) {
    const uint4 a = s4[i];
#pragma unroll
    for (int q = 0; q < NQ; ++q) c[q] += popc_and4(a, act[q] ? __ldcg(pv[q] + i) : z);
  }
#pragma unroll
  for (int q = 0; q < NQ; ++q) out[q] = act[q] ? warp_sum(c[q]) : 0u;
}

// Edge j and up to NQ-1 more edges of the group that share its row u (they
// follow it in the tile-ordered list): slot q gets the lane jq[q] and column
// vq[q] of one of them (act[q]), and they leave `todo`.  Warp-uniform.
template <int NQ>
__device__ __forceinline__ void take_same_row(unsigned& todo, uint32_t u, uint32_t v, uint32_t uj, int j,
                                              uint32_t vj, int* jq, uint32_t* vq, bool* act) {
  jq[0] = j;
  vq[0] = vj;
  act[0] = true;
#pragma unroll
  for (int q = 1; q < NQ; ++q) {
    jq[q] = -1;
    vq[q] = vj;
    act[q] = false;
    if (todo) {
      const int cand = __ffs(todo) - 1;
      const uint32_t uc = __shfl_sync(kFull, u, cand), vc = __shfl_sync(kFull, v, cand);
      if (uc == uj && act[q - 1]) {
        jq[q] = cand;
        vq[q] = vc;
        act[q] = true;
        todo &= todo - 1;
      }
    }
  }
}

// One group of up to 32 list entries [base, min(base+32, cnt)).  Entries
// whose state is not kAlive (when state != nullptr) are skipped.  On return
// lane j holds (my_e, my_s) of the group's j-th entry, my_ok = counted.
// su is this warp's W-word slice of shared memory.
template <int NQ = 4>
__device__ __forceinline__ void dense_group(const uint32_t* __restrict__ list, uint64_t base, uint64_t cnt,
                                            const uint64_t* __restrict__ ends, const DenseRows& R,
                                            const uint32_t* __restrict__ state, uint32_t* su, uint32_t& my_e,
                                            uint32_t& my_s, bool& my_ok, unsigned long long* wr = nullptr) {
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
  uint32_t cu = 0xffffffffu, W = 0;
  while (todo) {
    const int j = __ffs(todo) - 1;
    todo &= todo - 1;
    const uint32_t uj = __shfl_sync(kFull, u, j), vj = __shfl_sync(kFull, v, j);
    if (uj != cu) {
      __syncwarp();
      W = R.words(uj);
      dense_load_row(R.bits + R.off(uj), W, su);
      cu = uj;
      if (wr && l == 0) *wr += W;
    }
    // Up to NQ edges sharing row u: one shared-memory read of row u feeds
    // all of them.
    int jq[NQ];
    uint32_t vq[NQ], cq[NQ];
    bool act[NQ];
    take_same_row<NQ>(todo, u, v, uj, j, vj, jq, vq, act);
    rows_and_popc<NQ>(R, vq, act, su, 0, W / 4, cq);
    uint32_t nq = 0;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      if (act[q] && l == (unsigned)jq[q]) my_s = cq[q];
      nq += act[q];
    }
    if (wr && l == 0) *wr += (unsigned long long)nq * W;
  }
  __syncwarp();
}


// As dense_group, but an edge whose count can no longer reach its threshold
// is abandoned: the rows are ANDed in four segments, and after each one the
// count so far plus the set bits left in row u bounds the result.  The
// segments go from the last to the first: vertex ids ascend with degree, so
// the last words of a row hold the high-degree vertices and most of the set
// bits, and after them the bits left in row u are few enough to abandon most
// edges below the threshold after one or two segments.  An
// abandoned edge reports a count below the threshold (not its support).  The
// threshold is `thr`, or for a grouped union gthr[vgid[u]] (its graph's).
// Two edges that share row u run side by side, one per half of the warp (two
// load streams per warp).
__device__ __forceinline__ void dense_group_capped(const uint32_t* __restrict__ list, uint64_t base, uint64_t cnt,
                                                   const uint64_t* __restrict__ ends, const DenseRows& R,
                                                   uint32_t thr, uint32_t* su, uint32_t& my_e, uint32_t& my_s,
                                                   bool& my_ok, unsigned long long* wr = nullptr,
                                                   const uint32_t* __restrict__ gthr = nullptr,
                                                   const uint32_t* __restrict__ vgid = nullptr) {
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
  const uint32_t my_thr = (gthr && ok) ? gthr[vgid[u]] : thr;
  my_e = e;
  my_ok = ok;
  my_s = 0;
  unsigned todo = __ballot_sync(kFull, ok);
  uint32_t s1 = 0, s2 = 0, s3 = 0;  // set bits of row u in segments 1..3
  uint32_t cu = 0xffffffffu, W = 0, c1 = 0, c2 = 0, c3 = 0;
  while (todo) {
    const int j = __ffs(todo) - 1;
    todo &= todo - 1;
    const uint32_t uj = __shfl_sync(kFull, u, j), vj = __shfl_sync(kFull, v, j);
    if (uj != cu) {
      __syncwarp();
      W = R.words(uj);
      dense_load_row(R.bits + R.off(uj), W, su);
      cu = uj;
      // Segment bounds: four runs of whole 32-word strides.
      const uint32_t strides = (W + 31) / 32;
      c1 = min(W, (strides / 4) * 32);
      c2 = min(W, (strides / 2) * 32);
      c3 = min(W, ((3 * strides) / 4) * 32);
      uint32_t a = 0, b = 0, c = 0;
      for (uint32_t i = l; i < c3; i += 32) {
        const uint32_t pc = __popc(su[i]);
        if (i < c1) a += pc; else if (i < c2) b += pc; else c += pc;
      }
      s1 = warp_sum(a);
      s2 = warp_sum(b);
      s3 = warp_sum(c);
      if (wr && l == 0) *wr += W;
    }
    // The next edge with the same row u goes to the upper half of the warp:
    // two edges' segments are ANDed side by side (two load streams).
    int j2 = -1;
    uint32_t vj2 = 0;
    if (todo) {
      const int cand = __ffs(todo) - 1;
      const uint32_t uc = __shfl_sync(kFull, u, cand), vc = __shfl_sync(kFull, v, cand);
      if (uc == uj) {
        j2 = cand;
        vj2 = vc;
        todo &= todo - 1;
      }
    }
    const bool upper = l >= 16;
    const uint32_t tj = __shfl_sync(kFull, my_thr, j), tj2 = __shfl_sync(kFull, my_thr, j2 >= 0 ? j2 : j);
    const uint32_t t = upper ? tj2 : tj;
    bool go = !upper || j2 >= 0;
    const uint32_t* pv = R.bits + R.off(upper ? vj2 : vj);
    uint32_t wds = go ? W - c3 : 0u;  // row-v words this half reads
    uint32_t found = half_and_popc(pv, su, c3, W, go);
    go = go && found + s1 + s2 + s3 >= t;
    if (__any_sync(kFull, go)) {
      wds += go ? c3 - c2 : 0u;
      found += half_and_popc(pv, su, c2, c3, go);
      go = go && found + s1 + s2 >= t;
      if (__any_sync(kFull, go)) {
        wds += go ? c2 - c1 : 0u;
        found += half_and_popc(pv, su, c1, c2, go);
        go = go && found + s1 >= t;
        if (__any_sync(kFull, go)) {
          wds += go ? c1 : 0u;
          found += half_and_popc(pv, su, 0, c1, go);
        }
      }
    }
    const uint32_t f0 = __shfl_sync(kFull, found, 0), f1 = __shfl_sync(kFull, found, 16);
    if (l == (unsigned)j) my_s = f0;
    if (j2 >= 0 && l == (unsigned)j2) my_s = f1;
    if (wr && (l & 15u) == 0) *wr += wds;
  }
  __syncwarp();
}

}  // namespace kt
