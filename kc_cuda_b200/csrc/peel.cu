// Stage (e): truss peeling of the working graph.
//
// Levels: at truss level t every alive edge with support < t-2 is removed,
// round by round, until none is left (a cascade); the alive edges then form
// the t-truss.  If edges remain, their minimum support s makes them an
// (s+2)-truss, which is recorded, and the next level is t = s+3.  The last
// recorded level when no edge is left is kmax.
//
// Rounds: the frontier edges of round r carry state r; deleted edges keep
// their round, alive edges kAlive.  A warp takes a frontier edge (x, y) and
// intersects the two sorted rows: 32-wide tiles of both rows are compared
// with a 5-step shuffle search, and whichever tile ends lower is retired
// (both when the ends tie), so every common neighbour is met exactly once;
// when one row is more than peel_search_ratio (16) times longer the lanes
// binary-search the long row instead.  A common w closes the triangle {e, a, b}; it is skipped if a or b
// was deleted in an earlier round.  Each surviving side edge loses one
// triangle, decremented by exactly one frontier edge of the triangle (the
// one with the smallest id among those in this round); an edge whose support
// steps from t-2 to t-3 joins the next frontier, so each edge enters a
// frontier once.
//
// A cascade runs as one cooperative launch: rounds are separated by the
// bounded grid barrier and the frontier sizes never leave the device.
//
// Jumps: without per-edge trussness output, the first level may be a guess
// well above the lower bound (one cascade removes everything below it).  The
// support/state arrays are snapshotted first; a guess that empties the graph
// is undone and halved toward the last good level.
//
// The reference keeps doubled supports and subtracts 2 - [m1==st] - [m2==st]
// from both side edges (src/kc.cu:61-159, 886-1056), and steps k by fixed
// strides with host backups and rollbacks (src/kc.cu:1140-1309); the result
// is the same kmax and edge count.
#include <algorithm>
#include <chrono>
#include <memory>

#include "compact.cuh"
#include "dense.cuh"
#include "subgraph.h"

namespace kt {
namespace {

constexpr unsigned kPeelThreads = 256;

struct PeelArgs {
  const uint64_t* ends;
  const uint64_t* off;
  const uint32_t* adj;
  const uint32_t* eid;
  uint32_t* sup;
  uint32_t* state;
  uint32_t* truss;  // may be null
  const uint32_t* alive;
  uint64_t na;
  uint32_t* front[2];
  unsigned long long* cnt;  // 3 rotating frontier counters, [3] rounds done, [4] gave up, [5] recount rounds
  uint64_t cap;
  uint32_t thr;    // remove support < thr
  uint32_t tval;   // trussness recorded for removed edges
  uint32_t r0;     // first round number
  uint32_t* adeg;  // alive degree per vertex (for the byte accounting)
  DenseRows R;     // dense mode: alive adjacency bitsets (R.bits null otherwise)
  float wavg;      // mean words per bitset row
  uint64_t bit_words;  // words of all bitset rows (a multiple of 4)
  uint32_t gamma;  // recount round when nf * thr * gamma > alive * wavg
  uint32_t search_ratio;  // binary-search the long row when it is this many times longer
  uint32_t split;         // split rounds when frontier x chunks <= split x warps (0 = never)
  unsigned long long* acct;  // [0] sum of alive degrees of deleted edges, [1] decrements, [2] recounted edges
  DevWords* words;
  unsigned long long timeout_ns;
  // Batched unions: per-graph thresholds gthr[egr[e]] replace thr (0 = the
  // graph is finished and its edges are never frontier edges).
  const uint32_t* gthr;
  const uint32_t* egr;
  const uint32_t* gthr_max;  // batched: the largest running threshold (recount cost model)
  // A level tried from a snapshot: give up (the level's truss is empty) as
  // soon as fewer than this many edges can remain, t(t-1)/2 for level t
  // (0: peel to the end).  The state is then partial; the caller undoes it.
  uint64_t fail_below = 0;
};

__device__ __forceinline__ uint32_t edge_thr(const PeelArgs& A, uint32_t e) {
  return A.gthr ? A.gthr[A.egr[e]] : A.thr;
}

__device__ __forceinline__ void push_warp_full(bool want, uint32_t item, uint32_t* list, unsigned long long* cnt,
                                               uint64_t cap, uint32_t* err) {
  const unsigned b = __ballot_sync(kFull, want);
  if (!b) return;
  const unsigned leader = __ffs(b) - 1;
  unsigned long long base = 0;
  if (lane_id() == leader) base = atomicAdd(cnt, (unsigned long long)__popc(b));
  base = __shfl_sync(kFull, base, leader);
  if (want) {
    const unsigned long long p = base + __popc(b & lanemask_lt());
    if (p < cap)
      list[p] = item;
    else
      atomicOr(err, kDevErrCapacity);
  }
}

__device__ __forceinline__ uint64_t find_sorted(const uint32_t* a, uint64_t lo, uint64_t hi, uint32_t x) {
  const uint64_t end = hi;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (a[mid] < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < end && a[lo] == x) ? lo : end;
}

// Triangle {e, a, b} seen from frontier edge e in round r; returns which of
// a, b crossed below the threshold (to be pushed).
__device__ __forceinline__ void close_triangle(const PeelArgs& A, uint32_t e, uint32_t a, uint32_t b, uint32_t r,
                                               uint32_t thr, bool& pa, bool& pb, uint32_t& ndec) {
  const uint32_t sa = A.state[a], sb = A.state[b];
  if (sa < r || sb < r) return;  // broken in an earlier round
  if (sa > r && !(sb == r && b < e)) {
    ++ndec;
    if (atomicSub(&A.sup[a], 1u) == thr) {
      A.state[a] = r + 1;
      if (A.truss) A.truss[a] = A.tval;
      pa = true;
    }
  }
  if (sb > r && !(sa == r && a < e)) {
    ++ndec;
    if (atomicSub(&A.sup[b], 1u) == thr) {
      A.state[b] = r + 1;
      if (A.truss) A.truss[b] = A.tval;
      pb = true;
    }
  }
}

// One frontier edge, one warp.  Pushes into next / ncnt; adds the edge's
// alive degrees and its decrements to the per-thread tallies.
__device__ __forceinline__ void peel_edge(const PeelArgs& A, uint32_t e, uint32_t r, uint32_t* next,
                                          unsigned long long* ncnt, uint64_t& tdeg, uint64_t& tdec) {
  const uint64_t k = A.ends[e];
  uint32_t x = (uint32_t)(k >> 32), y = (uint32_t)k;
  if (lane_id() == 0) tdeg += (uint64_t)atomicSub(&A.adeg[x], 1u) + atomicSub(&A.adeg[y], 1u);
  const uint32_t thr = edge_thr(A, e);  // the triangle's edges share e's graph
  uint32_t ndec = 0;
  uint64_t xb = A.off[x], xe = A.off[x + 1], yb = A.off[y], ye = A.off[y + 1];
  if (xe - xb > ye - yb) {
    uint64_t t = xb;
    xb = yb;
    yb = t;
    t = xe;
    xe = ye;
    ye = t;
  }
  const uint64_t na = xe - xb, nb = ye - yb;
  uint32_t* err = &A.words->err;
  const unsigned lane = lane_id();
  if (A.R.sbits && (uint64_t)A.R.words(x) <= na + nb) {
    // Dense rows shorter than the two lists: AND the two bitset rows (32
    // words a step, one per lane); each common neighbour's edge ids come from
    // its position in the sorted rows, a popcount of the rows as built.  Bits
    // of edges deleted in earlier cascades are clear; deletions of this
    // cascade are caught by close_triangle's state test, as in the merge.
    const uint32_t* rx = A.R.bits + A.R.off(x);
    const uint32_t* ry = A.R.bits + A.R.off(y);
    const uint32_t W = A.R.words(x);
    const uint64_t ox = A.off[x], oy = A.off[y];
    for (uint32_t i0 = 0; i0 < W; i0 += 32) {
      const uint32_t i = i0 + lane;
      uint32_t mset = i < W ? __ldcg(rx + i) & __ldcg(ry + i) : 0u;
      while (__any_sync(kFull, mset != 0)) {
        bool pa = false, pb = false;
        uint32_t a = 0, b = 0;
        if (mset) {
          const uint32_t col = i * 32 + (uint32_t)(__ffs(mset) - 1);
          mset &= mset - 1;
          a = A.eid[ox + A.R.rank(x, col)];
          b = A.eid[oy + A.R.rank(y, col)];
          close_triangle(A, e, a, b, r, thr, pa, pb, ndec);
        }
        push_warp_full(pa, a, next, ncnt, A.cap, err);
        push_warp_full(pb, b, next, ncnt, A.cap, err);
      }
    }
    tdec += ndec;
    return;
  }
  if (nb > (uint64_t)A.search_ratio * na) {
    // Short row against a long one: binary search per lane.
    for (uint64_t q = xb + lane; q < xb + ((na + 31) & ~31ULL); q += 32) {
      bool pa = false, pb = false;
      uint32_t a = 0, b = 0;
      if (q < xe) {
        const uint64_t p = find_sorted(A.adj, yb, ye, A.adj[q]);
        if (p != ye) {
          a = A.eid[q];
          b = A.eid[p];
          close_triangle(A, e, a, b, r, thr, pa, pb, ndec);
        }
      }
      push_warp_full(pa, a, next, ncnt, A.cap, err);
      push_warp_full(pb, b, next, ncnt, A.cap, err);
    }
    tdec += ndec;
    return;
  }
  // Tile merge.
  uint64_t i = 0, j = 0;
  while (i < na && j < nb) {
    const uint32_t ta = (uint32_t)(na - i < 32 ? na - i : 32), tb = (uint32_t)(nb - j < 32 ? nb - j : 32);
    const uint32_t av = lane < ta ? A.adj[xb + i + lane] : 0xffffffffu;
    const uint32_t bv = lane < tb ? A.adj[yb + j + lane] : 0xffffffffu;
    const uint32_t alast = __shfl_sync(kFull, av, ta - 1);
    const uint32_t blast = __shfl_sync(kFull, bv, tb - 1);
    // Lower bound of av in the B tile (lanes < tb hold it, ascending).
    uint32_t q = 0;
#pragma unroll
    for (uint32_t s = 16; s >= 1; s >>= 1) {
      const uint32_t probe = __shfl_sync(kFull, bv, (q + s - 1) & 31);
      if (q + s <= tb && probe < av) q += s;
    }
    const uint32_t hit = __shfl_sync(kFull, bv, q & 31);
    bool pa = false, pb = false;
    uint32_t a = 0, b = 0;
    if (lane < ta && q < tb && hit == av) {
      a = A.eid[xb + i + lane];
      b = A.eid[yb + j + q];
      close_triangle(A, e, a, b, r, thr, pa, pb, ndec);
    }
    push_warp_full(pa, a, next, ncnt, A.cap, err);
    push_warp_full(pb, b, next, ncnt, A.cap, err);
    if (alast <= blast) i += ta;
    if (blast <= alast) j += tb;
  }
  tdec += ndec;
}

// Rounds with few frontier edges split each edge's bitset intersection into
// chunks of kSplitWords words, one warp per (edge, chunk), so a small
// frontier of edges with many triangles keeps the whole grid busy.
constexpr uint32_t kSplitWords = 8;

// Position of the r-th (from 0) set bit of m.
__device__ __forceinline__ uint32_t select_bit(uint32_t m, uint32_t r) {
  uint32_t pos = 0;
#pragma unroll
  for (uint32_t s = 16; s >= 1; s >>= 1) {
    const uint32_t low = __popc(m & ((1u << s) - 1u));
    if (r >= low) {
      r -= low;
      m >>= s;
      pos += s;
    }
  }
  return pos;
}

// Words [w0, w0 + kSplitWords) of frontier edge e's two bitset rows: the
// common neighbours found there are dealt one per lane (a warp scan of the
// words' popcounts, then a 3-step search for each task's word and a select of
// its bit), each closing its triangle as in peel_edge.
__device__ __forceinline__ void peel_edge_chunk(const PeelArgs& A, uint32_t e, uint32_t x, uint32_t y, uint32_t thr,
                                                uint32_t W, uint32_t w0, uint32_t r, uint32_t* next,
                                                unsigned long long* ncnt, uint64_t& tdec) {
  const unsigned lane = lane_id();
  const uint32_t i = w0 + lane;
  uint32_t m = 0;
  if (lane < kSplitWords && i < W) m = __ldcg(A.R.bits + A.R.off(x) + i) & __ldcg(A.R.bits + A.R.off(y) + i);
  const uint32_t c = __popc(m);
  const uint32_t incl = warp_incl_scan(c);
  const uint32_t T = __shfl_sync(kFull, incl, 31);
  const uint32_t excl = incl - c;
  const uint64_t ox = A.off[x], oy = A.off[y];
  uint32_t ndec = 0;
  for (uint32_t base = 0; base < T; base += 32) {
    const uint32_t t = base + lane;
    uint32_t lo = 0;  // the last word (lane < kSplitWords) whose first task is <= t
#pragma unroll
    for (uint32_t st = kSplitWords / 2; st >= 1; st >>= 1) {
      const uint32_t cand = lo + st;
      const uint32_t ec = __shfl_sync(kFull, excl, cand & 31);
      if (cand < kSplitWords && ec <= t) lo = cand;
    }
    const uint32_t oexcl = __shfl_sync(kFull, excl, lo), om = __shfl_sync(kFull, m, lo);
    bool pa = false, pb = false;
    uint32_t a = 0, b = 0;
    if (t < T) {
      const uint32_t col = (w0 + lo) * 32 + select_bit(om, t - oexcl);
      a = A.eid[ox + A.R.rank(x, col)];
      b = A.eid[oy + A.R.rank(y, col)];
      close_triangle(A, e, a, b, r, thr, pa, pb, ndec);
    }
    push_warp_full(pa, a, next, ncnt, A.cap, &A.words->err);
    push_warp_full(pb, b, next, ncnt, A.cap, &A.words->err);
  }
  tdec += ndec;
}

// A decrement round over (frontier edge, chunk) units; edges that use the
// sorted-list merge go whole to the warp of their first chunk.
__device__ __forceinline__ void split_round(const PeelArgs& A, const uint32_t* fr, uint64_t nf, uint64_t chunks,
                                            uint32_t r, uint32_t* next, unsigned long long* ncnt, uint64_t gwarp,
                                            uint64_t gwarps, uint64_t& tdeg, uint64_t& tdec) {
  for (uint64_t u = gwarp; u < nf * chunks; u += gwarps) {
    const uint64_t f = u / chunks;
    const uint32_t ch = (uint32_t)(u - f * chunks);
    const uint32_t e = fr[f];
    const uint64_t k = A.ends[e];
    const uint32_t x = (uint32_t)(k >> 32), y = (uint32_t)k;
    const uint64_t na = A.off[x + 1] - A.off[x], nb = A.off[y + 1] - A.off[y];
    const uint32_t W = A.R.words(x);
    if ((uint64_t)W > na + nb) {  // peel_edge would merge the lists
      if (ch == 0) peel_edge(A, e, r, next, ncnt, tdeg, tdec);
      continue;
    }
    if (ch * kSplitWords >= W) continue;
    if (ch == 0 && lane_id() == 0) tdeg += (uint64_t)atomicSub(&A.adeg[x], 1u) + atomicSub(&A.adeg[y], 1u);
    peel_edge_chunk(A, e, x, y, edge_thr(A, e), W, ch * kSplitWords, r, next, ncnt, tdec);
  }
}

__device__ __forceinline__ void flush_tallies(const PeelArgs& A, uint64_t tdeg, uint64_t tdec) {
  tdeg = warp_sum(tdeg);
  tdec = warp_sum(tdec);
  if (lane_id() == 0) {
    if (tdeg) atomicAdd(&A.acct[0], (unsigned long long)tdeg);
    if (tdec) atomicAdd(&A.acct[1], (unsigned long long)tdec);
  }
}

// Frontier of a level: alive edges with support below the threshold.
__device__ __forceinline__ void level_frontier(const PeelArgs& A, uint32_t r, uint64_t gtid, uint64_t gthreads) {
  for (uint64_t i = gtid; i < ((A.na + 31) & ~31ULL); i += gthreads) {
    bool want = false;
    uint32_t e = 0;
    if (i < A.na) {
      e = A.alive[i];
      if (A.state[e] == kAlive && A.sup[e] < edge_thr(A, e)) {
        A.state[e] = r;
        if (A.truss) A.truss[e] = A.tval;
        want = true;
      }
    }
    push_warp_full(want, e, A.front[0], &A.cnt[0], A.cap, &A.words->err);
  }
}

__device__ __forceinline__ void clear_edge_bits(const PeelArgs& A, uint32_t e) {
  const uint64_t k = A.ends[e];
  const uint32_t x = (uint32_t)(k >> 32), y = (uint32_t)k;
  const uint32_t cy = A.R.col(x, y), cx = A.R.col(y, x);
  atomicAnd(&A.R.bits[A.R.off(x) + (cy >> 5)], ~(1u << (cy & 31)));
  atomicAnd(&A.R.bits[A.R.off(y) + (cx >> 5)], ~(1u << (cx & 31)));
}

// Rebuilds the bitsets from the surviving edges when more edges were deleted
// since the bits were last current than survive: zero every word, then (after
// a grid barrier, in the caller) set the bits of the alive-list edges still
// alive -- fewer atomics than clearing the deleted edges one by one.
__device__ __forceinline__ void zero_bits(const PeelArgs& A, uint64_t gtid, uint64_t gthreads) {
  uint4* p = reinterpret_cast<uint4*>(A.R.bits);
  for (uint64_t w = gtid; w < A.bit_words / 4; w += gthreads) p[w] = make_uint4(0u, 0u, 0u, 0u);
}
__device__ __forceinline__ void set_alive_bits(const PeelArgs& A, uint64_t gtid, uint64_t gthreads) {
  for (uint64_t i = gtid; i < A.na; i += gthreads) {
    const uint32_t e = A.alive[i];
    if (A.state[e] != kAlive) continue;
    const uint64_t k = A.ends[e];
    const uint32_t x = (uint32_t)(k >> 32), y = (uint32_t)k;
    const uint32_t cy = A.R.col(x, y), cx = A.R.col(y, x);
    atomicOr(&A.R.bits[A.R.off(x) + (cy >> 5)], 1u << (cy & 31));
    atomicOr(&A.R.bits[A.R.off(y) + (cx >> 5)], 1u << (cx & 31));
  }
}

// Clears the bits of alive-list edges deleted in rounds (lo, hi].
__device__ __forceinline__ void clear_deleted(const PeelArgs& A, uint32_t lo, uint32_t hi, uint64_t gtid,
                                              uint64_t gthreads) {
  for (uint64_t i = gtid; i < A.na; i += gthreads) {
    const uint32_t e = A.alive[i];
    const uint32_t st = A.state[e];
    if (st > lo && st <= hi) clear_edge_bits(A, e);
  }
}

// Dense recount round r: every surviving edge gets its exact support in the
// graph without this round's frontier; those below the threshold form the
// next frontier.  Replaces per-triangle decrements when the frontier is a
// large part of the graph.
// Warps take the next 32-entry group of the alive list from `cursor` (zero
// at the start of the round), so the groups in flight stay a narrow window
// of the tile-ordered list and the rows they read stay in L2.
__device__ __forceinline__ void recount_round(const PeelArgs& A, uint32_t r, uint32_t* next,
                                              unsigned long long* ncnt, unsigned long long* cursor,
                                              uint64_t& trec, uint32_t* su) {
  const uint64_t groups = (A.na + 31) / 32;
  for (;;) {
    unsigned long long g = 0;
    if (lane_id() == 0) g = atomicAdd(cursor, 1ULL);
    g = __shfl_sync(kFull, g, 0);
    if (g >= groups) break;
    uint32_t e, sc;
    bool ok;
    dense_group<2>(A.alive, g * 32, A.na, A.ends, A.R, A.state, su, e, sc, ok);
    trec += __popc(__ballot_sync(kFull, ok));
    bool want = false;
    if (ok) {
      A.sup[e] = sc;
      if (sc < edge_thr(A, e)) {
        A.state[e] = r + 1;
        if (A.truss) A.truss[e] = A.tval;
        want = true;
      }
    }
    push_warp_full(want, e, next, ncnt, A.cap, &A.words->err);
  }
}

// One whole cascade in one cooperative launch.  Dense mode uses W words of
// shared memory per warp for the recount rounds.
// Resident blocks per SM the register allocation aims at (a build constant).
#ifndef KT_PEEL_MIN_BLOCKS
#define KT_PEEL_MIN_BLOCKS 5
#endif
__global__ void __launch_bounds__(kPeelThreads, KT_PEEL_MIN_BLOCKS) k_cascade(PeelArgs A) {
  extern __shared__ __align__(16) uint32_t dense_smem[];
  uint32_t* su = dense_smem + warp_id() * A.R.W;
  const uint64_t gthreads = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  level_frontier(A, A.r0, gtid, gthreads);
  if (!grid_barrier(A.words, A.timeout_ns)) return;
  const uint64_t gwarps = gthreads >> 5, gwarp = gtid >> 5;
  uint64_t tdeg = 0, tdec = 0, trec = 0;
  uint64_t alive = A.na;
  uint32_t cleared = A.r0 - 1;  // bits are current for deletions up to this round
  uint64_t pending = 0;          // edges deleted since then
  uint32_t i = 0, nrec = 0;
  bool ok = true;
  bool gave_up = false;
  while (true) {
    const uint64_t nf = ld_acquire_u64(&A.cnt[i % 3]);
    if (nf == 0) break;
    // Every block reads the same counts, so all of them give up together.
    if (alive - nf < A.fail_below) {
      gave_up = true;
      break;
    }
    const uint32_t r = A.r0 + i;
    uint32_t* fr = A.front[i & 1];
    uint32_t* nx = A.front[(i + 1) & 1];
    unsigned long long* nc = &A.cnt[(i + 1) % 3];
    const uint32_t thr = A.gthr_max ? *A.gthr_max : A.thr;
    const bool recount = A.R.bits && (double)nf * (double)(thr > 0 ? thr : 1) * (double)A.gamma >
                                         (double)alive * (double)A.wavg;
    pending += nf;
    if (recount) {
      ++nrec;
      // Group cursors: this recount uses slot 6 + (nrec & 1); the other slot,
      // last used by the previous recount (finished before the barrier that
      // ended its round), is cleared for the next one.
      if (gtid == 0) A.cnt[6 + ((nrec + 1) & 1)] = 0;
      if (pending > alive - nf) {
        zero_bits(A, gtid, gthreads);
        if (!grid_barrier(A.words, A.timeout_ns)) {
          ok = false;
          break;
        }
        set_alive_bits(A, gtid, gthreads);
      } else {
        clear_deleted(A, cleared, r, gtid, gthreads);
      }
      cleared = r;
      pending = 0;
      if (!grid_barrier(A.words, A.timeout_ns)) {
        ok = false;
        break;
      }
      recount_round(A, r, nx, nc, &A.cnt[6 + (nrec & 1)], trec, su);
    } else {
      // Few frontier edges for the grid: deal (edge, chunk) units instead.
      const uint64_t chunks = A.R.sbits ? (A.R.W + kSplitWords - 1) / kSplitWords : 1;
      if (chunks >= 2 && nf * chunks <= (uint64_t)A.split * gwarps)
        split_round(A, fr, nf, chunks, r, nx, nc, gwarp, gwarps, tdeg, tdec);
      else
        for (uint64_t f = gwarp; f < nf; f += gwarps) peel_edge(A, fr[f], r, nx, nc, tdeg, tdec);
    }
    if (gtid == 0) A.cnt[(i + 2) % 3] = 0;  // read at the start of round i-1, next written in round i+1
    if (!grid_barrier(A.words, A.timeout_ns)) {
      ok = false;
      break;
    }
    alive -= nf;
    ++i;
  }
  // Bring the bitsets up to date with this cascade's remaining deletions.
  if (ok && !gave_up && A.R.bits && pending) {
    if (pending > alive) {
      zero_bits(A, gtid, gthreads);
      if (grid_barrier(A.words, A.timeout_ns)) set_alive_bits(A, gtid, gthreads);
    } else {
      clear_deleted(A, cleared, A.r0 + i, gtid, gthreads);
    }
  }
  flush_tallies(A, tdeg, tdec);
  if (lane_id() == 0 && trec) atomicAdd(&A.acct[2], (unsigned long long)trec);
  if (gtid == 0) {
    A.cnt[3] = i;
    A.cnt[4] = gave_up;
    A.cnt[5] = nrec;
  }
}

// Host-stepped variant (one launch per round), used when cooperative launch
// is switched off.
__global__ void __launch_bounds__(kPeelThreads) k_level_frontier(PeelArgs A) {
  level_frontier(A, A.r0, (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, (uint64_t)gridDim.x * blockDim.x);
}

__global__ void __launch_bounds__(kPeelThreads) k_round(PeelArgs A, uint32_t i, uint64_t nf) {
  const uint64_t gwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t gwarp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint64_t tdeg = 0, tdec = 0;
  for (uint64_t f = gwarp; f < nf; f += gwarps)
    peel_edge(A, A.front[i & 1][f], A.r0 + i, A.front[(i + 1) & 1], &A.cnt[(i + 1) % 3], tdeg, tdec);
  flush_tallies(A, tdeg, tdec);
}

__global__ void k_peel_init(uint64_t m, uint32_t* __restrict__ state, uint32_t* __restrict__ alive, uint32_t n,
                            const uint64_t* __restrict__ off, uint32_t* __restrict__ adeg) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
    state[e] = kAlive;
    alive[e] = (uint32_t)e;
  }
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    adeg[v] = (uint32_t)(off[v + 1] - off[v]);
}

__global__ void k_alive_min(const uint32_t* __restrict__ alive, uint64_t na, const uint32_t* __restrict__ sup,
                            uint32_t* out) {
  uint32_t mn = 0xffffffffu, mx = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = sup[alive[i]];
    mn = min(mn, s);
    mx = max(mx, s);
  }
  mn = warp_min(mn);
  mx = warp_max(mx);
  if (lane_id() == 0) {
    if (mn != 0xffffffffu) atomicMin(out, mn);
    atomicMax(out + 1, mx);
  }
}

// Per-graph alive edges and minimum support after a level (batched unions).
__global__ void k_track(const uint32_t* __restrict__ alive, uint64_t na, const uint64_t* __restrict__ ends,
                        const uint32_t* __restrict__ sup, const uint32_t* __restrict__ vgid,
                        unsigned long long* __restrict__ gcnt, uint32_t* __restrict__ gmin) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ((na + 31) & ~31ULL);
       i += (uint64_t)gridDim.x * blockDim.x) {
    const bool valid = i < na;
    uint32_t g = 0xffffffffu, sv = 0xffffffffu;
    if (valid) {
      const uint32_t e = alive[i];
      g = vgid[(uint32_t)(ends[e] >> 32)];
      sv = sup[e];
    }
    // Graphs are contiguous in the edge order: aggregate equal graphs.
    const unsigned peers = __match_any_sync(kFull, g);
    const unsigned leader = __ffs(peers) - 1;
    const uint32_t mn = __reduce_min_sync(peers, sv);
    if (valid && lane_id() == leader) {
      atomicAdd(&gcnt[g], (unsigned long long)__popc(peers));
      atomicMin(&gmin[g], mn);
    }
  }
}

// Records every running graph's level and sets its next threshold (its
// minimum support + 1, i.e. level min + 3); a graph with no alive edge, or
// whose first level kept exactly stop[g] edges, is finished (threshold 0).
__global__ void k_track_record(uint32_t ngroups, unsigned long long* __restrict__ gcnt, uint32_t* __restrict__ gmin,
                               uint32_t* __restrict__ kmax, uint64_t* __restrict__ count,
                               uint32_t* __restrict__ gthr, const uint64_t* __restrict__ stop, bool first) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ngroups; g += gridDim.x * blockDim.x) {
    if (gthr[g]) {
      if (gcnt[g]) {
        kmax[g] = gmin[g] + 2;
        count[g] = gcnt[g];
        gthr[g] = first && stop && stop[g] && gcnt[g] == stop[g] ? 0u : gmin[g] + 1;
      } else {
        gthr[g] = 0;
      }
    }
    gcnt[g] = 0;
    gmin[g] = 0xffffffffu;
  }
}

__global__ void k_max_u32(const uint32_t* __restrict__ a, uint32_t n, uint32_t* out) {
  uint32_t mx = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ((n + 31) & ~31u); i += gridDim.x * blockDim.x)
    mx = max(mx, i < n ? a[i] : 0u);
  mx = warp_max(mx);
  if (lane_id() == 0 && mx) atomicMax(out, mx);
}

__global__ void k_track_init(uint64_t m, const uint64_t* __restrict__ ends, const uint32_t* __restrict__ vgid,
                             uint32_t* __restrict__ egr, uint32_t ngroups, const uint32_t* __restrict__ t0,
                             uint32_t tdef, uint32_t* __restrict__ gthr) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x)
    egr[e] = vgid[(uint32_t)(ends[e] >> 32)];
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ngroups; g += gridDim.x * blockDim.x) {
    const uint32_t t = t0 && t0[g] > 3 ? t0[g] : (tdef > 3 ? tdef : 3);
    gthr[g] = t - 2;
  }
}

struct StillAlive {
  const uint32_t* list;
  const uint32_t* state;
  const uint32_t* gthr;  // batched: drop the edges of finished graphs
  const uint32_t* egr;
  __device__ bool keep(uint64_t i) const {
    const uint32_t e = list[i];
    return state[e] == kAlive && (!gthr || gthr[egr[e]] != 0);
  }
  __device__ uint32_t value(uint64_t i) const { return list[i]; }
};

// Ends (u << 32 | v) of the alive edges of a list.
struct AliveEnds {
  const uint32_t* list;
  const uint32_t* state;
  const uint64_t* ends;
  __device__ bool keep(uint64_t i) const { return state[list[i]] == kAlive; }
  __device__ uint64_t value(uint64_t i) const { return ends[list[i]]; }
};

// Peel state of one working graph on the device.
struct Peeler {
  Ctx* c;
  const Sub* s;
  uint32_t* sup;
  uint32_t* truss;
  DBuf state, alive[2], front[2], cnt, mm, adeg, acct;
  uint64_t scanned = 0;  // alive-list entries scanned by level frontiers
  int ai = 0;
  uint64_t na = 0;
  uint32_t r = 1;  // next round number
  uint64_t fail_below = 0;  // set while a level is tried from a snapshot (PeelArgs::fail_below)
  unsigned coop_grid = 0;
  size_t smem = 0;
  PeelResult* res;

  const void* kernel() const { return (const void*)k_cascade; }

  void init() {
    const uint64_t m = s->m;
    state = DBuf(c, m * sizeof(uint32_t));
    alive[0] = DBuf(c, m * sizeof(uint32_t));
    alive[1] = DBuf(c, m * sizeof(uint32_t));
    front[0] = DBuf(c, m * sizeof(uint32_t));
    front[1] = DBuf(c, m * sizeof(uint32_t));
    cnt = DBuf(c, 8 * sizeof(unsigned long long));
    mm = DBuf(c, 8);
    adeg = DBuf(c, ((uint64_t)s->n + 1) * sizeof(uint32_t));
    if (!acct.get()) {
      acct = DBuf(c, 4 * sizeof(unsigned long long));
      zero(c, acct.get(), acct.bytes());
    }
    ai = 0;
    k_peel_init<<<grid_for(std::max<uint64_t>(m, s->n), 256, c->num_sms * 16), 256, 0, c->stream>>>(
        m, state.as<uint32_t>(), alive[0].as<uint32_t>(), s->n, s->off.as<uint64_t>(), adeg.as<uint32_t>());
    // Dense mode: keep the alive list in tile order (compaction preserves it).
    if (s->W)
      KT_CUDA(cudaMemcpyAsync(alive[0].get(), s->order.get(), m * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                              c->stream));
    KT_LAUNCHED(c);
    na = m;
    smem = dense_smem_bytes(s->W, kPeelThreads);
    coop_grid = 0;
    if (c->opt.persistent || s->W) {
      allow_max_dynamic_smem((const void*)k_cascade);
      int per_sm = 0;
      KT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cascade, kPeelThreads, smem));
      coop_grid = coop_blocks(c, per_sm);
    }
  }

  PeelArgs args(uint32_t t) {
    PeelArgs A;
    A.ends = s->ends.as<uint64_t>();
    A.off = s->off.as<uint64_t>();
    A.adj = s->adj.as<uint32_t>();
    A.eid = s->eid.as<uint32_t>();
    A.sup = sup;
    A.state = state.as<uint32_t>();
    A.truss = truss;
    A.alive = alive[ai].as<uint32_t>();
    A.na = na;
    A.front[0] = front[0].as<uint32_t>();
    A.front[1] = front[1].as<uint32_t>();
    A.cnt = cnt.as<unsigned long long>();
    A.cap = s->m;
    A.thr = t - 2;
    A.tval = t - 1;
    A.r0 = r;
    A.adeg = adeg.as<uint32_t>();
    A.acct = acct.as<unsigned long long>();
    A.R = s->W ? dense_rows(*s) : DenseRows{nullptr, 0, nullptr, nullptr, nullptr, nullptr, nullptr};
    if (!c->opt.peel_bitset) A.R.sbits = nullptr;
    A.wavg = s->W ? (float)((double)s->bit_words / std::max<uint32_t>(s->n, 1)) : 0.f;
    A.bit_words = s->W ? s->bit_words : 0;
    A.gamma = (uint32_t)std::max<int64_t>(1, c->opt.recount_gamma);
    A.search_ratio = (uint32_t)std::min<int64_t>(std::max<int64_t>(1, c->opt.peel_search_ratio), 1 << 20);
    A.split = (uint32_t)std::min<int64_t>(std::max<int64_t>(0, c->opt.peel_split), 1 << 20);
    A.words = dev_words(c);
    A.timeout_ns = (unsigned long long)c->opt.timeout_ms * 1000000ULL;
    A.gthr = track ? gthr.as<uint32_t>() : nullptr;
    A.egr = track ? egr.as<uint32_t>() : nullptr;
    A.gthr_max = track ? tmax.as<uint32_t>() : nullptr;
    A.fail_below = fail_below;
    return A;
  }

  // A level tried from a snapshot: the cascade gives up once its truss can
  // no longer hold t(t-1)/2 edges.
  uint64_t try_level(uint32_t t) {
    fail_below = (uint64_t)t * (t - 1) / 2;
    const uint64_t left = cascade(t);
    fail_below = 0;
    return left;
  }

  // Removes every alive edge with support < t-2, to the fixpoint; returns
  // the alive count.
  uint64_t cascade(uint32_t t) {
    PeelArgs A = args(t);
    zero(c, cnt.get(), cnt.bytes());
    cudaEvent_t e0;
    c->timer.begin(c->stream, &c->stats.ms_peel_kernel, &e0);
    uint64_t rounds = 0, recounts = 0;
    bool gave_up = false;
    scanned += na;
    const auto t_start = std::chrono::steady_clock::now();
    if (coop_grid) {
      void* p[] = {&A};
      uint64_t h[3];
      {
        CoopLock coop(c);
        KT_CUDA(cudaLaunchCooperativeKernel(kernel(), dim3(coop_grid), dim3(kPeelThreads), p, smem, c->stream));
        KT_LAUNCHED(c);
        copy_d2h(c, h, A.cnt + 3, sizeof(h));
      }
      rounds = h[0];
      gave_up = h[1] != 0;
      recounts = h[2];
    } else {
      k_level_frontier<<<grid_for(na, kPeelThreads, c->num_sms * 16), kPeelThreads, 0, c->stream>>>(A);
      KT_LAUNCHED(c);
      uint64_t left = na;
      for (uint32_t i = 0;; ++i) {
        const uint64_t nf = read_word<unsigned long long>(c, A.cnt + (i % 3));
        if (nf == 0) break;
        if (left - nf < A.fail_below) {
          gave_up = true;
          break;
        }
        left -= nf;
        ++rounds;
        KT_CUDA(cudaMemsetAsync(A.cnt + ((i + 1) % 3), 0, sizeof(unsigned long long), c->stream));
        k_round<<<grid_for(nf * 32, kPeelThreads, c->num_sms * 16), kPeelThreads, 0, c->stream>>>(A, i, nf);
        KT_LAUNCHED(c);
      }
    }
    c->timer.end(c->stream, e0, &c->stats.ms_peel_kernel);
    c->stats.peel_launches++;
    check_words(c, "truss peel");
    KT_LOG(c, "kt: cascade level %u on %llu alive of %llu edges (n %u, W %u): %llu rounds (%llu recount)%s, %.3f ms\n",
           t, (unsigned long long)na, (unsigned long long)s->m, s->n, s->W, (unsigned long long)rounds,
           (unsigned long long)recounts, gave_up ? ", gave up" : "",
           std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count());
    r += (uint32_t)rounds + 1;
    res->rounds += rounds;
    res->levels++;
    if (gave_up) return 0;  // the level is empty; the state is partial and the caller undoes it
    na = compact(c, na,
                 StillAlive{alive[ai].as<uint32_t>(), state.as<uint32_t>(), A.gthr, A.egr},
                 alive[ai ^ 1].as<uint32_t>());
    ai ^= 1;
    return na;
  }

  // Algorithmic bytes of this peel: 8 per alive-degree unit of every deleted
  // edge (neighbour id + edge id), 8 per support decrement (read-modify-
  // write), 4 per alive-list entry scanned by a level frontier.  The dense
  // recount rounds' bitset rows (4 W bytes per recounted edge, mostly from
  // L2) are kept apart in peel_recount_bytes.
  void account() {
    uint64_t h[3];
    copy_d2h(c, h, acct.get(), 24);
    const double wavg = s->W ? (double)s->bit_words / std::max<uint32_t>(s->n, 1) : 0.0;
    c->stats.peel_bytes += 8 * h[0] + 8 * h[1] + 4 * scanned;
    c->stats.peel_recount_bytes += (uint64_t)(4.0 * wavg * (double)h[2]);
    c->stats.peel_decrements += h[1];
  }

  // Batched unions: per-graph thresholds and records after a level.
  const GraphTrack* track = nullptr;
  DBuf tcnt, tmin, gthr, egr, tmax;
  void init_track(uint32_t t0) {
    const uint32_t G = std::max<uint32_t>(track->ngroups, 1);
    tcnt = DBuf(c, (uint64_t)G * 8);
    tmin = DBuf(c, (uint64_t)G * 4);
    gthr = DBuf(c, (uint64_t)G * 4);
    egr = DBuf(c, s->m * 4);
    tmax = DBuf(c, 4);
    zero(c, tcnt.get(), tcnt.bytes());
    KT_CUDA(cudaMemsetAsync(tmin.get(), 0xff, tmin.bytes(), c->stream));
    k_track_init<<<grid_for(std::max<uint64_t>(s->m, G), 256, c->num_sms * 16), 256, 0, c->stream>>>(
        s->m, s->ends.as<uint64_t>(), track->vgid, egr.as<uint32_t>(), track->ngroups, track->t0, t0,
        gthr.as<uint32_t>());
    KT_LAUNCHED(c);
    update_tmax();
  }
  void update_tmax() {
    zero(c, tmax.get(), 4);
    k_max_u32<<<grid_for(track->ngroups, 256, c->num_sms * 4), 256, 0, c->stream>>>(
        gthr.as<uint32_t>(), track->ngroups, tmax.as<uint32_t>());
    KT_LAUNCHED(c);
  }
  void record_groups(bool first) {
    if (na) {
      k_track<<<grid_for(na, 256, c->num_sms * 16), 256, 0, c->stream>>>(
          alive[ai].as<uint32_t>(), na, s->ends.as<uint64_t>(), sup, track->vgid, tcnt.as<unsigned long long>(),
          tmin.as<uint32_t>());
      KT_LAUNCHED(c);
    }
    k_track_record<<<grid_for(track->ngroups, 256, c->num_sms * 4), 256, 0, c->stream>>>(
        track->ngroups, tcnt.as<unsigned long long>(), tmin.as<uint32_t>(), track->kmax, track->count,
        gthr.as<uint32_t>(), track->stop, first);
    KT_LAUNCHED(c);
    update_tmax();
  }

  // Replaces the working graph by its alive part (renumbered, with its own
  // bitsets and exact supports) once most edges are gone; the alive edges
  // form a truss, so their supports in the new graph equal their current
  // ones.  Returns whether it compacted.
  bool compact_graph(std::unique_ptr<Sub>& own, DBuf& own_sup) {
    if (truss || track || na == 0 || na * 4 > s->m || s->m < (1u << 20)) return false;
    account();
    zero(c, acct.get(), acct.bytes());
    scanned = 0;
    DBuf keys(c, na * sizeof(uint64_t));
    const uint64_t k = kt::compact(c, na, AliveEnds{alive[ai].as<uint32_t>(), state.as<uint32_t>(),
                                                    s->ends.as<uint64_t>()},
                                   keys.as<uint64_t>());
    std::unique_ptr<Sub> ns(new Sub);
    // The alive list is in edge-id order unless the graph has bitsets (tile
    // order), so its ends are already sorted then.
    build_sub_from_keys(c, keys.as<uint64_t>(), k, s->n, *ns, s->W == 0);
    DBuf nsup(c, (ns->m ? ns->m : 1) * sizeof(uint32_t));
    edge_support(c, *ns, nsup.as<uint32_t>());
    own.swap(ns);
    own_sup = std::move(nsup);
    s = own.get();
    sup = own_sup.as<uint32_t>();
    init();
    return true;
  }

  // Finds the top level by bisection, between lo (the current state is the
  // lo-truss, non-empty) and hi (the hi-truss is empty): a level whose truss
  // is empty is undone from a snapshot of the state (supports, edge states,
  // alive degrees, bitsets; the alive list of the snapshot stays in the
  // other buffer), a non-empty one is kept.  A t-truss is non-empty exactly
  // for t <= kmax, so this ends with res at kmax and its edge count.
  void bisect(uint32_t lo, uint32_t hi, PeelResult& out) {
    DBuf ssup(c, s->m * sizeof(uint32_t)), sstate(c, s->m * sizeof(uint32_t)), sdeg(c, adeg.bytes()), sbits;
    if (s->W) sbits.alloc(c, s->bits.bytes());
    uint64_t na0 = 0;
    int ai0 = 0;
    auto copy = [&](void* dst, const void* src, size_t bytes) {
      KT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c->stream));
    };
    auto save = [&] {
      copy(ssup.get(), sup, s->m * sizeof(uint32_t));
      copy(sstate.get(), state.get(), s->m * sizeof(uint32_t));
      copy(sdeg.get(), adeg.get(), adeg.bytes());
      if (s->W) copy(sbits.get(), s->bits.get(), s->bits.bytes());
      na0 = na;
      ai0 = ai;
    };
    save();
    while (hi - lo > 1) {
      const uint32_t mid = lo + (hi - lo) / 2;
      const uint64_t left = try_level(mid);
      if (left) {
        uint32_t mn, mx;
        minmax(mn, mx);
        lo = mn + 2;  // >= mid
        out.kmax = lo;
        out.count = left;
        if (hi - lo > 1) save();
      } else {
        copy(sup, ssup.get(), s->m * sizeof(uint32_t));
        copy(state.get(), sstate.get(), s->m * sizeof(uint32_t));
        copy(adeg.get(), sdeg.get(), adeg.bytes());
        if (s->W) copy(s->bits.get(), sbits.get(), s->bits.bytes());
        na = na0;
        ai = ai0;
        hi = mid;
      }
    }
    KT_LOG(c, "kt: bisection ends at level %u with %llu edges\n", out.kmax, (unsigned long long)out.count);
  }

  // (min, max) support over alive edges.
  void minmax(uint32_t& mn, uint32_t& mx) {
    const uint32_t init[2] = {0xffffffffu, 0u};
    copy_h2d(c, mm.get(), init, 8);
    k_alive_min<<<grid_for(na, 256, c->num_sms * 8), 256, 0, c->stream>>>(alive[ai].as<uint32_t>(), na, sup,
                                                                            mm.as<uint32_t>());
    KT_LAUNCHED(c);
    uint32_t h[2];
    copy_d2h(c, h, mm.get(), 8);
    mn = h[0];
    mx = h[1];
  }
};

}  // namespace

void build_sub_from_keys(Ctx* c, uint64_t* keys, uint64_t m, uint32_t n_ids, Sub& out, bool sorted) {
  Graph g;
  build_graph(c, keys, m, n_ids, g, false, sorted);
  build_sub_all(c, g, out);
}

PeelResult truss_peel(Ctx* c, const Sub& s, uint32_t* sup, uint32_t t0, uint64_t stop_count, uint32_t* truss,
                      uint32_t guess, const GraphTrack* track) {
  PeelResult res;
  if (s.m == 0) return res;
  if (t0 < 3) t0 = 3;
  std::unique_ptr<Sub> own;
  DBuf own_sup;
  Peeler P{c, &s, sup, truss};
  P.res = &res;
  P.track = track;
  P.init();
  uint32_t t = t0;
  if (track) {
    // Batched: every graph climbs its own levels (min-support jumps, its own
    // first level and early stop); a cascade runs all of them at once.
    if (track->ngroups == 0) return res;
    P.init_track(t0);
    for (bool first = true; P.na; first = false) {
      P.cascade(t);
      P.record_groups(first);
    }
    P.account();
    return res;
  }
  // Jump phase: try `guess` (> t0) from a snapshot; halve toward t0 on failure.
  if (!truss && guess > t0) {
    DBuf snap_sup(c, s.m * sizeof(uint32_t)), snap_state(c, s.m * sizeof(uint32_t));
    DBuf snap_deg(c, P.adeg.bytes());
    DBuf snap_bits;
    if (s.W) {
      snap_bits.alloc(c, s.bits.bytes());
      KT_CUDA(cudaMemcpyAsync(snap_bits.get(), s.bits.get(), s.bits.bytes(), cudaMemcpyDeviceToDevice, c->stream));
    }
    KT_CUDA(cudaMemcpyAsync(snap_deg.get(), P.adeg.get(), P.adeg.bytes(), cudaMemcpyDeviceToDevice, c->stream));
    KT_CUDA(cudaMemcpyAsync(snap_sup.get(), sup, s.m * sizeof(uint32_t), cudaMemcpyDeviceToDevice, c->stream));
    KT_CUDA(cudaMemcpyAsync(snap_state.get(), P.state.get(), s.m * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                            c->stream));
    const uint64_t na0 = P.na;
    const int ai0 = P.ai;
    uint32_t g = guess;
    while (g > t0) {
      if (P.try_level(g)) {
        t = g;
        break;
      }
      // Undo: the alive list of the snapshot is still in the other buffer.
      KT_CUDA(cudaMemcpyAsync(sup, snap_sup.get(), s.m * sizeof(uint32_t), cudaMemcpyDeviceToDevice, c->stream));
      KT_CUDA(cudaMemcpyAsync(P.state.get(), snap_state.get(), s.m * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                              c->stream));
      KT_CUDA(cudaMemcpyAsync(P.adeg.get(), snap_deg.get(), P.adeg.bytes(), cudaMemcpyDeviceToDevice, c->stream));
      if (s.W)
        KT_CUDA(cudaMemcpyAsync(s.bits.get(), snap_bits.get(), s.bits.bytes(), cudaMemcpyDeviceToDevice, c->stream));
      P.ai = ai0;
      P.na = na0;
      g = t0 + (g - t0) / 2;
    }
    if (t != t0) {
      // The t-truss is non-empty: continue upward from it.
      uint32_t mn, mx;
      P.minmax(mn, mx);
      res.kmax = mn + 2;
      res.count = P.na;
      t = mn + 3;
      stop_count = 0;
    }
  }
  // Levels climbed one at a time before a long climb turns into a bisection
  // (peel_bisect_after, 0 = never), and the gap to the support bound that
  // makes it one (peel_bisect_gap).
  const uint64_t bisect_after = (uint64_t)std::max<int64_t>(0, c->opt.peel_bisect_after);
  const uint64_t bisect_gap = (uint64_t)std::max<int64_t>(1, c->opt.peel_bisect_gap);
  bool first = true;
  uint32_t climbed = 0;
  while (true) {
    const uint64_t left = P.cascade(t);
    if (left == 0) break;
    if (first && stop_count && left == stop_count) {
      res.kmax = t;
      res.count = left;
      res.stopped_early = true;
      P.account();
      return res;
    }
    first = false;
    uint32_t mn, mx;
    P.minmax(mn, mx);
    res.kmax = mn + 2;
    res.count = left;
    t = mn + 3;
    P.compact_graph(own, own_sup);
    if (!truss && bisect_after && ++climbed == bisect_after) {
      // No level above the support bound of the alive edges is non-empty
      // (removed edges keep supports below the current level's threshold).
      const uint32_t ub = support_bound(c, P.sup, P.s->m, mx + 2);
      if (ub >= t + bisect_gap) {
        KT_LOG(c, "kt: level %u, support bound %u: bisecting\n", t, ub);
        P.bisect(res.kmax, ub + 1, res);
        break;
      }
    }
  }
  if (res.kmax < 3) {
    res.kmax = 0;
    res.count = 0;
  }
  P.account();
  return res;
}

}  // namespace kt
