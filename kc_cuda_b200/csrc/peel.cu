// Stage (e): truss peeling of the working graph.
//
// Levels: at truss level t every alive edge with support < t-2 is removed,
// round by round, until none is left; the alive edges then form the t-truss.
// If edges remain, their minimum support s makes them an (s+2)-truss, which
// is recorded as the current answer, and the next level is t = s+3 (levels
// where nothing would be removed are skipped).  The last recorded level when
// no edge is left is kmax.
//
// Rounds: the frontier edges of round r carry state r; deleted edges keep
// their round, alive edges kAlive.  A warp takes a frontier edge (u, v) and
// looks up each entry w of the shorter row in the longer one.  A common w
// closes the triangle {e, a = (., w), b = (., w)}; it is skipped if a or b
// was deleted in an earlier round.  Each surviving side edge loses one
// triangle, decremented by exactly one frontier edge of the triangle (the
// one with the smallest id among those in this round).  An edge whose
// support steps from t-2 to t-3 (atomicSub returns t-2) joins the next
// frontier, so each edge enters a frontier once.
//
// The reference keeps doubled supports and subtracts 2 - [m1==st] - [m2==st]
// from both side edges (src/kc.cu:61-159, 886-1056), and steps k by fixed
// strides with host backups and rollbacks (src/kc.cu:1140-1309); the result
// is the same kmax and edge count.
#include <algorithm>

#include "compact.cuh"
#include "subgraph.h"

namespace kt {
namespace {

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

__global__ void k_peel_init(uint64_t m, uint32_t* __restrict__ state, uint32_t* __restrict__ alive) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
    state[e] = kAlive;
    alive[e] = (uint32_t)e;
  }
}

__global__ void k_peel_frontier(const uint32_t* __restrict__ alive, uint64_t na, const uint32_t* __restrict__ sup,
                                uint32_t* __restrict__ state, uint32_t thr, uint32_t r, uint32_t* __restrict__ truss,
                                uint32_t tval, uint32_t* __restrict__ front, unsigned long long* fcnt, uint64_t cap,
                                uint32_t* err) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ((na + 31) & ~31ULL);
       i += (uint64_t)gridDim.x * blockDim.x) {
    bool want = false;
    uint32_t e = 0;
    if (i < na) {
      e = alive[i];
      if (state[e] == kAlive && sup[e] < thr) {
        state[e] = r;
        if (truss) truss[e] = tval;
        want = true;
      }
    }
    push_warp_full(want, e, front, fcnt, cap, err);
  }
}

__global__ void k_peel_round(const uint32_t* __restrict__ front, uint64_t nf, const uint64_t* __restrict__ ends,
                             const uint64_t* __restrict__ off, const uint32_t* __restrict__ adj,
                             const uint32_t* __restrict__ eid, uint32_t* __restrict__ sup,
                             uint32_t* __restrict__ state, uint32_t thr, uint32_t r, uint32_t* __restrict__ truss,
                             uint32_t tval, uint32_t* __restrict__ next, unsigned long long* ncnt, uint64_t cap,
                             uint32_t* err) {
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t f = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); f < nf; f += warps) {
    const uint32_t e = front[f];
    const uint64_t k = ends[e];
    uint32_t x = (uint32_t)(k >> 32), y = (uint32_t)k;
    if (off[x + 1] - off[x] > off[y + 1] - off[y]) {
      const uint32_t t = x;
      x = y;
      y = t;
    }
    const uint64_t ab = off[x], ae = off[x + 1], bb = off[y], be = off[y + 1];
    for (uint64_t q = ab + lane_id(); q < ab + ((ae - ab + 31) & ~31ULL); q += 32) {
      bool pa = false, pb = false;
      uint32_t a = 0, b = 0;
      if (q < ae) {
        const uint64_t p = find_sorted(adj, bb, be, adj[q]);
        if (p != be) {
          a = eid[q];
          b = eid[p];
          const uint32_t sa = state[a], sb = state[b];
          if (sa >= r && sb >= r) {
            if (sa > r && !(sb == r && b < e)) {
              if (atomicSub(&sup[a], 1u) == thr) {
                state[a] = r + 1;
                if (truss) truss[a] = tval;
                pa = true;
              }
            }
            if (sb > r && !(sa == r && a < e)) {
              if (atomicSub(&sup[b], 1u) == thr) {
                state[b] = r + 1;
                if (truss) truss[b] = tval;
                pb = true;
              }
            }
          }
        }
      }
      push_warp_full(pa, a, next, ncnt, cap, err);
      push_warp_full(pb, b, next, ncnt, cap, err);
    }
  }
}

__global__ void k_alive_min(const uint32_t* __restrict__ alive, uint64_t na, const uint32_t* __restrict__ sup,
                            uint32_t* out) {
  uint32_t mn = 0xffffffffu;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += (uint64_t)gridDim.x * blockDim.x)
    mn = min(mn, sup[alive[i]]);
  mn = warp_min(mn);
  if (lane_id() == 0 && mn != 0xffffffffu) atomicMin(out, mn);
}

struct StillAlive {
  const uint32_t* list;
  const uint32_t* state;
  __device__ bool keep(uint64_t i) const { return state[list[i]] == kAlive; }
  __device__ uint32_t value(uint64_t i) const { return list[i]; }
};

}  // namespace

PeelResult truss_peel(Ctx* c, const Sub& s, uint32_t* sup, uint32_t t0, uint64_t stop_count, uint32_t* truss) {
  PeelResult res;
  const uint64_t m = s.m;
  if (m == 0) return res;
  if (t0 < 3) t0 = 3;
  DBuf state(c, m * sizeof(uint32_t));
  DBuf alive[2] = {DBuf(c, m * sizeof(uint32_t)), DBuf(c, m * sizeof(uint32_t))};
  DBuf front[2] = {DBuf(c, m * sizeof(uint32_t)), DBuf(c, m * sizeof(uint32_t))};
  DBuf cnt(c, 4 * sizeof(unsigned long long));
  DBuf mn(c, 4);
  unsigned long long* cn = cnt.as<unsigned long long>();
  uint32_t* err = &dev_words(c)->err;
  k_peel_init<<<grid_for(m, 256, c->num_sms * 16), 256, 0, c->stream>>>(m, state.as<uint32_t>(),
                                                                          alive[0].as<uint32_t>());
  KT_LAUNCHED(c);
  int ai = 0;
  uint64_t na = m;
  uint32_t t = t0;
  uint32_t r = 0;
  cudaEvent_t e0 = c->ev[2], e1 = c->ev[3];
  bool first = true;
  while (true) {
    // Remove everything below t-2, round by round.
    ++r;
    zero(c, cn, 4 * sizeof(unsigned long long));
    const uint32_t thr = t - 2, tval = t - 1;
    if (c->opt.record_kernel_times) KT_CUDA(cudaEventRecord(e0, c->stream));
    k_peel_frontier<<<grid_for(na, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        alive[ai].as<uint32_t>(), na, sup, state.as<uint32_t>(), thr, r, truss, tval, front[0].as<uint32_t>(), cn + 0,
        m, err);
    KT_LAUNCHED(c);
    int cur = 0;
    while (true) {
      const uint64_t nf = read_word<unsigned long long>(c, cn + cur);
      if (nf == 0) break;
      ++res.rounds;
      KT_CUDA(cudaMemsetAsync(cn + (cur ^ 1), 0, sizeof(unsigned long long), c->stream));
      k_peel_round<<<grid_for(nf * 32, 256, c->num_sms * 16), 256, 0, c->stream>>>(
          front[cur].as<uint32_t>(), nf, s.ends.as<uint64_t>(), s.off.as<uint64_t>(), s.adj.as<uint32_t>(),
          s.eid.as<uint32_t>(), sup, state.as<uint32_t>(), thr, r, truss, tval, front[cur ^ 1].as<uint32_t>(),
          cn + (cur ^ 1), m, err);
      KT_LAUNCHED(c);
      c->stats.peel_launches++;
      ++r;
      cur ^= 1;
    }
    if (c->opt.record_kernel_times) {
      KT_CUDA(cudaEventRecord(e1, c->stream));
      KT_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      KT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      c->stats.ms_peel_kernel += ms;
    }
    ++res.levels;
    check_words(c, "truss peel");
    // Survivors form the t-truss.
    na = compact(c, na, StillAlive{alive[ai].as<uint32_t>(), state.as<uint32_t>()}, alive[ai ^ 1].as<uint32_t>());
    ai ^= 1;
    if (na == 0) break;
    if (first && stop_count && na == stop_count) {
      res.kmax = t;
      res.count = na;
      res.stopped_early = true;
      return res;
    }
    first = false;
    KT_CUDA(cudaMemsetAsync(mn.get(), 0xff, 4, c->stream));
    k_alive_min<<<grid_for(na, 256, c->num_sms * 8), 256, 0, c->stream>>>(alive[ai].as<uint32_t>(), na, sup,
                                                                            mn.as<uint32_t>());
    KT_LAUNCHED(c);
    const uint32_t smin = read_word<uint32_t>(c, mn.as<uint32_t>());
    res.kmax = smin + 2;
    res.count = na;
    t = smin + 3;
  }
  if (res.kmax < 3) {
    res.kmax = 0;
    res.count = 0;
  }
  return res;
}

}  // namespace kt
