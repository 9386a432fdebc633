// Stage (c): k-core peeling on the full graph.
//
// A probe peels the current vertex set to its k-core: the vertices of degree
// < k form the first frontier, and each round removes the frontier and
// decrements the degrees of its surviving neighbours; a neighbour whose
// degree steps from k to k-1 (atomicSub returns k) joins the next frontier,
// so every vertex enters a frontier at most once.  Rows of more than
// kcore_big_row (option, 512) entries are cut into 32-entry windows dealt to
// every warp of the grid, so hub rows do not serialise on one warp.
//
// The search for the maximum core (the reference steps k by a fixed stride
// with host backups, src/kc.cu:770-884) ramps k geometrically from the
// current core (each success is permanent; removed vertices keep the probe's
// tag), then bisects; a probe that empties the graph is undone by reviving
// its tag and recounting degrees.  The tags of successful probes increase
// with their level, which lets any lower core be restored later without a
// snapshot: revive the vertices whose tag is newer than the last probe at or
// below that level, recount degrees, and probe once more.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "compact.cuh"
#include "kcore.h"

namespace kt {
namespace {

constexpr unsigned kBigRow = 2048;

struct AliveF {
  const uint32_t* rem;
  __device__ bool keep(uint64_t v) const { return rem[v] == kAlive; }
  __device__ uint32_t value(uint64_t v) const { return (uint32_t)v; }
};

__global__ void k_init_state(const uint32_t* __restrict__ deg0, uint64_t n, uint32_t* __restrict__ deg,
                             uint32_t* __restrict__ rem) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t d = deg0[v];
    deg[v] = d;
    rem[v] = d ? kAlive : 0u;  // isolated vertices leave at tag 0 (level 1)
  }
}

// Warp-aggregated push of `want` lanes into list[cnt...].
__device__ __forceinline__ void push_warp(bool want, uint32_t item, uint32_t* list, unsigned long long* cnt,
                                          uint64_t cap, uint32_t* err) {
  const unsigned b = __ballot_sync(__activemask(), want);
  if (!b) return;
  const unsigned leader = __ffs(b) - 1;
  unsigned long long base = 0;
  if (lane_id() == leader) base = atomicAdd(cnt, (unsigned long long)__popc(b));
  base = __shfl_sync(__activemask(), base, leader);
  if (want) {
    const unsigned long long p = base + __popc(b & lanemask_lt());
    if (p < cap)
      list[p] = item;
    else
      atomicOr(err, kDevErrCapacity);
  }
}

constexpr unsigned kBigBatch = 1024;  // big rows per batch of dealt windows

// Deals the kWin-entry windows of the big rows big[0..nbig) to every warp of
// the grid, so one long row is spread over the whole GPU instead of one
// block: each block lists the rows' first window numbers (the same block scan
// in every block, kBigBatch rows at a time) and warp w takes windows w,
// w + warps, ...; `drop(b, e)` handles entries [b, e) (at most kWin) of a
// row.  Every thread of the block must call it (it synchronises the block);
// blocks have 256 threads.
template <unsigned kWin, class Drop>
__device__ __forceinline__ void deal_big_windows(const uint32_t* __restrict__ big, uint64_t nbig,
                                                 const uint64_t* __restrict__ off, uint64_t* woff, uint64_t* tmp,
                                                 Drop drop) {
  const uint64_t gwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const uint64_t gwarp = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp_id();
  constexpr unsigned per = kBigBatch / 256;  // rows per thread
  for (uint64_t base = 0; base < nbig; base += kBigBatch) {
    const uint64_t left = nbig - base;
    const uint32_t cnt = left < kBigBatch ? (uint32_t)left : kBigBatch;
    uint64_t w[per];
    uint64_t sum = 0;
#pragma unroll
    for (unsigned j = 0; j < per; ++j) {
      const uint32_t r = threadIdx.x * per + j;
      w[j] = 0;
      if (r < cnt) {
        const uint32_t v = big[base + r];
        w[j] = (off[v + 1] - off[v] + kWin - 1) / kWin;
      }
      sum += w[j];
    }
    uint64_t total;
    uint64_t pre = block_excl_scan<uint64_t>(sum, tmp, &total);
#pragma unroll
    for (unsigned j = 0; j < per; ++j) {
      const uint32_t r = threadIdx.x * per + j;
      if (r < cnt) woff[r] = pre;
      pre += w[j];
    }
    if (threadIdx.x == 0) woff[cnt] = total;
    __syncthreads();
    for (uint64_t x = gwarp; x < total; x += gwarps) {
      uint32_t lo = 0, hi = cnt;  // last row with woff <= x
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (woff[mid] <= x)
          lo = mid;
        else
          hi = mid;
      }
      const uint32_t v = big[base + lo];
      const uint64_t b = off[v] + (x - woff[lo]) * kWin, e = min(off[v + 1], b + kWin);
      drop(b, e);
    }
    __syncthreads();
  }
}

__global__ void k_frontier_init(const uint32_t* __restrict__ alive, uint64_t n_alive, const uint32_t* __restrict__ deg,
                                uint32_t* __restrict__ rem, uint32_t k, uint32_t tag, uint32_t* __restrict__ front,
                                unsigned long long* fcnt, uint64_t cap, uint32_t* err) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ((n_alive + 31) & ~31ULL);
       i += (uint64_t)gridDim.x * blockDim.x) {
    bool want = false;
    uint32_t v = 0;
    if (i < n_alive) {
      v = alive[i];
      if (rem[v] == kAlive && deg[v] < k) {
        rem[v] = tag;
        want = true;
      }
    }
    push_warp(want, v, front, fcnt, cap, err);
  }
}

// Removes the frontier: warp per vertex; rows longer than big_row go to the
// big list for k_expand_big.
__global__ void k_expand(const uint32_t* __restrict__ front, uint64_t nf, const uint64_t* __restrict__ off,
                         const uint32_t* __restrict__ adj, uint32_t* __restrict__ deg, uint32_t* __restrict__ rem,
                         uint32_t k, uint32_t tag, uint32_t* __restrict__ next, unsigned long long* ncnt,
                         uint32_t* __restrict__ big, unsigned long long* nbig, uint64_t cap, uint32_t* err,
                         uint32_t big_row) {
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t f = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); f < nf; f += warps) {
    const uint32_t v = front[f];
    const uint64_t b = off[v], e = off[v + 1];
    if (e - b > big_row) {
      if (lane_id() == 0) {
        const unsigned long long p = atomicAdd(nbig, 1ULL);
        if (p < cap)
          big[p] = v;
        else
          atomicOr(err, kDevErrCapacity);
      }
      continue;
    }
    for (uint64_t j = b + lane_id(); j < ((e - b + 31) & ~31ULL) + b; j += 32) {
      bool want = false;
      uint32_t w = 0;
      if (j < e) {
        w = adj[j];
        if (rem[w] == kAlive) {
          const uint32_t old = atomicSub(&deg[w], 1u);
          if (old == k) {
            rem[w] = tag;
            want = true;
          }
        }
      }
      push_warp(want, w, next, ncnt, cap, err);
    }
  }
}

// Big rows: one block per row (rows round-robin over blocks), each warp
// taking 32-entry windows of it.
__global__ void k_expand_big(const uint32_t* __restrict__ big, const unsigned long long* nbig_p,
                             const uint64_t* __restrict__ off, const uint32_t* __restrict__ adj,
                             uint32_t* __restrict__ deg, uint32_t* __restrict__ rem, uint32_t k, uint32_t tag,
                             uint32_t* __restrict__ next, unsigned long long* ncnt, uint64_t cap, uint32_t* err) {
  const uint64_t nbig = *nbig_p;
  for (uint64_t bi = blockIdx.x; bi < nbig; bi += gridDim.x) {
    const uint32_t v = big[bi];
    const uint64_t b = off[v], e = off[v + 1];
    for (uint64_t j0 = b + warp_id() * 32; j0 < e; j0 += blockDim.x) {
      const uint64_t j = j0 + lane_id();
      bool want = false;
      uint32_t w = 0;
      if (j < e) {
        w = adj[j];
        if (rem[w] == kAlive) {
          const uint32_t old = atomicSub(&deg[w], 1u);
          if (old == k) {
            rem[w] = tag;
            want = true;
          }
        }
      }
      push_warp(want, w, next, ncnt, cap, err);
    }
  }
}

// deg[v] = alive neighbours of v, for v in the alive list (big rows by blocks).
__global__ void k_recount(const uint32_t* __restrict__ alive, uint64_t n_alive, const uint64_t* __restrict__ off,
                          const uint32_t* __restrict__ adj, const uint32_t* __restrict__ rem,
                          uint32_t* __restrict__ deg, uint32_t* __restrict__ big, unsigned long long* nbig,
                          uint64_t cap, uint32_t* err, uint32_t big_row) {
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t i = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); i < n_alive; i += warps) {
    const uint32_t v = alive[i];
    const uint64_t b = off[v], e = off[v + 1];
    if (e - b > big_row) {
      if (lane_id() == 0) {
        deg[v] = 0;
        const unsigned long long p = atomicAdd(nbig, 1ULL);
        if (p < cap)
          big[p] = v;
        else
          atomicOr(err, kDevErrCapacity);
      }
      continue;
    }
    uint32_t c = 0;
    for (uint64_t j = b + lane_id(); j < e; j += 32) c += rem[adj[j]] == kAlive;
    c = warp_sum(c);
    if (lane_id() == 0) deg[v] = c;
  }
}

// Big rows of the recount: one block per row, a warp-level count and one
// atomic per warp per row.
__global__ void k_recount_big(const uint32_t* __restrict__ big, const unsigned long long* nbig_p,
                              const uint64_t* __restrict__ off, const uint32_t* __restrict__ adj,
                              const uint32_t* __restrict__ rem, uint32_t* __restrict__ deg) {
  const uint64_t nbig = *nbig_p;
  for (uint64_t bi = blockIdx.x; bi < nbig; bi += gridDim.x) {
    const uint32_t v = big[bi];
    const uint64_t b = off[v], e = off[v + 1];
    uint32_t c = 0;
    for (uint64_t j = b + threadIdx.x; j < e; j += blockDim.x) c += rem[adj[j]] == kAlive;
    c = warp_sum(c);
    if (lane_id() == 0 && c) atomicAdd(&deg[v], c);
  }
}

__global__ void k_revive(uint32_t* __restrict__ rem, uint64_t n, uint32_t newer_than) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t r = rem[v];
    if (r != kAlive && r > newer_than) rem[v] = kAlive;
  }
}

// Minimum alive degree into *out; with `sum`, also the sum of the alive
// degrees (twice the alive edges).
__global__ void k_min_alive_deg(const uint32_t* __restrict__ alive, uint64_t n_alive, const uint32_t* __restrict__ deg,
                                const uint32_t* __restrict__ rem, uint32_t* out,
                                unsigned long long* sum = nullptr) {
  uint32_t mn = 0xffffffffu;
  uint64_t s = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_alive; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = alive[i];
    if (rem[v] == kAlive) {
      mn = min(mn, deg[v]);
      s += deg[v];
    }
  }
  mn = warp_min(mn);
  if (lane_id() == 0 && mn != 0xffffffffu) atomicMin(out, mn);
  if (sum) {
    s = warp_sum(s);
    if (lane_id() == 0 && s) atomicAdd(sum, (unsigned long long)s);
  }
}

__global__ void k_members(const uint32_t* __restrict__ rem, uint64_t n, uint8_t* __restrict__ out) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    out[v] = rem[v] == kAlive;
}

__global__ void k_core_from_tags(const uint32_t* __restrict__ rem, uint64_t n, const uint32_t* __restrict__ level,
                                 uint32_t* __restrict__ core) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t r = rem[v];
    core[v] = r == kAlive ? 0u : level[r] - 1;
  }
}


// Compacted copy of the alive part: row i of the new graph is alive[i] with
// only its alive neighbours, renumbered.
__global__ void k_compact_rows(const uint32_t* __restrict__ alive, uint64_t na, const uint64_t* __restrict__ off,
                               const uint32_t* __restrict__ adj, const uint32_t* __restrict__ rem,
                               const uint32_t* __restrict__ newid, const uint64_t* __restrict__ noff,
                               uint32_t* __restrict__ nadj) {
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t i = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); i < na; i += warps) {
    const uint32_t v = alive[i];
    const uint64_t b = off[v], e = off[v + 1];
    if (e - b > kBigRow) continue;  // k_compact_big_rows
    uint64_t pos = noff[i];
    const uint64_t end = noff[i + 1];
    for (uint64_t j = b + lane_id(); j < b + ((e - b + 31) & ~31ULL); j += 32) {
      bool keep = false;
      uint32_t w = 0;
      if (j < e) {
        w = adj[j];
        keep = rem[w] == kAlive;
      }
      const unsigned bal = __ballot_sync(kFull, keep);
      const uint64_t p = pos + __popc(bal & lanemask_lt());
      if (keep && p < end) nadj[p] = newid[w];
      pos += __popc(bal);
    }
  }
}

// Alive-list indices whose rows are longer than kBigRow (compacted apart).
struct BigAliveRow {
  const uint32_t* alive;
  const uint64_t* off;
  __device__ bool keep(uint64_t i) const {
    const uint32_t v = alive[i];
    return off[v + 1] - off[v] > kBigRow;
  }
  __device__ uint32_t value(uint64_t i) const { return (uint32_t)i; }
};

// Rows longer than kBigRow in the compaction: their 256-entry chunks are
// dealt to every warp of the grid (each block lists the rows' first chunk
// numbers with the same block scan, kBigBatch rows at a time); a warp loads
// its chunk's 8 entries per lane, their alive flags and new ids before it
// uses any of them (so 8 loads of each kind are in flight per lane), and
// the chunk's kept entries go to the row's next free positions (a per-row
// cursor, one atomic per chunk), so a hub row is spread over the whole GPU.
// Entry order within these rows is not kept; nothing downstream needs it.
constexpr unsigned kCompactChunk = 256;  // entries per warp step (8 per lane)

__global__ void __launch_bounds__(256) k_compact_big_rows(const uint32_t* __restrict__ rows, uint64_t nrows,
                                                          const uint32_t* __restrict__ alive,
                                                          const uint64_t* __restrict__ off,
                                                          const uint32_t* __restrict__ adj,
                                                          const uint32_t* __restrict__ rem,
                                                          const uint32_t* __restrict__ newid,
                                                          const uint64_t* __restrict__ noff,
                                                          uint32_t* __restrict__ cursor, uint32_t* __restrict__ nadj) {
  __shared__ uint64_t woff[kBigBatch + 1];
  __shared__ uint64_t tmp[33];
  constexpr unsigned kPer = kCompactChunk / 32;
  const uint64_t gwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const uint64_t gwarp = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp_id();
  const unsigned l = lane_id();
  constexpr unsigned per = kBigBatch / 256;  // rows per thread
  for (uint64_t base = 0; base < nrows; base += kBigBatch) {
    const uint64_t left = nrows - base;
    const uint32_t cnt = left < kBigBatch ? (uint32_t)left : kBigBatch;
    uint64_t w[per];
    uint64_t sum = 0;
#pragma unroll
    for (unsigned j = 0; j < per; ++j) {
      const uint32_t r = threadIdx.x * per + j;
      w[j] = 0;
      if (r < cnt) {
        const uint32_t v = alive[rows[base + r]];
        w[j] = (off[v + 1] - off[v] + kCompactChunk - 1) / kCompactChunk;
      }
      sum += w[j];
    }
    uint64_t total;
    uint64_t pre = block_excl_scan<uint64_t>(sum, tmp, &total);
#pragma unroll
    for (unsigned j = 0; j < per; ++j) {
      const uint32_t r = threadIdx.x * per + j;
      if (r < cnt) woff[r] = pre;
      pre += w[j];
    }
    if (threadIdx.x == 0) woff[cnt] = total;
    __syncthreads();
    for (uint64_t x = gwarp; x < total; x += gwarps) {
      uint32_t lo = 0, hi = cnt;  // last row with woff <= x
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (woff[mid] <= x)
          lo = mid;
        else
          hi = mid;
      }
      const uint32_t i = rows[base + lo];
      const uint32_t v = alive[i];
      const uint64_t e = off[v + 1];
      const uint64_t j0 = off[v] + (x - woff[lo]) * kCompactChunk + l;
      uint32_t u[kPer];
#pragma unroll
      for (unsigned k = 0; k < kPer; ++k) u[k] = j0 + 32 * k < e ? adj[j0 + 32 * k] : 0u;
      bool keep[kPer];
#pragma unroll
      for (unsigned k = 0; k < kPer; ++k) keep[k] = j0 + 32 * k < e && rem[u[k]] == kAlive;
#pragma unroll
      for (unsigned k = 0; k < kPer; ++k) u[k] = keep[k] ? newid[u[k]] : 0u;
      unsigned bal[kPer];
      uint32_t kept = 0;
#pragma unroll
      for (unsigned k = 0; k < kPer; ++k) {
        bal[k] = __ballot_sync(kFull, keep[k]);
        kept += __popc(bal[k]);
      }
      if (!kept) continue;
      uint32_t at = 0;
      if (l == 0) at = atomicAdd(&cursor[base + lo], kept);
      at = __shfl_sync(kFull, at, 0);
      const uint64_t row0 = noff[i], row1 = noff[i + 1];
      uint64_t p0 = row0 + at;
#pragma unroll
      for (unsigned k = 0; k < kPer; ++k) {
        const uint64_t p = p0 + __popc(bal[k] & lanemask_lt());
        if (keep[k] && p < row1) nadj[p] = u[k];
        p0 += __popc(bal[k]);
      }
    }
    __syncthreads();
  }
}

__global__ void k_compact_meta(const uint32_t* __restrict__ alive, uint64_t na, const uint32_t* __restrict__ deg,
                               const uint32_t* __restrict__ oldmap, uint32_t* __restrict__ newid,
                               uint32_t* __restrict__ ndeg, uint32_t* __restrict__ nmap) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = alive[i];
    newid[v] = (uint32_t)i;
    ndeg[i] = deg[v];
    nmap[i] = oldmap ? oldmap[v] : v;
  }
}

__global__ void k_members_mapped(const uint32_t* __restrict__ rem, uint64_t n, const uint32_t* __restrict__ map,
                                 uint8_t* __restrict__ out) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    if (rem[v] == kAlive) out[map[v]] = 1;
}


struct ProbeArgs {
  const uint64_t* off;
  const uint32_t* adj;
  uint32_t* deg;
  uint32_t* rem;
  const uint32_t* alive;
  uint64_t n_alive;
  uint32_t* front[2];
  uint32_t* big;
  unsigned long long* cnt;  // [0..2] frontier sizes, [3..4] big-row counts, [5] rounds, [6] removed, [7] stopped
  uint64_t cap;
  uint32_t k, tag;
  bool may_stop;     // stop once fewer than k+1 vertices can remain (the k-core is then empty)
  uint32_t big_row;  // rows longer than this are dealt to all warps in windows
  DevWords* words;
  unsigned long long timeout_ns;
};

__device__ __forceinline__ void drop_neighbours(const ProbeArgs& A, uint64_t b, uint64_t e, uint32_t* next,
                                                unsigned long long* ncnt) {
  for (uint64_t j = b + lane_id(); j < b + ((e - b + 31) & ~31ULL); j += 32) {
    bool want = false;
    uint32_t w = 0;
    if (j < e) {
      w = A.adj[j];
      if (A.rem[w] == kAlive) {
        const uint32_t old = atomicSub(&A.deg[w], 1u);
        if (old == A.k) {
          A.rem[w] = A.tag;
          want = true;
        }
      }
    }
    push_warp(want, w, next, ncnt, A.cap, &A.words->err);
  }
}

// drop_neighbours for up to 256 entries [b, e): each lane loads its 8
// entries, their alive flags, then decrements their degrees, before it uses
// any result, so 8 loads and 8 atomics of each lane are in flight at once
// (the big rows' windows in a probe).
__device__ __forceinline__ void drop_neighbours_wide(const ProbeArgs& A, uint64_t b, uint64_t e, uint32_t* next,
                                                     unsigned long long* ncnt) {
  constexpr unsigned kPer = 8;
  const uint64_t j0 = b + lane_id();
  uint32_t w[kPer];
#pragma unroll
  for (unsigned k = 0; k < kPer; ++k) w[k] = j0 + 32 * k < e ? A.adj[j0 + 32 * k] : 0u;
  bool live[kPer];
#pragma unroll
  for (unsigned k = 0; k < kPer; ++k) live[k] = j0 + 32 * k < e && A.rem[w[k]] == kAlive;
  uint32_t old[kPer];
#pragma unroll
  for (unsigned k = 0; k < kPer; ++k) old[k] = live[k] ? atomicSub(&A.deg[w[k]], 1u) : 0u;
#pragma unroll
  for (unsigned k = 0; k < kPer; ++k) {
    const bool want = live[k] && old[k] == A.k;
    if (want) A.rem[w[k]] = A.tag;
    push_warp(want, w[k], next, ncnt, A.cap, &A.words->err);
  }
}

// A whole probe (frontier init and every round) in one cooperative launch.
__global__ void __launch_bounds__(256, 4) k_probe(ProbeArgs A) {
  __shared__ uint64_t woff[kBigBatch + 1];
  __shared__ uint64_t wtmp[33];
  const uint64_t gthreads = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t gwarps = gthreads >> 5, gwarp = gtid >> 5;
  for (uint64_t i = gtid; i < ((A.n_alive + 31) & ~31ULL); i += gthreads) {
    bool want = false;
    uint32_t v = 0;
    if (i < A.n_alive) {
      v = A.alive[i];
      if (A.rem[v] == kAlive && A.deg[v] < A.k) {
        A.rem[v] = A.tag;
        want = true;
      }
    }
    push_warp(want, v, A.front[0], &A.cnt[0], A.cap, &A.words->err);
  }
  if (!grid_barrier(A.words, A.timeout_ns)) return;
  uint32_t i = 0;
  uint64_t removed = 0;
  bool stopped = false;
  while (true) {
    const uint64_t nf = ld_acquire_u64(&A.cnt[i % 3]);
    if (nf == 0) break;
    removed += nf;
    // Every block reads the same counts, so all of them stop together.
    if (A.may_stop && A.n_alive - removed < (uint64_t)A.k + 1) {
      stopped = true;
      break;
    }
    const uint32_t* fr = A.front[i & 1];
    uint32_t* nx = A.front[(i + 1) & 1];
    unsigned long long* nc = &A.cnt[(i + 1) % 3];
    unsigned long long* bc = &A.cnt[3 + (i & 1)];
    for (uint64_t f = gwarp; f < nf; f += gwarps) {
      const uint32_t v = fr[f];
      const uint64_t b = A.off[v], e = A.off[v + 1];
      if (e - b > A.big_row) {
        if (lane_id() == 0) {
          const unsigned long long p = atomicAdd(bc, 1ULL);
          if (p < A.cap)
            A.big[p] = v;
          else
            atomicOr(&A.words->err, kDevErrCapacity);
        }
        continue;
      }
      drop_neighbours(A, b, e, nx, nc);
    }
    if (gtid == 0) {
      A.cnt[(i + 2) % 3] = 0;        // read at the start of round i-1
      A.cnt[3 + ((i + 1) & 1)] = 0;  // big count of round i-1, read before the barrier ending it
    }
    if (!grid_barrier(A.words, A.timeout_ns)) return;
    const uint64_t nbig = ld_acquire_u64(bc);
    if (nbig) {
      // Rows longer than big_row: their 256-entry windows dealt to every warp.
      deal_big_windows<256>(A.big, nbig, A.off, woff, wtmp,
                            [&](uint64_t b, uint64_t e) { drop_neighbours_wide(A, b, e, nx, nc); });
      if (!grid_barrier(A.words, A.timeout_ns)) return;
    }
    ++i;
  }
  if (gtid == 0) {
    A.cnt[5] = i;
    A.cnt[6] = removed;
    A.cnt[7] = stopped;
  }
}

// Full core decomposition in one cooperative launch: the level loop runs on
// the device, so thousands of graphs of a batched union (or one graph) are
// decomposed without a host round trip per level.
//
// Level k removes every alive vertex of degree <= k (core number k): a pass
// over a vertex list takes the vertices of degree <= k as the first frontier,
// and the frontier rounds then run as in k_probe (a neighbour stepping from
// k+1 to k joins the next frontier).  Passes are windowed: a full pass over
// the compact alive list opens a window of `window` levels [k, top] and
// lists the candidates, the alive vertices of degree <= top; within the
// window each level's pass reads only the candidates, and a neighbour whose
// degree steps from top+1 to top during the rounds joins them.  So the alive
// list is read once per window instead of once per level.  A pass that finds
// no vertex of degree k moves k to the smallest degree it saw (levels
// without vertices are skipped).
struct DecompArgs {
  const uint64_t* off;
  const uint32_t* adj;
  uint32_t* deg;
  uint32_t* rem;       // kAlive, or 0 once removed
  uint32_t* core;      // out: core number of every removed vertex
  uint32_t* list[2];   // compact alive lists (ping-pong, rewritten by full passes)
  uint32_t* cand[2];   // window candidates (ping-pong, rewritten by every pass)
  uint32_t* front[2];
  uint32_t* big;
  // [0..2] frontier sizes, [3..4] big-row counts; by pass % 3: [5..7]
  // alive-list sizes, [8..10] minimum degrees, [11..13] candidate counts;
  // [14] rounds, [15] levels, [16] passes, [17] full passes, [18] last level
  unsigned long long* cnt;
  uint64_t n_list;     // entries of list[0] at launch
  uint64_t cap;
  uint32_t big_row;    // rows longer than this are dealt to all warps in windows
  uint32_t window;     // levels per window (>= 1)
  DevWords* words;
  unsigned long long timeout_ns;
};

struct DropRule {
  uint32_t k, top;
  uint32_t* next;              // frontier of the next round
  unsigned long long* ncnt;
  uint32_t* cand;              // candidates of this pass
  unsigned long long* ccnt;
};

__device__ __forceinline__ void drop_neighbours_core(const DecompArgs& A, uint64_t b, uint64_t e, const DropRule& R) {
  for (uint64_t j = b + lane_id(); j < b + ((e - b + 31) & ~31ULL); j += 32) {
    bool want = false, join = false;
    uint32_t w = 0;
    if (j < e) {
      w = A.adj[j];
      if (A.rem[w] == kAlive) {
        const uint32_t old = atomicSub(&A.deg[w], 1u);
        if (old == R.k + 1) {
          A.rem[w] = 0u;
          A.core[w] = R.k;
          want = true;
        } else if (old == R.top + 1) {
          join = true;  // its degree entered the window
        }
      }
    }
    push_warp(want, w, R.next, R.ncnt, A.cap, &A.words->err);
    push_warp(join, w, R.cand, R.ccnt, A.cap, &A.words->err);
  }
}

// One thread per block reads a device counter after a grid barrier and
// shares it through shared memory (one L2 request per block, not per warp).
__device__ __forceinline__ unsigned long long block_read(const unsigned long long* p, unsigned long long* sh) {
  if (threadIdx.x == 0) *sh = ld_acquire_u64(p);
  __syncthreads();
  const unsigned long long v = *sh;
  __syncthreads();
  return v;
}

__global__ void __launch_bounds__(256, 4) k_core_levels(DecompArgs A) {
  __shared__ unsigned long long sh;
  __shared__ uint64_t woff[kBigBatch + 1];
  __shared__ uint64_t wtmp[33];
  const uint64_t gthreads = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t gwarps = gthreads >> 5, gwarp = gtid >> 5;
  uint64_t nl = A.n_list;  // entries of the current alive list
  uint64_t nc = 0;         // entries of the current candidate list
  uint32_t k = 1;          // every alive vertex has degree >= k
  uint32_t top = 0;        // candidates: every alive vertex of degree <= top
  bool full = true;        // the next pass reads the alive list
  uint32_t i = 0;          // frontier round index, continued across levels
  uint32_t ps = 0, li = 0, ci = 0;
  unsigned long long levels_run = 0, full_passes = 0;
  while (true) {
    unsigned long long* lc = &A.cnt[5 + ps % 3];
    unsigned long long* mc = &A.cnt[8 + ps % 3];
    unsigned long long* cc = &A.cnt[11 + ps % 3];
    if (gtid == 0) {
      // Read two passes ago, before the barriers that ended the last pass.
      A.cnt[5 + (ps + 1) % 3] = 0;
      A.cnt[8 + (ps + 1) % 3] = ~0ULL;
      A.cnt[11 + (ps + 1) % 3] = 0;
      // The pass pushes the frontier of round i + 1.  Slot i % 3 (empty; it
      // ended the last level) may still be being read by slower blocks, so it
      // is left alone; slot (i + 2) % 3 and round i + 1's big-row count were
      // read before the barriers that ended round i - 1, and are cleared.
      A.cnt[(i + 2) % 3] = 0;
      A.cnt[3 + ((i + 1) & 1)] = 0;
    }
    if (full) {
      top = k + A.window - 1;
      ++full_passes;
    }
    const uint32_t* src = full ? (li ? A.list[1] : A.list[0]) : (ci ? A.cand[1] : A.cand[0]);
    const uint64_t nsrc = full ? nl : nc;
    uint32_t* lnext = li ? A.list[0] : A.list[1];
    uint32_t* cnext = ci ? A.cand[0] : A.cand[1];
    uint32_t mn = 0xffffffffu;
    for (uint64_t j = gtid; j < ((nsrc + 31) & ~31ULL); j += gthreads) {
      bool out = false, keep = false, cand = false;
      uint32_t v = 0;
      if (j < nsrc) {
        v = src[j];
        if (A.rem[v] == kAlive) {
          const uint32_t d = A.deg[v];
          if (d <= k) {
            A.rem[v] = 0u;
            A.core[v] = k;
            out = true;
          } else {
            keep = full;
            cand = d <= top;
            mn = min(mn, d);
          }
        }
      }
      push_warp(out, v, (i & 1) ? A.front[0] : A.front[1], &A.cnt[(i + 1) % 3], A.cap, &A.words->err);
      if (full) push_warp(keep, v, lnext, lc, A.cap, &A.words->err);
      push_warp(cand, v, cnext, cc, A.cap, &A.words->err);
    }
    mn = warp_min(mn);
    if (lane_id() == 0 && mn != 0xffffffffu) atomicMin(mc, (unsigned long long)mn);
    if (!grid_barrier(A.words, A.timeout_ns)) return;
    if (full) {
      nl = block_read(lc, &sh);
      li ^= 1;
    }
    const unsigned long long dmin = block_read(mc, &sh);
    ++ps;
    // The pass's frontier is round i + 1's; i advances even when it is empty,
    // so the next pass counts into a slot no slower block is still reading.
    ++i;
    if (block_read(&A.cnt[i % 3], &sh) == 0) {
      nc = block_read(cc, &sh);
      ci ^= 1;
      if (full) {
        if (nl == 0) break;  // nothing alive
        k = (uint32_t)dmin;  // the candidates hold level dmin's vertices when it is in the window
        full = k > top;
      } else if (nc) {
        k = (uint32_t)dmin;  // the smallest candidate degree (<= top)
      } else {
        k = top + 1;  // no alive vertex of degree <= top: open the next window
        full = true;
      }
      continue;
    }
    ++levels_run;
    // Frontier rounds of level k.
    DropRule R{k, top, nullptr, nullptr, cnext, cc};
    while (true) {
      const uint64_t nf = block_read(&A.cnt[i % 3], &sh);
      if (nf == 0) break;
      const uint32_t* fr = (i & 1) ? A.front[1] : A.front[0];
      R.next = (i & 1) ? A.front[0] : A.front[1];
      R.ncnt = &A.cnt[(i + 1) % 3];
      unsigned long long* bc = &A.cnt[3 + (i & 1)];
      for (uint64_t f = gwarp; f < nf; f += gwarps) {
        const uint32_t v = fr[f];
        const uint64_t b = A.off[v], e = A.off[v + 1];
        if (e - b > A.big_row) {
          if (lane_id() == 0) {
            const unsigned long long p = atomicAdd(bc, 1ULL);
            if (p < A.cap)
              A.big[p] = v;
            else
              atomicOr(&A.words->err, kDevErrCapacity);
          }
          continue;
        }
        drop_neighbours_core(A, b, e, R);
      }
      if (gtid == 0) {
        A.cnt[(i + 2) % 3] = 0;
        A.cnt[3 + ((i + 1) & 1)] = 0;
      }
      if (!grid_barrier(A.words, A.timeout_ns)) return;
      const uint64_t nbig = block_read(bc, &sh);
      if (nbig) {
        deal_big_windows<32>(A.big, nbig, A.off, woff, wtmp,
                             [&](uint64_t b, uint64_t e) { drop_neighbours_core(A, b, e, R); });
        if (!grid_barrier(A.words, A.timeout_ns)) return;
      }
      ++i;
    }
    // Every candidate push of this pass is in (rounds end with a barrier).
    nc = block_read(cc, &sh);
    ci ^= 1;
    ++k;  // every survivor now has degree >= k
    full = k > top;
  }
  if (gtid == 0) {
    A.cnt[14] = i;
    A.cnt[15] = levels_run;
    A.cnt[16] = ps;
    A.cnt[17] = full_passes;
    A.cnt[18] = k;
  }
}

uint32_t big_row(const Ctx* c) {
  return (uint32_t)std::min<int64_t>(std::max<int64_t>(32, c->opt.kcore_big_row), 1 << 30);
}

}  // namespace

void KCore::reset_state(Ctx* c, const Graph& gr) {
  n = gr.n;
  deg.ensure(c, (n ? n : 1) * sizeof(uint32_t));
  rem.ensure(c, (n ? n : 1) * sizeof(uint32_t));
  alive.ensure(c, (n ? n : 1) * sizeof(uint32_t));
  front[0].ensure(c, (n ? n : 1) * sizeof(uint32_t));
  front[1].ensure(c, (n ? n : 1) * sizeof(uint32_t));
  big.ensure(c, (n ? n : 1) * sizeof(uint32_t));
  cnt.ensure(c, 8 * sizeof(unsigned long long));
  if (n) {
    k_init_state<<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(gr.deg.as<uint32_t>(), n,
                                                                             deg.as<uint32_t>(), rem.as<uint32_t>());
    KT_LAUNCHED(c);
  }
  rebuild_alive(c);
}

void KCore::init(Ctx* c, const Graph& gr) {
  base = &gr;
  compacted = false;
  local_level = 0;
  levels.assign(1, 1);  // tag 0 = isolated, left at level 1
  succ.assign(1, 0);
  reset_state(c, gr);
}

void KCore::rebuild_alive(Ctx* c) {
  n_alive = compact(c, n, AliveF{rem.as<uint32_t>()}, alive.as<uint32_t>());
}

void KCore::compact_to_alive(Ctx* c, uint32_t level) {
  const Graph& g = cur();
  const uint64_t na = n_alive;
  Graph L;
  L.n = na;
  DBuf newid(c, (n ? n : 1) * sizeof(uint32_t));
  DBuf nmap(c, (na ? na : 1) * sizeof(uint32_t));
  L.deg.alloc(c, (na + 1) * sizeof(uint32_t));
  zero(c, L.deg.get(), (na + 1) * sizeof(uint32_t));
  k_compact_meta<<<grid_for(na, 256, c->num_sms * 16), 256, 0, c->stream>>>(
      alive.as<uint32_t>(), na, deg.as<uint32_t>(), map(), newid.as<uint32_t>(), L.deg.as<uint32_t>(),
      nmap.as<uint32_t>());
  KT_LAUNCHED(c);
  L.off.alloc(c, (na + 1) * sizeof(uint64_t));
  scan_u32_to_u64(c, L.deg.as<uint32_t>(), L.off.as<uint64_t>(), na + 1);
  const uint64_t n2 = read_word<uint64_t>(c, L.off.as<uint64_t>() + na);
  L.m = n2 / 2;
  L.adj.alloc(c, (n2 ? n2 : 1) * sizeof(uint32_t));
  k_compact_rows<<<grid_for(na * 32, 256, c->num_sms * 16), 256, 0, c->stream>>>(
      alive.as<uint32_t>(), na, g.off.as<uint64_t>(), g.adj.as<uint32_t>(), rem.as<uint32_t>(),
      newid.as<uint32_t>(), L.off.as<uint64_t>(), L.adj.as<uint32_t>());
  KT_LAUNCHED(c);
  {
    DBuf rows(c, (na ? na : 1) * sizeof(uint32_t));
    const uint64_t nbig = compact(c, na, BigAliveRow{alive.as<uint32_t>(), g.off.as<uint64_t>()},
                                  rows.as<uint32_t>());
    if (nbig) {
      DBuf cursor(c, nbig * sizeof(uint32_t));
      zero(c, cursor.get(), cursor.bytes());
      k_compact_big_rows<<<c->num_sms * 8, 256, 0, c->stream>>>(
          rows.as<uint32_t>(), nbig, alive.as<uint32_t>(), g.off.as<uint64_t>(), g.adj.as<uint32_t>(),
          rem.as<uint32_t>(), newid.as<uint32_t>(), L.off.as<uint64_t>(), cursor.as<uint32_t>(),
          L.adj.as<uint32_t>());
      KT_LAUNCHED(c);
    }
  }
  L.max_deg = g.max_deg;  // an upper bound is enough here
  newid.release();
  // Install; the previous compaction, if any, is kept for restores.
  if (compacted) {
    Saved sv;
    sv.local = std::move(local);
    sv.idmap = std::move(idmap);
    sv.level = local_level;
    saved.push_back(std::move(sv));
    local = Graph();
  }
  local.off = std::move(L.off);
  local.adj = std::move(L.adj);
  local.deg = std::move(L.deg);
  local.edges.release();
  local.n = L.n;
  local.m = L.m;
  local.max_deg = L.max_deg;
  idmap = std::move(nmap);
  compacted = true;
  local_level = level;
  levels.assign(1, level);
  succ.assign(1, 0);
  reset_state(c, local);
}

void KCore::recount(Ctx* c) {
  if (!n_alive) return;
  const Graph& g = cur();
  zero(c, cnt.get(), cnt.bytes());
  unsigned long long* nbig = cnt.as<unsigned long long>() + 4;
  k_recount<<<grid_for(n_alive * 32, 256, c->num_sms * 16), 256, 0, c->stream>>>(
      alive.as<uint32_t>(), n_alive, g.off.as<uint64_t>(), g.adj.as<uint32_t>(), rem.as<uint32_t>(),
      deg.as<uint32_t>(), big.as<uint32_t>(), nbig, n, &dev_words(c)->err, big_row(c));
  KT_LAUNCHED(c);
  k_recount_big<<<c->num_sms * 4, 256, 0, c->stream>>>(big.as<uint32_t>(), nbig, g.off.as<uint64_t>(),
                                                       g.adj.as<uint32_t>(), rem.as<uint32_t>(),
                                                       deg.as<uint32_t>());
  KT_LAUNCHED(c);
}

uint64_t KCore::probe(Ctx* c, uint32_t k, bool may_stop) {
  const uint32_t tag = (uint32_t)levels.size();
  if (tag >= 0xfffffff0u) throw Error(KT_ERR_LIMIT, "k-core: too many probes");
  levels.push_back(k);
  if (!n_alive) return 0;
  const Graph& g = cur();
  unsigned long long* cn = cnt.as<unsigned long long>();
  zero(c, cnt.get(), cnt.bytes());
  uint32_t* err = &dev_words(c)->err;
  uint64_t removed = 0;
  if (c->opt.persistent) {
    ProbeArgs A;
    A.off = g.off.as<uint64_t>();
    A.adj = g.adj.as<uint32_t>();
    A.deg = deg.as<uint32_t>();
    A.rem = rem.as<uint32_t>();
    A.alive = alive.as<uint32_t>();
    A.n_alive = n_alive;
    A.front[0] = front[0].as<uint32_t>();
    A.front[1] = front[1].as<uint32_t>();
    A.big = big.as<uint32_t>();
    A.cnt = cn;
    A.cap = n;
    A.k = k;
    A.tag = tag;
    A.may_stop = may_stop;
    A.big_row = big_row(c);
    A.words = dev_words(c);
    A.timeout_ns = (unsigned long long)c->opt.timeout_ms * 1000000ULL;
    if (!coop_grid) {
      int per_sm = 0;
      KT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_probe, 256, 0));
      coop_grid = coop_blocks(c, per_sm);
    }
    void* p[] = {&A};
    uint64_t h[3];
    {
      CoopLock coop(c);
      KT_CUDA(cudaLaunchCooperativeKernel((const void*)k_probe, dim3(coop_grid), dim3(256), p, 0, c->stream));
      KT_LAUNCHED(c);
      copy_d2h(c, h, cn + 5, 24);
    }
    rounds += h[0];
    removed = h[2] ? n_alive : h[1];  // stopped: the k-core is empty (the state is partial)
  } else {
    k_frontier_init<<<grid_for(n_alive, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        alive.as<uint32_t>(), n_alive, deg.as<uint32_t>(), rem.as<uint32_t>(), k, tag, front[0].as<uint32_t>(),
        cn + 0, n, err);
    KT_LAUNCHED(c);
    int cur_f = 0;
    while (true) {
      const uint64_t nf = read_word<unsigned long long>(c, cn + cur_f);
      if (nf == 0) break;
      removed += nf;
      if (may_stop && n_alive - removed < (uint64_t)k + 1) {
        removed = n_alive;  // the k-core is empty (the state is partial)
        break;
      }
      ++rounds;
      KT_CUDA(cudaMemsetAsync(cn + (cur_f ^ 1), 0, sizeof(unsigned long long), c->stream));
      KT_CUDA(cudaMemsetAsync(cn + 4, 0, sizeof(unsigned long long), c->stream));
      k_expand<<<grid_for(nf * 32, 256, c->num_sms * 16), 256, 0, c->stream>>>(
          front[cur_f].as<uint32_t>(), nf, g.off.as<uint64_t>(), g.adj.as<uint32_t>(), deg.as<uint32_t>(),
          rem.as<uint32_t>(), k, tag, front[cur_f ^ 1].as<uint32_t>(), cn + (cur_f ^ 1), big.as<uint32_t>(),
          cn + 4, n, err, big_row(c));
      KT_LAUNCHED(c);
      k_expand_big<<<c->num_sms * 4, 256, 0, c->stream>>>(big.as<uint32_t>(), cn + 4, g.off.as<uint64_t>(),
                                                          g.adj.as<uint32_t>(), deg.as<uint32_t>(),
                                                          rem.as<uint32_t>(), k, tag, front[cur_f ^ 1].as<uint32_t>(),
                                                          cn + (cur_f ^ 1), n, err);
      KT_LAUNCHED(c);
      cur_f ^= 1;
    }
  }
  ++probes;
  check_words(c, "k-core probe");
  return n_alive - removed;
}

uint32_t KCore::find_max_core(Ctx* c) {
  if (!n_alive) {
    cmax = 0;
    return 0;
  }
  // Upper bound: a k-core holds >= k(k+1)/2 edges.
  const double m = (double)base->m;
  uint64_t ub = (uint64_t)std::floor((std::sqrt(1.0 + 8.0 * m) - 1.0) / 2.0);
  ub = std::min<uint64_t>(ub, base->max_deg);
  uint64_t lo = 1, hi = ub + 1;  // the 1-core (non-isolated vertices) is non-empty
  bool ramp = true;
  DBuf mn(c, 16), snap;
  while (hi - lo > 1) {
    uint64_t k = ramp ? std::min<uint64_t>(lo * 2, hi - 1) : lo + (hi - lo) / 2;
    if (k <= lo) k = lo + 1;
    const uint32_t tag = (uint32_t)levels.size();
    const auto t0 = std::chrono::steady_clock::now();
    const uint64_t before = n_alive;
    // Degrees before the probe: a failed probe is undone by reviving its tag
    // and copying them back (the alive set is then the one they belong to).
    snap.ensure(c, n * sizeof(uint32_t));
    KT_CUDA(cudaMemcpyAsync(snap.get(), deg.get(), n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, c->stream));
    const uint64_t left = probe(c, (uint32_t)k, true);
    KT_LOG(c, "kt: k-core probe %llu: %llu of %llu alive vertices left, %.3f ms\n", (unsigned long long)k,
           (unsigned long long)left, (unsigned long long)before,
           std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    if (left) {
      lo = k;
      succ.push_back(tag);
      rebuild_alive(c);
      // The probe left the k-core; its minimum degree d >= k makes it the
      // d-core too, so every level up to d is known to be non-empty.
      // mn: [0] the minimum alive degree, [2..3] the sum of alive degrees.
      KT_CUDA(cudaMemsetAsync(mn.get(), 0xff, 4, c->stream));
      KT_CUDA(cudaMemsetAsync(mn.as<uint32_t>() + 2, 0, 8, c->stream));
      k_min_alive_deg<<<grid_for(n_alive, 256, c->num_sms * 8), 256, 0, c->stream>>>(
          alive.as<uint32_t>(), n_alive, deg.as<uint32_t>(), rem.as<uint32_t>(), mn.as<uint32_t>(),
          reinterpret_cast<unsigned long long*>(mn.as<uint32_t>() + 2));
      KT_LAUNCHED(c);
      uint32_t h[4];
      copy_d2h(c, h, mn.get(), sizeof(h));
      const uint32_t d = h[0];
      uint64_t deg_sum = 0;
      std::memcpy(&deg_sum, h + 2, 8);
      if (d != 0xffffffffu && d > lo) lo = std::min<uint64_t>(d, hi - 1);
      // Work on a compacted copy once the core's edges are a small part of
      // the current graph's: a copy that keeps most of them costs more than
      // the probes it would speed up.  (The copy holds the k-core, which
      // every level from k up can be restored from.)
      if (c->opt.kcore_compact > 0 && (deg_sum / 2) * (uint64_t)c->opt.kcore_compact < cur().m) {
        const auto tc = std::chrono::steady_clock::now();
        const uint64_t from = n;
        compact_to_alive(c, (uint32_t)k);
        KT_LOG(c, "kt: k-core compacted copy of the %llu-core: %llu of %llu vertices, %llu edges, %.3f ms\n",
               (unsigned long long)k, (unsigned long long)n, (unsigned long long)from,
               (unsigned long long)local.m,
               std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tc).count());
      }
    } else {
      hi = k;
      ramp = false;
      // Undo: revive this probe's vertices and restore their degrees.
      k_revive<<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(rem.as<uint32_t>(), n, tag - 1);
      KT_LAUNCHED(c);
      levels.pop_back();
      KT_CUDA(cudaMemcpyAsync(deg.get(), snap.get(), n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, c->stream));
    }
  }
  cmax = (uint32_t)lo;
  return cmax;
}

void KCore::restore_core(Ctx* c, uint32_t k) {
  if (compacted && k < local_level) {
    // Below the compacted core: start over from the deepest earlier
    // compaction at or below level k, else from the input graph.
    while (!saved.empty() && saved.back().level > k) saved.pop_back();
    if (!saved.empty()) {
      local = std::move(saved.back().local);
      idmap = std::move(saved.back().idmap);
      local_level = saved.back().level;
      saved.pop_back();
      levels.assign(1, local_level);
      succ.assign(1, 0);
      reset_state(c, local);
    } else {
      compacted = false;
      local = Graph();
      idmap.release();
      levels.assign(1, 1);
      succ.assign(1, 0);
      reset_state(c, *base);
    }
  }
  // Last successful probe at or below level k; everything newer is revived.
  uint32_t keep = 0;
  for (uint32_t t : succ)
    if (levels[t] <= k) keep = std::max(keep, t);
  k_revive<<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(rem.as<uint32_t>(), n, keep);
  KT_LAUNCHED(c);
  levels.resize(keep + 1);
  std::vector<uint32_t> s2;
  for (uint32_t t : succ)
    if (t <= keep) s2.push_back(t);
  succ.swap(s2);
  rebuild_alive(c);
  recount(c);
  const uint32_t tag = (uint32_t)levels.size();
  if (probe(c, k)) succ.push_back(tag);
  rebuild_alive(c);
}

void KCore::members(Ctx* c, uint8_t* dout) {
  if (!base->n) return;
  if (compacted) {
    zero(c, dout, base->n);
    if (n) {
      k_members_mapped<<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(rem.as<uint32_t>(), n,
                                                                                   idmap.as<uint32_t>(), dout);
      KT_LAUNCHED(c);
    }
    return;
  }
  k_members<<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(rem.as<uint32_t>(), n, dout);
  KT_LAUNCHED(c);
}

void KCore::core_numbers(Ctx* c, uint32_t* dcore) {
  if (compacted) throw Error(KT_ERR_INVALID, "core_numbers needs an uncompacted state");
  if (c->opt.persistent) {
    core_numbers_persistent(c, dcore);
    return;
  }
  // Peel level by level: the alive set is always a d-core where d is its
  // minimum degree, so the probe at d+1 removes exactly the core-d vertices.
  DBuf mn(c, 4);
  while (n_alive) {
    KT_CUDA(cudaMemsetAsync(mn.get(), 0xff, 4, c->stream));
    k_min_alive_deg<<<grid_for(n_alive, 256, c->num_sms * 8), 256, 0, c->stream>>>(
        alive.as<uint32_t>(), n_alive, deg.as<uint32_t>(), rem.as<uint32_t>(), mn.as<uint32_t>());
    KT_LAUNCHED(c);
    const uint32_t d = read_word<uint32_t>(c, mn.as<uint32_t>());
    probe(c, d + 1);
    rebuild_alive(c);
  }
  DBuf lv(c, levels.size() * sizeof(uint32_t));
  copy_h2d(c, lv.get(), levels.data(), levels.size() * sizeof(uint32_t));
  if (n) {
    k_core_from_tags<<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(rem.as<uint32_t>(), n,
                                                                                 lv.as<uint32_t>(), dcore);
    KT_LAUNCHED(c);
  }
  sync(c);
}

}  // namespace kt

namespace kt {

void KCore::core_numbers_persistent(Ctx* c, uint32_t* dcore) {
  if (!n) return;
  zero(c, dcore, n * sizeof(uint32_t));  // isolated vertices: core 0
  if (!n_alive) return;
  const Graph& g = cur();
  DBuf list2(c, n * sizeof(uint32_t)), cand0(c, n * sizeof(uint32_t)), cand1(c, n * sizeof(uint32_t));
  DBuf cn(c, 24 * sizeof(unsigned long long));
  zero(c, cn.get(), cn.bytes());
  KT_CUDA(cudaMemsetAsync(cn.as<unsigned long long>() + 8, 0xff, 3 * sizeof(unsigned long long), c->stream));
  DecompArgs A;
  A.off = g.off.as<uint64_t>();
  A.adj = g.adj.as<uint32_t>();
  A.deg = deg.as<uint32_t>();
  A.rem = rem.as<uint32_t>();
  A.core = dcore;
  A.list[0] = alive.as<uint32_t>();
  A.list[1] = list2.as<uint32_t>();
  A.cand[0] = cand0.as<uint32_t>();
  A.cand[1] = cand1.as<uint32_t>();
  A.front[0] = front[0].as<uint32_t>();
  A.front[1] = front[1].as<uint32_t>();
  A.big = big.as<uint32_t>();
  A.cnt = cn.as<unsigned long long>();
  A.n_list = n_alive;
  A.cap = n;
  A.big_row = big_row(c);
  A.window = (uint32_t)std::min<int64_t>(std::max<int64_t>(1, c->opt.kcore_window), 1 << 20);
  A.words = dev_words(c);
  A.timeout_ns = (unsigned long long)c->opt.timeout_ms * 1000000ULL;
  int per_sm = 0;
  KT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_core_levels, 256, 0));
  if (c->opt.kcore_blocks_per_sm > 0) per_sm = (int)std::min<int64_t>(per_sm, c->opt.kcore_blocks_per_sm);
  const unsigned grid = coop_blocks(c, per_sm);
  void* p[] = {&A};
  uint64_t h[5];
  {
    CoopLock coop(c);
    KT_CUDA(cudaLaunchCooperativeKernel((const void*)k_core_levels, dim3(grid), dim3(256), p, 0, c->stream));
    KT_LAUNCHED(c);
    copy_d2h(c, h, cn.as<unsigned long long>() + 14, sizeof(h));
  }
  rounds += h[0];
  probes += h[1];
  check_words(c, "core decomposition");
  KT_LOG(c, "kt: core decomposition of %llu vertices: %llu levels, %llu rounds, %llu passes (%llu full), max core %llu\n",
         (unsigned long long)n_alive, (unsigned long long)h[1], (unsigned long long)h[0], (unsigned long long)h[2],
         (unsigned long long)h[3], (unsigned long long)(h[4] ? h[4] - 1 : 0));
  n_alive = 0;  // the state is consumed
}

}  // namespace kt
