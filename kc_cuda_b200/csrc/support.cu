// Stage (d): support (triangles through each edge) of the working graph.
//
// Vertex-centric, no atomics on the counts: a block owns a vertex v at a
// time, marks N(v) in a shared-memory bitmap over the subgraph's vertex ids,
// and for every lower neighbour u (new id < v, so deg(u) <= deg(v)) a warp
// scans N(u) against the bitmap; the popcount is |N(u) n N(v)|, written to
// the edge (u, v).  Each edge is counted once, from its higher-degree end,
// scanning the shorter list.  Blocks are persistent and take vertices from
// the highest degree down through an atomic cursor.
//
// The reference counts triangles on the degree-oriented graph with a
// warp-per-vertex merge and scatters 2 per triangle to all three edges with
// atomics (tricount_direct, src/kc.cu:505-651); its support is twice this.
//
// Graphs whose vertex count exceeds the bitmap limit use k_support_search:
// warp per edge, lanes binary-search the shorter row in the longer one.
#include <algorithm>

#include <vector>

#include "dense.cuh"
#include "subgraph.h"

namespace kt {
namespace {

constexpr unsigned kSupThreads = 256;
constexpr unsigned kSupThreadsWide = 1024;  // bitmap kernel when its bitmap limits blocks per SM

// Batched unions: the bitmap covers only v's own graph, bits indexed from
// vbase[v] (graphs are contiguous and no edge crosses graphs); `range` =
// most vertices of one graph.
__global__ void __launch_bounds__(kSupThreadsWide) k_support_bitmap(uint32_t n, const uint64_t* __restrict__ off,
                                                                const uint32_t* __restrict__ adj,
                                                                const uint32_t* __restrict__ eid,
                                                                const uint64_t* __restrict__ up,
                                                                uint32_t* __restrict__ sup,
                                                                unsigned long long* cursor,
                                                                const uint32_t* __restrict__ vbase, uint32_t range) {
  extern __shared__ uint32_t bits[];
  __shared__ uint32_t s_v;
  const uint32_t words = (range + 31) / 32;
  for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) bits[i] = 0;
  __syncthreads();
  while (true) {
    if (threadIdx.x == 0) {
      const unsigned long long t = atomicAdd(cursor, 1ULL);
      s_v = t < n ? (uint32_t)(n - 1 - t) : 0xffffffffu;
    }
    __syncthreads();
    const uint32_t v = s_v;
    if (v == 0xffffffffu) break;
    const uint32_t base = vbase ? vbase[v] : 0u;
    const uint64_t vb = off[v], ve = off[v + 1], vu = up[v];
    for (uint64_t j = vb + threadIdx.x; j < ve; j += blockDim.x) {
      const uint32_t w = adj[j] - base;
      atomicOr(&bits[w >> 5], 1u << (w & 31));
    }
    __syncthreads();
    // Lower neighbours u of v: entries [vb, vu).
    for (uint64_t j = vb + warp_id(); j < vu; j += blockDim.x >> 5) {
      const uint32_t u = adj[j];
      const uint64_t ub = off[u], ue = off[u + 1];
      uint32_t cnt = 0;
      for (uint64_t q = ub + lane_id(); q < ue; q += 32) {
        const uint32_t w = adj[q] - base;
        cnt += (bits[w >> 5] >> (w & 31)) & 1u;
      }
      cnt = warp_sum(cnt);
      if (lane_id() == 0) sup[eid[j]] = cnt;
    }
    __syncthreads();
    for (uint64_t j = vb + threadIdx.x; j < ve; j += blockDim.x) {
      const uint32_t w = adj[j] - base;
      bits[w >> 5] = 0;
    }
    __syncthreads();
  }
}

// Position of x in sorted a[lo, hi), or hi.
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

__global__ void k_support_search(uint64_t m, const uint64_t* __restrict__ ends, const uint64_t* __restrict__ off,
                                 const uint32_t* __restrict__ adj, uint32_t* __restrict__ sup) {
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t e = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); e < m; e += warps) {
    const uint64_t k = ends[e];
    uint32_t a = (uint32_t)(k >> 32), b = (uint32_t)k;
    if (off[a + 1] - off[a] > off[b + 1] - off[b]) {
      const uint32_t t = a;
      a = b;
      b = t;
    }
    const uint64_t ab = off[a], ae = off[a + 1], bb = off[b], be = off[b + 1];
    uint32_t cnt = 0;
    for (uint64_t q = ab + lane_id(); q < ae; q += 32) cnt += find_sorted(adj, bb, be, adj[q]) != be;
    cnt = warp_sum(cnt);
    if (lane_id() == 0) sup[e] = cnt;
  }
}

// Dense mode: row bitsets from the sorted rows.
__global__ void k_bits_build(uint32_t n, const uint64_t* __restrict__ off, const uint32_t* __restrict__ adj,
                             DenseRows R) {
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t u = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); u < n; u += warps) {
    uint32_t* row = R.bits + R.off((uint32_t)u);
    for (uint64_t j = off[u] + lane_id(); j < off[u + 1]; j += 32) {
      const uint32_t v = R.col((uint32_t)u, adj[j]);
      atomicOr(&row[v >> 5], 1u << (v & 31));
    }
  }
}

// spre[w] = set bits of row u before its word w (warp per row).
__global__ void k_row_prefix(uint32_t n, DenseRows R, uint32_t* __restrict__ spre) {
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t u = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); u < n; u += warps) {
    const uint64_t base = R.off((uint32_t)u);
    const uint32_t W = R.words((uint32_t)u);
    uint32_t run = 0;
    for (uint32_t i0 = 0; i0 < W; i0 += 32) {
      const uint32_t i = i0 + lane_id();
      const uint32_t pc = i < W ? __popc(R.bits[base + i]) : 0u;
      const uint32_t inc = warp_incl_scan(pc);
      if (i < W) spre[base + i] = run + inc - pc;
      run += __shfl_sync(kFull, inc, 31);
    }
  }
}

// Per-graph rows of a grouped union: graph g's rows hold gw[g] words and
// start at word gbase[g].
__global__ void k_group_rows(uint32_t n, const uint32_t* __restrict__ vgid, const uint32_t* __restrict__ vbase,
                             const uint64_t* __restrict__ gbase, const uint32_t* __restrict__ gw,
                             uint64_t* __restrict__ roff, uint32_t* __restrict__ rw) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t g = vgid[v];
    roff[v] = gbase[g] + (uint64_t)(v - vbase[v]) * gw[g];
    rw[v] = gw[g];
  }
}

// Warps take 32-edge groups from a cursor, so the groups in flight stay a
// narrow window of the tile-ordered list (a grid-stride loop lets warps drift
// apart, and the rows they read then no longer fit in L2).  `row_words`
// accumulates the row words read.
//
// Exact counts, up to NQ edges sharing row u per shared-memory read of it;
// four resident blocks per SM (what the rows' shared memory allows for the
// bench graph's cores) bound the registers to 64.
template <int NQ>
__global__ void __launch_bounds__(256, 4) k_dense_support(uint64_t m, const uint32_t* __restrict__ order,
                                                          const uint64_t* __restrict__ ends, DenseRows R,
                                                          uint32_t* __restrict__ sup,
                                                          unsigned long long* __restrict__ row_words,
                                                          unsigned long long* __restrict__ cursor) {
  extern __shared__ __align__(16) uint32_t dense_smem[];
  uint32_t* su = dense_smem + warp_id() * R.W;
  const uint64_t groups = (m + 31) / 32;
  unsigned long long wr = 0;  // row words this lane accounts for (lane 0)
  for (;;) {
    unsigned long long g = 0;
    if (lane_id() == 0) g = atomicAdd(cursor, 1ULL);
    g = __shfl_sync(kFull, g, 0);
    if (g >= groups) break;
    uint32_t e, s;
    bool ok;
    dense_group<NQ>(order, g * 32, m, ends, R, nullptr, su, e, s, ok, &wr);
    if (ok) sup[e] = s;
  }
  wr = warp_sum(wr);
  if (lane_id() == 0 && wr) atomicAdd(row_words, wr);
}

// Capped counts (search phase): threshold `cap`, or gcap[vgid[u]] per graph
// of a grouped union.
__global__ void __launch_bounds__(256) k_dense_support_capped(uint64_t m, const uint32_t* __restrict__ order,
                                                              const uint64_t* __restrict__ ends, DenseRows R,
                                                              uint32_t cap, const uint32_t* __restrict__ gcap,
                                                              const uint32_t* __restrict__ vgid,
                                                              uint32_t* __restrict__ sup,
                                                              unsigned long long* __restrict__ row_words,
                                                              unsigned long long* __restrict__ cursor) {
  extern __shared__ __align__(16) uint32_t dense_smem[];
  uint32_t* su = dense_smem + warp_id() * R.W;
  const uint64_t groups = (m + 31) / 32;
  unsigned long long wr = 0;  // row words this lane accounts for (lanes 0 and 16)
  for (;;) {
    unsigned long long g = 0;
    if (lane_id() == 0) g = atomicAdd(cursor, 1ULL);
    g = __shfl_sync(kFull, g, 0);
    if (g >= groups) break;
    uint32_t e, s;
    bool ok;
    dense_group_capped(order, g * 32, m, ends, R, cap, su, e, s, ok, &wr, gcap, vgid);
    if (ok) sup[e] = s;
  }
  wr = warp_sum(wr);
  if (lane_id() == 0 && wr) atomicAdd(row_words, wr);
}

// Tile keys: (u >> tb) << 16 | (v >> tb), stable-sorted with the edge ids.
__global__ void k_tile_keys(uint64_t m, const uint64_t* __restrict__ ends, uint32_t tb, uint64_t* __restrict__ keys,
                            uint32_t* __restrict__ ids) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = ends[e];
    keys[e] = ((k >> (32 + tb)) << 16) | (((uint32_t)k) >> tb);
    ids[e] = (uint32_t)e;
  }
}

// Grid of the resident blocks of `kernel` with the rows' shared memory.
unsigned dense_grid(Ctx* c, const void* kernel, const Sub& s, size_t smem) {
  allow_max_dynamic_smem(kernel);
  int per_sm = 0;
  KT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, smem));
  return grid_for((s.m + 31) / 32 * 32, 256, std::max(1, per_sm) * c->num_sms);
}

template <int NQ>
void launch_exact(Ctx* c, const Sub& s, uint32_t* sup, unsigned long long* row_words, unsigned long long* cursor) {
  const size_t smem = dense_smem_bytes(s.W, 256);
  const unsigned grid = dense_grid(c, (const void*)k_dense_support<NQ>, s, smem);
  k_dense_support<NQ><<<grid, 256, smem, c->stream>>>(s.m, s.order.as<uint32_t>(), s.ends.as<uint64_t>(),
                                                      dense_rows(s), sup, row_words, cursor);
  KT_LAUNCHED(c);
}

// Exact counts: option support_rows (1, 2 or 4) edges sharing row u per
// shared-memory read of it.  Capped counts: two edges sharing row u side by
// side, one per half of the warp.
void launch_dense_support(Ctx* c, const Sub& s, uint32_t* sup, bool capped, uint32_t cap, const uint32_t* gcap,
                          unsigned long long* row_words, unsigned long long* cursor) {
  if (capped) {
    const size_t smem = dense_smem_bytes(s.W, 256);
    const unsigned grid = dense_grid(c, (const void*)k_dense_support_capped, s, smem);
    k_dense_support_capped<<<grid, 256, smem, c->stream>>>(s.m, s.order.as<uint32_t>(), s.ends.as<uint64_t>(),
                                                           dense_rows(s), cap, gcap,
                                                           gcap ? s.vgid.as<uint32_t>() : nullptr, sup, row_words,
                                                           cursor);
    KT_LAUNCHED(c);
  } else if (c->opt.support_rows <= 1) {
    launch_exact<1>(c, s, sup, row_words, cursor);
  } else if (c->opt.support_rows == 2) {
    launch_exact<2>(c, s, sup, row_words, cursor);
  } else {
    launch_exact<4>(c, s, sup, row_words, cursor);
  }
}

// Algorithmic bytes of a merge-based support count over the degree-oriented
// graph: 4 * sum over oriented edges (u -> v) of (d+(u) + d+(v)).
__global__ void k_support_alg(uint64_t m, const uint64_t* __restrict__ ends, const uint64_t* __restrict__ off,
                              const uint64_t* __restrict__ up, unsigned long long* out) {
  uint64_t s = 0;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = ends[e];
    const uint32_t u = (uint32_t)(k >> 32), v = (uint32_t)k;
    s += (off[u + 1] - up[u]) + (off[v + 1] - up[v]);
  }
  s = warp_sum(s);
  if (lane_id() == 0 && s) atomicAdd(out, (unsigned long long)s);
}

// hist[min(sup, cap)] += 1, warp-aggregated over equal bins.
__global__ void k_sup_hist(const uint32_t* __restrict__ sup, uint64_t m, uint32_t cap,
                           unsigned long long* __restrict__ hist) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ((m + 31) & ~31ULL);
       i += (uint64_t)gridDim.x * blockDim.x) {
    const bool ok = i < m;
    const uint32_t b = ok ? min(sup[i], cap) : 0xffffffffu;
    const unsigned peers = __match_any_sync(kFull, b);
    if (ok && lane_id() == (unsigned)(__ffs(peers) - 1)) atomicAdd(&hist[b], (unsigned long long)__popc(peers));
  }
}

}  // namespace

uint32_t support_bound(Ctx* c, const uint32_t* sup, uint64_t m, uint32_t cap) {
  if (m == 0 || cap < 3) return 0;
  DBuf hist(c, ((uint64_t)cap + 1) * 8);
  zero(c, hist.get(), hist.bytes());
  k_sup_hist<<<grid_for(m, 256, c->num_sms * 16), 256, 0, c->stream>>>(sup, m, cap,
                                                                       hist.as<unsigned long long>());
  KT_LAUNCHED(c);
  std::vector<unsigned long long> h(cap + 1);
  copy_d2h(c, h.data(), hist.get(), h.size() * sizeof(unsigned long long));
  // at_least = edges with support >= t-2, accumulated while t descends.
  unsigned long long at_least = h[cap] + h[cap - 1];
  for (uint32_t t = cap; t >= 3; --t) {
    at_least += h[t - 2];
    if (at_least >= (unsigned long long)t * (t - 1) / 2) return t;
  }
  return 0;
}

bool build_bits(Ctx* c, Sub& s) {
  s.W = 0;
  s.bits.release();
  s.sbits.release();
  s.spre.release();
  s.roff.release();
  s.rw.release();
  s.bit_words = 0;
  if (s.n == 0 || s.m == 0) return false;
  // Rows: one block of bitsets per graph for a grouped union (every graph
  // within the vertex limit), else one block for the whole graph.
  const bool grouped = s.vgid.get() != nullptr && !s.group_n.empty();
  uint32_t W = 0;
  uint64_t words = 0;
  std::vector<uint64_t> gbase;
  std::vector<uint32_t> gw;
  if (grouped) {
    if ((int64_t)s.max_group > c->opt.dense_max_n) return false;
    gbase.resize(s.group_n.size());
    gw.resize(s.group_n.size());
    for (size_t g = 0; g < s.group_n.size(); ++g) {
      gbase[g] = words;
      gw[g] = ((s.group_n[g] + 31) / 32 + 3) & ~3u;  // rows of whole 16-byte vectors
      words += (uint64_t)s.group_n[g] * gw[g];
      W = std::max(W, gw[g]);
    }
  } else {
    if ((int64_t)s.n > c->opt.dense_max_n) return false;
    W = ((s.n + 31) / 32 + 3) & ~3u;  // rows of whole 16-byte vectors
    words = (uint64_t)s.n * W;
  }
  // Dense enough: adjacency entries * fill >= words of all rows.
  if (2.0 * (double)s.m * (double)c->opt.dense_min_fill < (double)words) return false;
  const uint64_t bytes = words * 4;
  if (c->budget && c->in_use + 2 * bytes > c->budget) return false;
  s.bits.alloc(c, bytes);
  zero(c, s.bits.get(), bytes);
  if (grouped) {
    const uint32_t G = (uint32_t)gw.size();
    DBuf dgb(c, G * 8ull), dgw(c, G * 4ull);
    copy_h2d(c, dgb.get(), gbase.data(), G * 8ull);
    copy_h2d(c, dgw.get(), gw.data(), G * 4ull);
    s.roff.alloc(c, (uint64_t)s.n * 8);
    s.rw.alloc(c, (uint64_t)s.n * 4);
    k_group_rows<<<grid_for(s.n, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        s.n, s.vgid.as<uint32_t>(), s.vbase.as<uint32_t>(), dgb.as<uint64_t>(), dgw.as<uint32_t>(),
        s.roff.as<uint64_t>(), s.rw.as<uint32_t>());
    KT_LAUNCHED(c);
  }
  s.W = W;
  s.bit_words = words;
  k_bits_build<<<grid_for((uint64_t)s.n * 32, 256, c->num_sms * 16), 256, 0, c->stream>>>(
      s.n, s.off.as<uint64_t>(), s.adj.as<uint32_t>(), dense_rows(s));
  KT_LAUNCHED(c);
  // The rows as built and their per-word prefix counts (positions of
  // neighbours for the peel), when two more copies fit the budget.
  s.sbits.release();
  s.spre.release();
  if (!c->budget || c->in_use + 3 * bytes <= c->budget) {
    s.sbits.alloc(c, bytes);
    s.spre.alloc(c, bytes);
    KT_CUDA(cudaMemcpyAsync(s.sbits.get(), s.bits.get(), bytes, cudaMemcpyDeviceToDevice, c->stream));
    k_row_prefix<<<grid_for((uint64_t)s.n * 32, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        s.n, dense_rows(s), s.spre.as<uint32_t>());
    KT_LAUNCHED(c);
  }
  // Tile order: blocks of 2^tb vertices, two blocks' bitsets within ~48 MB.
  uint32_t tb = 16;
  const uint64_t tile_bytes = (uint64_t)std::max<int64_t>(1, c->opt.dense_tile_mb) << 20;
  while (tb > 6 && 2ull * (1ull << tb) * W * 4 > tile_bytes) --tb;
  s.tile_bits = tb;
  s.order.alloc(c, s.m * sizeof(uint32_t));
  DBuf keys(c, s.m * sizeof(uint64_t));
  k_tile_keys<<<grid_for(s.m, 256, c->num_sms * 16), 256, 0, c->stream>>>(s.m, s.ends.as<uint64_t>(), tb,
                                                                            keys.as<uint64_t>(),
                                                                            s.order.as<uint32_t>());
  KT_LAUNCHED(c);
  radix_sort_u64(c, keys.as<uint64_t>(), s.order.as<uint32_t>(), s.m, 32);
  return true;
}

void edge_support(Ctx* c, const Sub& s, uint32_t* sup, uint32_t cap, const uint32_t* gcap) {
  if (s.m == 0) return;
  // acc[0]: merge-model list entries, acc[1]: dense row words read, acc[2]:
  // the dense kernel's group cursor.
  DBuf acc(c, 24);
  zero(c, acc.get(), 24);
  cudaEvent_t e0;
  if (c->opt.verbose) KT_CUDA(cudaEventRecord(c->ev[2], c->stream));
  c->timer.begin(c->stream, &c->stats.ms_support_kernel, &e0);
  if (s.W) {
    unsigned long long* a = acc.as<unsigned long long>();
    const bool capped = cap || (gcap && s.vgid.get());
    launch_dense_support(c, s, sup, capped, cap, s.vgid.get() ? gcap : nullptr, a + 1, a + 2);
  } else if ((int64_t)(s.vbase.get() ? s.max_group : s.n) <= c->opt.support_bitmap_max_n) {
    const uint32_t range = s.vbase.get() ? s.max_group : s.n;
    const size_t smem = ((range + 31) / 32) * sizeof(uint32_t);
    if (smem > 48 * 1024)
      allow_max_dynamic_smem((const void*)k_support_bitmap);
    // Large bitmaps leave room for few blocks per SM: then wider blocks.
    const unsigned threads = smem > 24 * 1024 ? kSupThreadsWide : kSupThreads;
    int per_sm = 0;
    KT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_support_bitmap, threads, smem));
    if (per_sm < 1) throw Error(KT_ERR_LIMIT, "support: bitmap does not fit in shared memory");
    DBuf cur(c, 8);
    zero(c, cur.get(), 8);
    const unsigned grid = (unsigned)std::min<uint64_t>((uint64_t)per_sm * c->num_sms, s.n);
    k_support_bitmap<<<grid, threads, smem, c->stream>>>(s.n, s.off.as<uint64_t>(), s.adj.as<uint32_t>(),
                                                             s.eid.as<uint32_t>(), s.up.as<uint64_t>(), sup,
                                                             cur.as<unsigned long long>(),
                                                             s.vbase.get() ? s.vbase.as<uint32_t>() : nullptr,
                                                             range);
    KT_LAUNCHED(c);
  } else {
    k_support_search<<<grid_for(s.m * 32, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        s.m, s.ends.as<uint64_t>(), s.off.as<uint64_t>(), s.adj.as<uint32_t>(), sup);
    KT_LAUNCHED(c);
  }
  c->timer.end(c->stream, e0, &c->stats.ms_support_kernel);
  if (c->opt.verbose) KT_CUDA(cudaEventRecord(c->ev[3], c->stream));
  c->stats.support_launches++;
  // Algorithmic bytes (outside the timed span): the merge model, and the
  // bytes the kernel that ran moved.
  k_support_alg<<<grid_for(s.m, 256, c->num_sms * 8), 256, 0, c->stream>>>(s.m, s.ends.as<uint64_t>(),
                                                                             s.off.as<uint64_t>(),
                                                                             s.up.as<uint64_t>(),
                                                                             acc.as<unsigned long long>());
  KT_LAUNCHED(c);
  uint64_t h[2];
  copy_d2h(c, h, acc.get(), 16);
  const uint64_t merge = 4 * h[0] + 4 * s.m + 8 * ((uint64_t)s.n + 1);
  c->stats.support_bytes += merge;
  c->stats.support_row_words += h[1];
  // Dense: row words, plus per edge its list entry (4), ends (8) and result (4).
  c->stats.support_kernel_bytes += s.W ? 4 * h[1] + 16 * s.m : merge;
  KT_LOG(c, "kt: support (%s) on %u vertices (widest group %u), %llu edges: %llu row words, %.3f ms\n",
         s.W ? (cap || (gcap && s.vgid.get()) ? "dense capped" : "dense") : "list", s.n,
         s.vbase.get() ? s.max_group : s.n, (unsigned long long)s.m, (unsigned long long)h[1],
         c->opt.verbose ? event_ms(c->ev[2], c->ev[3]) : 0.0);
}

}  // namespace kt
