// Induced subgraph of the surviving vertices, relabelled by ascending
// (degree, id), with sorted rows, edge ids and (dense mode) row bitsets.
//
// The reference builds the same relabelled, oriented structure on the host
// (construct_Graph and build_nbr_direct, src/kc_gpu.cpp:68-126,
// src/kc.cu:1405-1580, with CPU sorts of the ranks and of every row).  Here:
// sort (degree << 32 | id) keys for the new order; write every surviving
// adjacency entry's new column into its new row, and sort each row -- in a
// shared-memory bitmap of the row's id range when the rows are dense
// enough, else by one radix sort of (new u << 32 | new v) over all entries;
// the upper entries (neighbour > row) number the edges row by row (an
// exclusive scan of the upper-part sizes); the row bitsets of dense mode are
// built; a lower entry (r, c < r) takes the id of (c, r) from the position of
// r in row c -- a popcount of the bitsets, or a binary search.
#include <algorithm>
#include <vector>

#include "compact.cuh"
#include "dense.cuh"
#include "subgraph.h"

namespace kt {
namespace {

__global__ void k_order_keys(const uint32_t* __restrict__ alive, uint64_t na, const uint32_t* __restrict__ deg,
                             const uint32_t* __restrict__ group_of, uint64_t* __restrict__ keys) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = alive[i];
    if (group_of)  // graph (16 bits) | degree (20 bits, saturated) | id (28 bits)
      keys[i] = ((uint64_t)group_of[v] << 48) | ((uint64_t)min(deg[v], 0xfffffu) << 28) | v;
    else
      keys[i] = ((uint64_t)deg[v] << 32) | v;
  }
}

__global__ void k_group_meta(const uint32_t* __restrict__ orig, uint64_t na, const uint32_t* __restrict__ group_of,
                             uint32_t* __restrict__ vgid, uint32_t* __restrict__ gstart,
                             uint32_t* __restrict__ gsize) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t g = group_of[orig[i]];
    vgid[i] = g;
    if (i == 0 || group_of[orig[i - 1]] != g) gstart[g] = (uint32_t)i;
    atomicAdd(&gsize[g], 1u);
  }
}

__global__ void k_group_base(const uint32_t* __restrict__ vgid, uint64_t na, const uint32_t* __restrict__ gstart,
                             uint32_t* __restrict__ vbase) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += (uint64_t)gridDim.x * blockDim.x)
    vbase[i] = gstart[vgid[i]];
}

// Decodes the sorted order keys: orig[i] = the vertex, newid[v] = i, sdeg[i]
// = its degree (read from deg when the key holds a saturated copy).
__global__ void k_order_apply(const uint64_t* __restrict__ keys, uint64_t na, uint32_t* __restrict__ orig,
                              uint32_t* __restrict__ newid, uint32_t* __restrict__ sdeg,
                              const uint32_t* __restrict__ deg, bool grouped) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    const uint32_t v = grouped ? (uint32_t)(k & 0xfffffffULL) : (uint32_t)k;
    orig[i] = v;  // ids of the graph being read; mapped below if it is a compacted copy
    newid[v] = (uint32_t)i;
    sdeg[i] = grouped ? deg[v] : (uint32_t)(k >> 32);
  }
}

// Emits (r << 32 | newid[w]) for every alive neighbour w of orig[r], at
// off[r] + rank.  Warp per row.
__global__ void k_emit(const uint32_t* __restrict__ orig, uint64_t na, const uint64_t* __restrict__ goff,
                       const uint32_t* __restrict__ gadj, const uint32_t* __restrict__ rem,
                       const uint32_t* __restrict__ newid, const uint64_t* __restrict__ soff,
                       uint64_t* __restrict__ keys) {
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t r = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); r < na; r += warps) {
    const uint32_t v = orig[r];
    const uint64_t b = goff[v], e = goff[v + 1];
    uint64_t pos = soff[r];
    const uint64_t row_end = soff[r + 1];  // a degree mismatch must not spill into the next row
    for (uint64_t j = b + lane_id(); j < b + ((e - b + 31) & ~31ULL); j += 32) {
      bool keep = false;
      uint32_t w = 0;
      if (j < e) {
        w = gadj[j];
        keep = rem == nullptr || rem[w] == kAlive;
      }
      const unsigned bal = __ballot_sync(kFull, keep);
      const uint64_t p = pos + __popc(bal & lanemask_lt());
      if (keep && p < row_end) keys[p] = ((uint64_t)r << 32) | newid[w];
      pos += __popc(bal);
    }
  }
}

// As k_emit, but the entries are the new column ids alone, written into the
// rows of adj (unsorted within a row).
__global__ void k_emit_cols(const uint32_t* __restrict__ orig, uint64_t na, const uint64_t* __restrict__ goff,
                            const uint32_t* __restrict__ gadj, const uint32_t* __restrict__ rem,
                            const uint32_t* __restrict__ newid, const uint64_t* __restrict__ soff,
                            uint32_t* __restrict__ adj) {
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t r = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); r < na; r += warps) {
    const uint32_t v = orig[r];
    const uint64_t b = goff[v], e = goff[v + 1];
    uint64_t pos = soff[r];
    const uint64_t row_end = soff[r + 1];  // a degree mismatch must not spill into the next row
    for (uint64_t j = b + lane_id(); j < b + ((e - b + 31) & ~31ULL); j += 32) {
      bool keep = false;
      uint32_t w = 0;
      if (j < e) {
        w = gadj[j];
        keep = rem == nullptr || rem[w] == kAlive;
      }
      const unsigned bal = __ballot_sync(kFull, keep);
      const uint64_t p = pos + __popc(bal & lanemask_lt());
      if (keep && p < row_end) adj[p] = newid[w];
      pos += __popc(bal);
    }
  }
}

// Sorts every row of adj in place when its columns are distinct and lie in
// [base, base + range) (base = vbase[r] for a grouped union, else 0; range =
// the row's graph's size, or `range` for all rows): block per row, columns
// marked in a shared-memory bitmap, then written back in ascending order
// (each thread a run of bitmap words, placed by a block scan of their
// popcounts) -- a counting sort of distinct keys.
__global__ void __launch_bounds__(256) k_rows_bitmap_sort(uint64_t na, const uint64_t* __restrict__ off,
                                                          uint32_t* __restrict__ adj,
                                                          const uint32_t* __restrict__ vbase,
                                                          const uint32_t* __restrict__ vgid,
                                                          const uint32_t* __restrict__ gsize, uint32_t range) {
  extern __shared__ uint32_t bm[];
  __shared__ uint32_t tmp[33];
  for (uint64_t r = blockIdx.x; r < na; r += gridDim.x) {
    const uint32_t base = vbase ? vbase[r] : 0u;
    const uint32_t rng = vgid ? gsize[vgid[r]] : range;
    const uint32_t words = (rng + 31) / 32;
    const uint64_t b = off[r], e = off[r + 1];
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) bm[i] = 0;
    __syncthreads();
    for (uint64_t j = b + threadIdx.x; j < e; j += blockDim.x) {
      const uint32_t col = adj[j] - base;
      if (col < rng) atomicOr(&bm[col >> 5], 1u << (col & 31));
    }
    __syncthreads();
    const uint32_t per = (words + blockDim.x - 1) / blockDim.x;
    const uint32_t w0 = min(words, threadIdx.x * per), w1 = min(words, w0 + per);
    uint32_t cnt = 0;
    for (uint32_t w = w0; w < w1; ++w) cnt += __popc(bm[w]);
    uint32_t total;
    uint64_t pos = b + block_excl_scan<uint32_t>(cnt, tmp, &total);
    for (uint32_t w = w0; w < w1; ++w) {
      uint32_t bits = bm[w];
      while (bits) {
        const uint32_t k = __ffs(bits) - 1;
        bits &= bits - 1;
        if (pos < e) adj[pos] = base + w * 32 + k;
        ++pos;
      }
    }
    __syncthreads();
  }
}

__global__ void k_rows_from_keys(const uint64_t* __restrict__ keys, uint64_t n2, uint32_t* __restrict__ adj) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += (uint64_t)gridDim.x * blockDim.x)
    adj[i] = (uint32_t)keys[i];
}

// up[r] = first position in row r holding a neighbour > r.
__global__ void k_upper_start(const uint64_t* __restrict__ off, const uint32_t* __restrict__ adj, uint64_t n,
                              uint64_t* __restrict__ up, uint32_t* __restrict__ upcnt) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t lo = off[r], hi = off[r + 1];
    const uint64_t end = hi;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (adj[mid] <= (uint32_t)r)
        lo = mid + 1;
      else
        hi = mid;
    }
    up[r] = lo;
    upcnt[r] = (uint32_t)(end - lo);
  }
}

// Edge ids of the upper entries (neighbour > row): they number themselves in
// row order, and give each edge its ends.  Warp per row.
__global__ void k_upper_ids(const uint64_t* __restrict__ off, const uint32_t* __restrict__ adj, uint64_t n,
                            const uint64_t* __restrict__ up, const uint64_t* __restrict__ eoff,
                            uint32_t* __restrict__ eid, uint64_t* __restrict__ ends) {
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t r = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); r < n; r += warps) {
    const uint64_t e = off[r + 1], u0 = up[r];
    for (uint64_t j = u0 + lane_id(); j < e; j += 32) {
      const uint64_t id = eoff[r] + (j - u0);
      eid[j] = (uint32_t)id;
      ends[id] = (r << 32) | adj[j];
    }
  }
}

// Edge ids of the lower entries: entry (r, c < r) takes the id of the upper
// entry (c, r), found by binary search in row c's upper part, or -- when the
// rows' bitsets are built (R.spre) -- by the position of r in row c, a
// popcount away.  Warp per row.
__global__ void k_lower_ids(const uint64_t* __restrict__ off, const uint32_t* __restrict__ adj, uint64_t n,
                            const uint64_t* __restrict__ up, const uint64_t* __restrict__ eoff, DenseRows R,
                            uint32_t* __restrict__ eid) {
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t r = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); r < n; r += warps) {
    const uint64_t b = off[r], u0 = up[r];
    for (uint64_t j = b + lane_id(); j < u0; j += 32) {
      const uint32_t col = adj[j];
      uint64_t pos;  // position of r in row col
      if (R.spre) {
        pos = off[col] + R.rank(col, R.col(col, (uint32_t)r));
      } else {
        uint64_t lo = up[col], hi = off[col + 1];
        while (lo < hi) {
          const uint64_t mid = (lo + hi) >> 1;
          if (adj[mid] < (uint32_t)r)
            lo = mid + 1;
          else
            hi = mid;
        }
        pos = lo;
      }
      eid[j] = (uint32_t)(eoff[col] + (pos - up[col]));
    }
  }
}

struct DegPositive {
  const uint32_t* deg;
  __device__ bool keep(uint64_t v) const { return deg[v] > 0; }
  __device__ uint32_t value(uint64_t v) const { return (uint32_t)v; }
};

__global__ void k_map_ids(uint32_t* __restrict__ ids, uint64_t n, const uint32_t* __restrict__ idmap) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    ids[i] = idmap[ids[i]];
}

void build_from_list(Ctx* c, const Graph& g, const uint32_t* alive, uint64_t na, const uint32_t* deg,
                     const uint32_t* rem, const uint32_t* idmap, Sub& s, const uint32_t* group_of = nullptr,
                     uint32_t ngroups = 0) {
  if (na >= 0xffffffffULL) throw Error(KT_ERR_LIMIT, "subgraph: too many vertices");
  s.n = (uint32_t)na;
  s.orig.alloc(c, (na ? na : 1) * sizeof(uint32_t));
  s.off.alloc(c, (na + 1) * sizeof(uint64_t));
  s.up.alloc(c, (na ? na : 1) * sizeof(uint64_t));
  if (na == 0) {
    zero(c, s.off.get(), sizeof(uint64_t));
    s.m = 0;
    s.adj.alloc(c, 4);
    s.eid.alloc(c, 4);
    s.ends.alloc(c, 8);
    return;
  }
  // New order.
  DBuf okeys(c, na * sizeof(uint64_t));
  k_order_keys<<<grid_for(na, 256, c->num_sms * 16), 256, 0, c->stream>>>(alive, na, deg, group_of,
                                                                             okeys.as<uint64_t>());
  KT_LAUNCHED(c);
  radix_sort_u64(c, okeys.as<uint64_t>(), nullptr, na, 64);
  DBuf newid(c, (g.n ? g.n : 1) * sizeof(uint32_t));
  DBuf sdeg(c, (na + 1) * sizeof(uint32_t));
  zero(c, sdeg.get(), (na + 1) * sizeof(uint32_t));
  k_order_apply<<<grid_for(na, 256, c->num_sms * 16), 256, 0, c->stream>>>(
      okeys.as<uint64_t>(), na, s.orig.as<uint32_t>(), newid.as<uint32_t>(), sdeg.as<uint32_t>(), deg,
      group_of != nullptr);
  KT_LAUNCHED(c);
  okeys.release();
  DBuf gsize;  // vertices of each graph of a grouped union
  if (group_of) {
    // orig holds ids of g here (mapped below); group them.
    s.vgid.alloc(c, na * sizeof(uint32_t));
    s.vbase.alloc(c, na * sizeof(uint32_t));
    DBuf gstart(c, (uint64_t)ngroups * sizeof(uint32_t));
    gsize.alloc(c, (uint64_t)ngroups * sizeof(uint32_t));
    zero(c, gsize.get(), gsize.bytes());
    k_group_meta<<<grid_for(na, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        s.orig.as<uint32_t>(), na, group_of, s.vgid.as<uint32_t>(), gstart.as<uint32_t>(), gsize.as<uint32_t>());
    KT_LAUNCHED(c);
    k_group_base<<<grid_for(na, 256, c->num_sms * 16), 256, 0, c->stream>>>(s.vgid.as<uint32_t>(), na,
                                                                              gstart.as<uint32_t>(),
                                                                              s.vbase.as<uint32_t>());
    KT_LAUNCHED(c);
    std::vector<uint32_t> sizes(ngroups);
    copy_d2h(c, sizes.data(), gsize.get(), ngroups * sizeof(uint32_t));
    s.max_group = 0;
    for (uint32_t x : sizes) s.max_group = std::max(s.max_group, x);
    s.group_n = std::move(sizes);
  }
  scan_u32_to_u64(c, sdeg.as<uint32_t>(), s.off.as<uint64_t>(), na + 1);
  const uint64_t n2 = read_word<uint64_t>(c, s.off.as<uint64_t>() + na);
  if (n2 & 1) throw Error(KT_ERR_CUDA, "subgraph: odd adjacency size (inconsistent degrees)");
  s.m = n2 / 2;
  if (s.m >= 0xffffffffULL) throw Error(KT_ERR_LIMIT, "subgraph: more than 2^32-1 edges");
  // Sorted rows.  A row's columns are distinct ids of its own graph (new ids
  // [vbase, vbase + size) in a grouped union, [0, n') otherwise).  When the
  // rows are dense enough that a bitmap of that range per row costs no more
  // than a few passes over the entries, each row is sorted in shared memory
  // (k_rows_bitmap_sort); otherwise every entry is emitted as
  // (row << 32 | column) and one radix sort orders them all.
  uint64_t bitmap_words = 0;  // bitmap words cleared and scanned over all rows
  uint32_t max_range = 0;
  if (group_of) {
    for (uint32_t x : s.group_n) bitmap_words += (uint64_t)x * ((x + 31) / 32);
    max_range = s.max_group;
  } else {
    bitmap_words = na * ((na + 31) / 32);
    max_range = (uint32_t)na;
  }
  const uint32_t kMaxBitmapRange = 1u << 18;  // 32 KB of shared memory
  const bool bitmap_rows = n2 && max_range <= kMaxBitmapRange && bitmap_words <= 4 * n2;
  s.adj.alloc(c, (n2 ? n2 : 1) * sizeof(uint32_t));
  if (bitmap_rows) {
    k_emit_cols<<<grid_for(na * 32, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        s.orig.as<uint32_t>(), na, g.off.as<uint64_t>(), g.adj.as<uint32_t>(), rem, newid.as<uint32_t>(),
        s.off.as<uint64_t>(), s.adj.as<uint32_t>());
    KT_LAUNCHED(c);
    newid.release();
    const size_t smem = (size_t)((max_range + 31) / 32) * sizeof(uint32_t);
    if (smem > 48 * 1024)
      allow_max_dynamic_smem((const void*)k_rows_bitmap_sort);
    k_rows_bitmap_sort<<<(unsigned)std::min<uint64_t>(na, (uint64_t)c->num_sms * 32), 256, smem, c->stream>>>(
        na, s.off.as<uint64_t>(), s.adj.as<uint32_t>(), group_of ? s.vbase.as<uint32_t>() : nullptr,
        group_of ? s.vgid.as<uint32_t>() : nullptr, group_of ? gsize.as<uint32_t>() : nullptr, (uint32_t)na);
    KT_LAUNCHED(c);
  } else {
    DBuf keys(c, (n2 ? n2 : 1) * sizeof(uint64_t));
    k_emit<<<grid_for(na * 32, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        s.orig.as<uint32_t>(), na, g.off.as<uint64_t>(), g.adj.as<uint32_t>(), rem, newid.as<uint32_t>(),
        s.off.as<uint64_t>(), keys.as<uint64_t>());
    KT_LAUNCHED(c);
    newid.release();
    // Row in bits 32.., column in bits 0..: constant digits are skipped.
    radix_sort_u64(c, keys.as<uint64_t>(), nullptr, n2, 64);
    if (n2) {
      k_rows_from_keys<<<grid_for(n2, 256, c->num_sms * 16), 256, 0, c->stream>>>(keys.as<uint64_t>(), n2,
                                                                                    s.adj.as<uint32_t>());
      KT_LAUNCHED(c);
    }
  }
  gsize.release();
  // Edge ids: the upper entries number themselves; then the bitsets (dense
  // mode, built from the sorted rows); then the lower entries' ids, from the
  // bitsets' popcounts when they are there, else by binary search.
  DBuf upcnt(c, (na + 1) * sizeof(uint32_t));
  zero(c, upcnt.get(), (na + 1) * sizeof(uint32_t));
  k_upper_start<<<grid_for(na, 256, c->num_sms * 16), 256, 0, c->stream>>>(
      s.off.as<uint64_t>(), s.adj.as<uint32_t>(), na, s.up.as<uint64_t>(), upcnt.as<uint32_t>());
  KT_LAUNCHED(c);
  DBuf eoff(c, (na + 1) * sizeof(uint64_t));
  scan_u32_to_u64(c, upcnt.as<uint32_t>(), eoff.as<uint64_t>(), na + 1);
  upcnt.release();
  s.eid.alloc(c, (n2 ? n2 : 1) * sizeof(uint32_t));
  s.ends.alloc(c, (s.m ? s.m : 1) * sizeof(uint64_t));
  k_upper_ids<<<grid_for(na * 32, 256, c->num_sms * 16), 256, 0, c->stream>>>(
      s.off.as<uint64_t>(), s.adj.as<uint32_t>(), na, s.up.as<uint64_t>(), eoff.as<uint64_t>(),
      s.eid.as<uint32_t>(), s.ends.as<uint64_t>());
  KT_LAUNCHED(c);
  // Maximum degree (the last vertex in ascending-degree order).
  uint32_t md = 0;
  copy_d2h(c, &md, sdeg.as<uint32_t>() + (na - 1), sizeof(uint32_t));
  s.max_deg = md;
  build_bits(c, s);
  DenseRows R = dense_rows(s);
  if (!s.W) R.spre = nullptr;
  k_lower_ids<<<grid_for(na * 32, 256, c->num_sms * 16), 256, 0, c->stream>>>(
      s.off.as<uint64_t>(), s.adj.as<uint32_t>(), na, s.up.as<uint64_t>(), eoff.as<uint64_t>(), R,
      s.eid.as<uint32_t>());
  KT_LAUNCHED(c);
  if (idmap) {
    k_map_ids<<<grid_for(na, 256, c->num_sms * 16), 256, 0, c->stream>>>(s.orig.as<uint32_t>(), na, idmap);
    KT_LAUNCHED(c);
  }
}

}  // namespace

void build_sub(Ctx* c, const Graph& g, const KCore& kc, Sub& s) {
  (void)g;
  build_from_list(c, kc.cur(), kc.alive.as<uint32_t>(), kc.n_alive, kc.deg.as<uint32_t>(), kc.rem.as<uint32_t>(),
                  kc.map(), s);
}

void build_sub_grouped(Ctx* c, const Graph& g, const uint32_t* alive, uint64_t na, const uint32_t* deg,
                       const uint32_t* rem, const uint32_t* group_of, uint32_t ngroups, Sub& s) {
  if (g.n >= (1ull << 28)) throw Error(KT_ERR_LIMIT, "batched union: more than 2^28 vertices in a wave");
  if (ngroups > 65536) throw Error(KT_ERR_LIMIT, "batched union: more than 65536 graphs in a wave");
  build_from_list(c, g, alive, na, deg, rem, nullptr, s, group_of, ngroups);
}

void build_sub_grouped_from_keys(Ctx* c, uint64_t* keys, uint64_t m, uint32_t n_ids, const uint32_t* group_of,
                                 uint32_t ngroups, Sub& s, bool sorted) {
  Graph g;
  build_graph(c, keys, m, n_ids, g, false, sorted);
  DBuf list(c, (g.n ? g.n : 1) * sizeof(uint32_t));
  const uint64_t na = compact(c, g.n, DegPositive{g.deg.as<uint32_t>()}, list.as<uint32_t>());
  build_sub_grouped(c, g, list.as<uint32_t>(), na, g.deg.as<uint32_t>(), nullptr, group_of, ngroups, s);
}

void build_sub_all(Ctx* c, const Graph& g, Sub& s) {
  DBuf list(c, (g.n ? g.n : 1) * sizeof(uint32_t));
  const uint64_t na = compact(c, g.n, DegPositive{g.deg.as<uint32_t>()}, list.as<uint32_t>());
  build_from_list(c, g, list.as<uint32_t>(), na, g.deg.as<uint32_t>(), nullptr, nullptr, s);
}

}  // namespace kt
