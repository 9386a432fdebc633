// Stage (b): edge records -> cleaned undirected graph on the device.
//
// Two routes to the same Graph (sorted canonical edge list, symmetric CSR,
// degrees):
//
// * Grouped input -- the reference's input contract (lines grouped by the
//   second column in ascending order, every edge listed in both directions,
//   no repeats, no self-loops), with each row's first-column values in
//   ascending order.  The rows are the lines themselves, as the reference
//   builds them by concatenation (init_graph, src/kc_gpu.cpp:38-65, degrees
//   from run lengths at src/kc_gpu.cpp:283-302): one pass checks the order,
//   writes the adjacency and the row offsets; a second pass checks symmetry
//   (every arc (y -> x) with x < y is found in row x by binary search, and
//   the arcs with x > y are as many as those with x < y) and writes the
//   canonical edge list, which is the x > y arcs in line order.  Any check
//   that fails sends the records to the general route; nothing is modified
//   before that decision.
// * General route -- records in any order with repeats and self-loops:
//   canonical keys min << 32 | max (~0 = no edge) radix sorted over
//   2*ceil(log2 n) bits, repeats dropped by a sorted-unique compaction, and
//   the symmetric CSR filled from the unique list: degrees with warp-
//   aggregated atomics (runs of equal u in the sorted list collapse to one
//   atomic), an exclusive scan for the uint64 row offsets, and a cursor
//   scatter (rows unsorted; the k-core stage does not need them sorted, the
//   subgraph stage re-sorts).
#include "stages.h"

namespace kt {
namespace {

__global__ void k_degrees(const uint64_t* __restrict__ edges, uint64_t m, uint32_t* __restrict__ deg) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ((m + 31) & ~31ULL);
       i += (uint64_t)gridDim.x * blockDim.x) {
    const bool valid = i < m;
    const uint64_t k = valid ? edges[i] : ~0ULL;
    const uint32_t u = (uint32_t)(k >> 32), v = (uint32_t)k;
    // The list is sorted, so equal u values are adjacent: one atomic per run.
    const unsigned peers = __match_any_sync(kFull, u);
    if (valid && lane_id() == (unsigned)(__ffs(peers) - 1)) atomicAdd(&deg[u], (uint32_t)__popc(peers));
    if (valid) atomicAdd(&deg[v], 1u);
  }
}

__global__ void k_fill(const uint64_t* __restrict__ edges, uint64_t m, const uint64_t* __restrict__ off,
                       uint32_t* __restrict__ cur, uint32_t* __restrict__ adj) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ((m + 31) & ~31ULL);
       i += (uint64_t)gridDim.x * blockDim.x) {
    const bool valid = i < m;
    const uint64_t k = valid ? edges[i] : ~0ULL;
    const uint32_t u = (uint32_t)(k >> 32), v = (uint32_t)k;
    const unsigned peers = __match_any_sync(kFull, u);
    const unsigned leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (valid && lane_id() == leader) base = atomicAdd(&cur[u], (uint32_t)__popc(peers));
    base = __shfl_sync(kFull, base, leader);
    if (valid) {
      adj[off[u] + base + __popc(peers & lanemask_lt())] = v;
      adj[off[v] + atomicAdd(&cur[v], 1u)] = u;
    }
  }
}

__global__ void k_max_u32(const uint32_t* __restrict__ a, uint64_t n, uint32_t* out) {
  uint32_t mx = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    mx = max(mx, a[i]);
  mx = warp_max(mx);
  if (lane_id() == 0 && mx) atomicMax(out, mx);
}

// A record a << 32 | b (either order) as the canonical min << 32 | max.
__device__ __forceinline__ uint64_t canon_key(uint64_t k) {
  const uint32_t a = (uint32_t)(k >> 32), b = (uint32_t)k;
  return a < b ? k : (((uint64_t)b << 32) | a);
}

// record -> min << vb | max (both below 2^vb - 1); the "no edge" key ~0
// becomes 2^(2 vb) - 1, which sorts after every real key.  The sort then
// runs over 2 vb bits instead of 32 + vb.
__global__ void k_pack(uint64_t* __restrict__ keys, uint64_t n, int vb) {
  const uint64_t none = (((uint64_t)1) << (2 * vb)) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    const uint64_t c = canon_key(k);
    keys[i] = k == ~0ULL ? none : ((c >> 32) << vb) | (uint32_t)c;
  }
}

// record -> canonical key, with `from` (the "no edge" key) replaced by `to`.
__global__ void k_canon_remap(uint64_t* __restrict__ keys, uint64_t n, uint64_t from, uint64_t to) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    keys[i] = k == from ? to : canon_key(k);
  }
}

__global__ void k_remap(uint64_t* __restrict__ keys, uint64_t n, uint64_t from, uint64_t to) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    if (keys[i] == from) keys[i] = to;
}

// ------------------------------------------------------------ grouped input

// Largest run of vertex ids without lines between two groups that one
// thread fills in; inputs with longer gaps take the general route.
constexpr uint64_t kMaxGap = 4096;

// Pass 1 over the records y << 32 | x in line order: *bad is set unless
// every line is a record, y never decreases, and x strictly increases within
// a group.  Writes adj[i] = x, off[v] = first line of row v for every
// v in [0, n] (rows without lines get the next row's start), and up[y] =
// the first line of row y with x > y (left at ~0 when there is none).
__global__ void k_grouped_rows(const uint64_t* __restrict__ keys, uint64_t nk, uint64_t n,
                               uint64_t* __restrict__ off, uint64_t* __restrict__ up, uint32_t* __restrict__ adj,
                               uint32_t* __restrict__ bad) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nk; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    if (k == ~0ULL) {  // a blank line or a self-loop
      atomicOr(bad, 1u);
      continue;
    }
    const uint64_t y = k >> 32;
    const uint32_t x = (uint32_t)k;
    adj[i] = x;
    bool row_start = true;
    bool prev_up = false;
    if (i == 0) {
      if (y + 1 > kMaxGap) {
        atomicOr(bad, 1u);
      } else {
        for (uint64_t v = 0; v <= y; ++v) off[v] = 0;
      }
    } else {
      const uint64_t p = keys[i - 1];
      if (p != ~0ULL) {  // a ~0 line flags itself
        const uint64_t py = p >> 32;
        if (y < py) {
          atomicOr(bad, 1u);
        } else if (y > py) {
          if (y - py > kMaxGap) {
            atomicOr(bad, 1u);
          } else {
            for (uint64_t v = py + 1; v <= y; ++v) off[v] = i;
          }
        } else {
          row_start = false;
          if ((uint32_t)p >= x) atomicOr(bad, 1u);
          prev_up = (uint32_t)p > y;
        }
      }
    }
    if (i == nk - 1) {
      if (n - y > kMaxGap) {
        atomicOr(bad, 1u);
      } else {
        for (uint64_t v = y + 1; v <= n; ++v) off[v] = nk;
      }
    }
    if (x > y && (row_start || !prev_up)) up[y] = i;
  }
}

// Per vertex: degree, upper-part start (rows without x > y end there), the
// upper count, and the largest degree.
__global__ void k_grouped_degrees(uint64_t n, const uint64_t* __restrict__ off, uint64_t* __restrict__ up,
                                  uint32_t* __restrict__ deg, uint32_t* __restrict__ ucnt, uint32_t* __restrict__ mx) {
  uint32_t m = 0;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = off[v], e = off[v + 1];
    uint64_t u = up[v];
    if (u == ~0ULL) {
      u = e;
      up[v] = u;
    }
    deg[v] = (uint32_t)(e - b);
    ucnt[v] = (uint32_t)(e - u);
    m = max(m, (uint32_t)(e - b));
  }
  m = warp_max(m);
  if (lane_id() == 0 && m) atomicMax(mx, m);
}

// Pass 2: the arcs with x > y are the canonical edges y << 32 | x, written
// at their row's edge offset (they come out sorted); the arcs with x < y are
// written transposed, x << 32 | y, at their row's offset among those (row y's
// offset is off[y] - eoff[y]; they come out sorted by y).  Runs only once the
// x > y arcs are known to be half of the lines, so every index is below that
// half.
__global__ void k_grouped_split(const uint64_t* __restrict__ keys, uint64_t nk, const uint64_t* __restrict__ off,
                                const uint64_t* __restrict__ up, const uint64_t* __restrict__ eoff,
                                uint64_t* __restrict__ edges, uint64_t* __restrict__ low) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nk; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    const uint32_t y = (uint32_t)(k >> 32), x = (uint32_t)k;
    if (x > y)
      edges[eoff[y] + (i - up[y])] = k;
    else
      low[(off[y] - eoff[y]) + (i - off[y])] = ((uint64_t)x << 32) | y;
  }
}

// Pass 3: symmetry.  The transposed x < y arcs, stable-sorted by their x,
// are sorted canonical keys; the input is symmetric exactly when they equal
// the edge list entry by entry (every edge then appears once in each
// direction).
__global__ void k_equal_u64(const uint64_t* __restrict__ a, const uint64_t* __restrict__ b, uint64_t n,
                            uint32_t* __restrict__ bad) {
  bool diff = false;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    diff |= a[i] != b[i];
  if (__any_sync(kFull, diff) && lane_id() == 0) atomicOr(bad, 1u);
}

__global__ void k_unpack(uint64_t* __restrict__ keys, uint64_t n, int vb) {
  const uint64_t none = (((uint64_t)1) << (2 * vb)) - 1, low = (((uint64_t)1) << vb) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    keys[i] = k == none ? ~0ULL : ((k >> vb) << 32) | (k & low);
  }
}

int bits_for(uint64_t n) {
  int b = 0;
  while ((1ULL << b) < n) ++b;
  return b;
}

// The grouped-input route; false (g and keys untouched) when the records
// are not in that form.
bool build_graph_grouped(Ctx* c, const uint64_t* keys, uint64_t nk, uint64_t n, Graph& g) {
  if (nk == 0 || (nk & 1) || n == 0 || n > 0xffffffffULL) return false;
  const unsigned grid = grid_for(nk, 256, c->num_sms * 16);
  DBuf flags(c, 8);  // [0] bad, [1] largest degree
  zero(c, flags.get(), 8);
  DBuf off(c, (n + 1) * sizeof(uint64_t)), up(c, n * sizeof(uint64_t)), adj(c, nk * sizeof(uint32_t));
  KT_CUDA(cudaMemsetAsync(up.get(), 0xff, up.bytes(), c->stream));
  k_grouped_rows<<<grid, 256, 0, c->stream>>>(keys, nk, n, off.as<uint64_t>(), up.as<uint64_t>(), adj.as<uint32_t>(),
                                              flags.as<uint32_t>());
  KT_LAUNCHED(c);
  if (read_word<uint32_t>(c, flags.as<uint32_t>())) {
    KT_LOG(c, "kt: graph build: lines not in grouped form, sorting them\n");
    return false;
  }
  DBuf deg(c, n * sizeof(uint32_t)), ucnt(c, (n + 1) * sizeof(uint32_t));
  zero(c, ucnt.as<uint32_t>() + n, sizeof(uint32_t));
  k_grouped_degrees<<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(
      n, off.as<uint64_t>(), up.as<uint64_t>(), deg.as<uint32_t>(), ucnt.as<uint32_t>(), flags.as<uint32_t>() + 1);
  KT_LAUNCHED(c);
  DBuf eoff(c, (n + 1) * sizeof(uint64_t));
  scan_u32_to_u64(c, ucnt.as<uint32_t>(), eoff.as<uint64_t>(), n + 1);
  ucnt.release();
  // Arcs with x > y must be exactly half of the lines (the other half being
  // their reverses, checked next).
  if (2 * read_word<uint64_t>(c, eoff.as<uint64_t>() + n) != nk) {
    KT_LOG(c, "kt: graph build: grouped lines are not symmetric, sorting them\n");
    return false;
  }
  const uint64_t m = nk / 2;
  DBuf edges(c, m * sizeof(uint64_t)), low(c, m * sizeof(uint64_t));
  k_grouped_split<<<grid, 256, 0, c->stream>>>(keys, nk, off.as<uint64_t>(), up.as<uint64_t>(), eoff.as<uint64_t>(),
                                               edges.as<uint64_t>(), low.as<uint64_t>());
  KT_LAUNCHED(c);
  up.release();
  eoff.release();
  // Sorted by x, the high half (stable: y stays ascending within each x).
  radix_sort_u64(c, low.as<uint64_t>(), nullptr, m, 32 + bits_for(n), 32);
  k_equal_u64<<<grid_for(m, 256, c->num_sms * 16), 256, 0, c->stream>>>(low.as<uint64_t>(), edges.as<uint64_t>(),
                                                                          m, flags.as<uint32_t>());
  KT_LAUNCHED(c);
  low.release();
  uint32_t h[2];
  copy_d2h(c, h, flags.get(), 8);
  if (h[0]) {
    KT_LOG(c, "kt: graph build: grouped lines are not symmetric, sorting them\n");
    return false;
  }
  g.n = n;
  g.m = m;
  g.off = std::move(off);
  g.adj = std::move(adj);
  g.edges = std::move(edges);
  g.deg = std::move(deg);
  g.max_deg = h[1];
  return true;
}

void build_graph_sorted(Ctx* c, uint64_t* keys, uint64_t nkeys, uint64_t n, Graph& g, bool presorted);

// Sets *bad when keys[i] >= keys[i+1] for some i (not strictly ascending).
__global__ void k_not_ascending(const uint64_t* __restrict__ keys, uint64_t n, unsigned int* bad) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i + 1 < n; i += (uint64_t)gridDim.x * blockDim.x)
    if (keys[i] >= keys[i + 1]) *bad = 1u;
}

}  // namespace

void build_graph(Ctx* c, uint64_t* keys, uint64_t nkeys, uint64_t n, Graph& g, bool lines, bool sorted) {
  // Vertex counts travel as u32 through the later stages: the all-ones id
  // (which would make n = 2^32) is refused.
  if (n > 0xffffffffULL) throw Error(KT_ERR_LIMIT, "vertex id 4294967295: ids must be below 2^32 - 1");
  c->stats.csr_grouped = 0;
  if (lines && build_graph_grouped(c, keys, nkeys, n, g)) {
    c->stats.csr_grouped = 1;
    return;
  }
  bool presorted = false;
  if (sorted && nkeys > 1) {
    DBuf bad(c, 4);
    zero(c, bad.get(), 4);
    k_not_ascending<<<grid_for(nkeys, 256, c->num_sms * 16), 256, 0, c->stream>>>(keys, nkeys,
                                                                                  bad.as<unsigned int>());
    KT_LAUNCHED(c);
    presorted = read_word<unsigned int>(c, bad.as<unsigned int>()) == 0;
  }
  build_graph_sorted(c, keys, nkeys, n, g, presorted);
}

namespace {

void build_graph_sorted(Ctx* c, uint64_t* keys, uint64_t nkeys, uint64_t n, Graph& g, bool presorted) {
  g.n = n;
  if (presorted) {
    // Canonical, ascending and distinct already (survivors taken from a
    // working graph's edge list): no sort, no dedup.
    g.edges.alloc(c, nkeys * sizeof(uint64_t));
    KT_CUDA(cudaMemcpyAsync(g.edges.get(), keys, nkeys * sizeof(uint64_t), cudaMemcpyDeviceToDevice, c->stream));
    g.m = nkeys;
  } else {
    // Keys are min << 32 | max with both halves below 2^vb - 1; the radix sort
    // skips digits shared by every key, so it runs 2 ceil(vb / 8) passes once
    // the "no edge" key ~0 is rewritten to ((2^vb - 1) << 32) | (2^vb - 1)
    // (still last).  When packing to min << vb | max saves a pass (2 vb bits,
    // ceil(2 vb / 8) passes), the keys are packed instead.
    const int vb = bits_for(n + 1);
    const bool small = vb < 32 && nkeys;
    const bool pack = small && (2 * vb + 7) / 8 < 2 * ((vb + 7) / 8);
    const uint64_t sentinel = ((((uint64_t)1 << (vb & 31)) - 1) << 32) | (((uint64_t)1 << (vb & 31)) - 1);
    // Records may hold either end first: every route makes them canonical.
    if (pack) {
      k_pack<<<grid_for(nkeys, 256, c->num_sms * 16), 256, 0, c->stream>>>(keys, nkeys, vb);
      KT_LAUNCHED(c);
    } else if (nkeys) {
      k_canon_remap<<<grid_for(nkeys, 256, c->num_sms * 16), 256, 0, c->stream>>>(keys, nkeys, ~0ULL,
                                                                                   small ? sentinel : ~0ULL);
      KT_LAUNCHED(c);
    }
    if (nkeys > 1) radix_sort_u64(c, keys, nullptr, nkeys, 64);
    if (pack) {
      k_unpack<<<grid_for(nkeys, 256, c->num_sms * 16), 256, 0, c->stream>>>(keys, nkeys, vb);
      KT_LAUNCHED(c);
    } else if (small) {
      k_remap<<<grid_for(nkeys, 256, c->num_sms * 16), 256, 0, c->stream>>>(keys, nkeys, sentinel, ~0ULL);
      KT_LAUNCHED(c);
    }
    g.edges.alloc(c, (nkeys ? nkeys : 1) * sizeof(uint64_t));
    g.m = unique_sorted_u64(c, keys, g.edges.as<uint64_t>(), nkeys);
  }
  if ((uint64_t)2 * g.m >= 0xffffffffULL * 4ULL) throw Error(KT_ERR_LIMIT, "graph too large");
  g.deg.alloc(c, (n ? n : 1) * sizeof(uint32_t));
  zero(c, g.deg.get(), (n ? n : 1) * sizeof(uint32_t));
  const unsigned grid = grid_for(g.m, 256, c->num_sms * 16);
  if (g.m) {
    k_degrees<<<grid, 256, 0, c->stream>>>(g.edges.as<uint64_t>(), g.m, g.deg.as<uint32_t>());
    KT_LAUNCHED(c);
  }
  g.off.alloc(c, (n + 1) * sizeof(uint64_t));
  // off[n] = 2m: scan n+1 entries with a zero appended.
  DBuf degx(c, (n + 1) * sizeof(uint32_t));
  zero(c, degx.get(), (n + 1) * sizeof(uint32_t));
  if (n) KT_CUDA(cudaMemcpyAsync(degx.get(), g.deg.get(), n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, c->stream));
  scan_u32_to_u64(c, degx.as<uint32_t>(), g.off.as<uint64_t>(), n + 1);
  g.adj.alloc(c, (g.m ? 2 * g.m : 1) * sizeof(uint32_t));
  if (g.m) {
    zero(c, degx.get(), (n + 1) * sizeof(uint32_t));  // reused as per-row cursors
    k_fill<<<grid, 256, 0, c->stream>>>(g.edges.as<uint64_t>(), g.m, g.off.as<uint64_t>(), degx.as<uint32_t>(),
                                        g.adj.as<uint32_t>());
    KT_LAUNCHED(c);
  }
  DBuf mx(c, 4);
  zero(c, mx.get(), 4);
  if (n) {
    k_max_u32<<<grid_for(n, 256, c->num_sms * 8), 256, 0, c->stream>>>(g.deg.as<uint32_t>(), n, mx.as<uint32_t>());
    KT_LAUNCHED(c);
  }
  g.max_deg = read_word<uint32_t>(c, mx.as<uint32_t>());
}

}  // namespace

}  // namespace kt
