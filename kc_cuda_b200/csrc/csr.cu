// Stage (b): canonical edge keys -> cleaned undirected graph on the device.
//
// keys (min << 32 | max, ~0 = no edge) are radix sorted over 2*ceil(log2 n)
// bits, repeats are dropped by a sorted-unique compaction, and the symmetric
// CSR is filled from the unique list: degrees with warp-aggregated atomics
// (runs of equal u in the sorted list collapse to one atomic), an exclusive
// scan for the uint64 row offsets, and a cursor scatter (rows unsorted; the
// k-core stage does not need them sorted, the subgraph stage re-sorts).
// Replaces init_graph (src/kc_gpu.cpp:38-65), whose rows come straight from
// the file because the reference requires pre-cleaned, grouped input.
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

// u << 32 | v -> u << vb | v (both below 2^vb - 1); the "no edge" key ~0
// becomes 2^(2 vb) - 1, which sorts after every real key.  The sort then
// runs over 2 vb bits instead of 32 + vb.
__global__ void k_pack(uint64_t* __restrict__ keys, uint64_t n, int vb) {
  const uint64_t none = (((uint64_t)1) << (2 * vb)) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    keys[i] = k == ~0ULL ? none : ((k >> 32) << vb) | (uint32_t)k;
  }
}

__global__ void k_remap(uint64_t* __restrict__ keys, uint64_t n, uint64_t from, uint64_t to) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    if (keys[i] == from) keys[i] = to;
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

}  // namespace

void build_graph(Ctx* c, uint64_t* keys, uint64_t nkeys, uint64_t n, Graph& g) {
  // Vertex counts travel as u32 through the later stages: the all-ones id
  // (which would make n = 2^32) is refused.
  if (n > 0xffffffffULL) throw Error(KT_ERR_LIMIT, "vertex id 4294967295: ids must be below 2^32 - 1");
  g.n = n;
  // Keys are min << 32 | max with both halves below 2^vb - 1; the radix sort
  // skips digits shared by every key, so it runs 2 ceil(vb / 8) passes once
  // the "no edge" key ~0 is rewritten to ((2^vb - 1) << 32) | (2^vb - 1)
  // (still last).  When packing to min << vb | max saves a pass (2 vb bits,
  // ceil(2 vb / 8) passes), the keys are packed instead.
  const int vb = bits_for(n + 1);
  const bool small = vb < 32 && nkeys;
  const bool pack = small && (2 * vb + 7) / 8 < 2 * ((vb + 7) / 8);
  const uint64_t sentinel = ((((uint64_t)1 << (vb & 31)) - 1) << 32) | (((uint64_t)1 << (vb & 31)) - 1);
  if (pack) {
    k_pack<<<grid_for(nkeys, 256, c->num_sms * 16), 256, 0, c->stream>>>(keys, nkeys, vb);
    KT_LAUNCHED(c);
  } else if (small) {
    k_remap<<<grid_for(nkeys, 256, c->num_sms * 16), 256, 0, c->stream>>>(keys, nkeys, ~0ULL, sentinel);
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

}  // namespace kt
