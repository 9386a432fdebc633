// Batched solving of many graphs (thousands, of uneven sizes) per launch
// sequence, and the device generator of the batched mix.
//
// A batch is cut into waves that fit the context's HBM budget.  A wave is
// one disjoint union: every graph's vertex ids are offset by the vertex
// count of the graphs before it (vbase), all their edges go through ONE
// sort/dedup/CSR build, ONE core decomposition, and -- on the union of the
// graphs' cores, grouped by graph -- ONE support count and ONE peel whose
// levels are shared by all graphs while every graph keeps its own record
// (per-graph alive edges and minimum support after each level).  Triangles
// never cross graphs, so each graph's answer is exactly its own.
//
// Per graph the two phases of the single-graph driver are kept: the truss of
// its maximum core gives L (and the answer when L = cmax + 1); otherwise its
// (L-1)-core joins the second union.
//
// Graphs of the batched mix (ktg_mix_spec: R-MAT or Erdos-Renyi, one planted
// clique) are generated on the device from their seeds straight into the
// wave's key buffer, with the host generator's integer conventions
// (ktgen_core.h), so a device-generated graph equals ktg_make's.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <exception>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

#include "batch.h"
#include "compact.cuh"
#include "handles.h"
#include "ktgen.h"
#include "ktgen_core.h"
#include "solve.h"

namespace kt {
namespace {

// Device specs of the generated graphs of a wave.
struct GenSpec {
  uint64_t seed;
  uint64_t n;
  uint64_t draws;
  uint64_t gen_off;  // first draw index of this graph in the wave's draw space
  uint64_t key_off;  // first key slot
  uint64_t vbase;    // first union vertex id
  uint32_t kind;
  uint32_t scale;
};

__global__ void k_gen_draws(const GenSpec* __restrict__ specs, uint32_t ns, uint64_t total, ktg_rmat_t thr,
                            uint64_t* __restrict__ keys) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = ns;  // last spec with gen_off <= i
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (specs[mid].gen_off <= i)
        lo = mid;
      else
        hi = mid;
    }
    const GenSpec& s = specs[lo];
    const uint64_t j = i - s.gen_off;
    const uint64_t xy = s.kind == KTG_RMAT ? ktg_rmat_draw(s.seed, thr, s.scale, j) : ktg_er_draw(s.seed, s.n, j);
    const uint64_t k = ktg_canon(xy, s.n);
    keys[s.key_off + j] = k == ~0ULL ? ~0ULL : (((k >> 32) + s.vbase) << 32) | ((uint32_t)k + s.vbase);
  }
}

// Extra keys of a wave (clique edges of generated graphs, records of host
// graphs; already canonical union keys) from one staging buffer into their
// graphs' key ranges: graph g's run [src[g], src[g+1]) of the staging buffer
// goes to keys[dst[g]...].
__global__ void k_place_extra(const uint64_t* __restrict__ stage, uint64_t total, const uint64_t* __restrict__ src,
                              const uint64_t* __restrict__ dst, uint32_t ng, uint64_t* __restrict__ keys) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = ng;  // last graph with src <= i
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (src[mid] <= i)
        lo = mid;
      else
        hi = mid;
    }
    keys[dst[lo] + (i - src[lo])] = stage[i];
  }
}

__global__ void k_group_of(const uint64_t* __restrict__ vbase, uint32_t ng, uint64_t n, uint32_t* __restrict__ gid) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = ng;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (vbase[mid] <= v)
        lo = mid;
      else
        hi = mid;
    }
    gid[v] = lo;
  }
}

__global__ void k_group_max(const uint32_t* __restrict__ val, const uint32_t* __restrict__ gid, uint64_t n,
                            uint32_t* __restrict__ out) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < ((n + 31) & ~31ULL);
       v += (uint64_t)gridDim.x * blockDim.x) {
    const bool ok = v < n;
    const uint32_t g = ok ? gid[v] : 0xffffffffu;
    const uint32_t x = ok ? val[v] : 0u;
    const unsigned peers = __match_any_sync(kFull, g);
    const uint32_t mx = __reduce_max_sync(peers, x);
    if (ok && lane_id() == (unsigned)(__ffs(peers) - 1)) atomicMax(&out[g], mx);
  }
}

// Per graph: vertices in its maximum core (core == cmax[g]) and vertices
// with an edge (core >= 1).
__global__ void k_group_counts(const uint32_t* __restrict__ core, const uint32_t* __restrict__ gid, uint64_t n,
                               const uint32_t* __restrict__ cmax, unsigned long long* __restrict__ in_max,
                               unsigned long long* __restrict__ with_edge) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < ((n + 31) & ~31ULL);
       v += (uint64_t)gridDim.x * blockDim.x) {
    const bool ok = v < n;
    const uint32_t g = ok ? gid[v] : 0xffffffffu;
    const uint32_t k = ok ? core[v] : 0u;
    const unsigned peers = __match_any_sync(kFull, g);
    const unsigned a = __popc(__ballot_sync(kFull, ok && k >= 1) & peers);
    const unsigned b = __popc(__ballot_sync(kFull, ok && k >= 1 && k == cmax[ok ? g : 0]) & peers);
    if (ok && lane_id() == (unsigned)(__ffs(peers) - 1)) {
      if (a) atomicAdd(&with_edge[g], (unsigned long long)a);
      if (b) atomicAdd(&in_max[g], (unsigned long long)b);
    }
  }
}

// Per graph: vertices with core >= need[g] (need 0: none counted).
__global__ void k_group_at_least(const uint32_t* __restrict__ core, const uint32_t* __restrict__ gid, uint64_t n,
                                 const uint32_t* __restrict__ need, unsigned long long* __restrict__ cnt) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < ((n + 31) & ~31ULL);
       v += (uint64_t)gridDim.x * blockDim.x) {
    const bool ok = v < n;
    const uint32_t g = ok ? gid[v] : 0xffffffffu;
    const uint32_t k = ok ? need[g] : 0u;
    const bool in = ok && k && core[v] >= k;
    const unsigned peers = __match_any_sync(kFull, g);
    const unsigned a = __popc(__ballot_sync(kFull, in) & peers);
    if (ok && a && lane_id() == (unsigned)(__ffs(peers) - 1)) atomicAdd(&cnt[g], (unsigned long long)a);
  }
}

// Vertices of graph g with core >= need[g] (need 0 = graph not taken).
struct CoreAtLeast {
  const uint32_t* core;
  const uint32_t* gid;
  const uint32_t* need;
  __device__ bool keep(uint64_t v) const {
    const uint32_t k = need[gid[v]];
    return k && core[v] >= k;
  }
  __device__ uint32_t value(uint64_t v) const { return (uint32_t)v; }
};

__global__ void k_mark(const uint32_t* __restrict__ list, uint64_t na, uint32_t* __restrict__ rem) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += (uint64_t)gridDim.x * blockDim.x)
    rem[list[i]] = kAlive;
}

// deg[v] = alive neighbours, warp per alive vertex.
__global__ void k_alive_degree(const uint32_t* __restrict__ list, uint64_t na, const uint64_t* __restrict__ off,
                               const uint32_t* __restrict__ adj, const uint32_t* __restrict__ rem,
                               uint32_t* __restrict__ deg) {
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t i = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); i < na; i += warps) {
    const uint32_t v = list[i];
    uint32_t c = 0;
    for (uint64_t j = off[v] + lane_id(); j < off[v + 1]; j += 32) c += rem[adj[j]] == kAlive;
    c = warp_sum(c);
    if (lane_id() == 0) deg[v] = c;
  }
}

// Clique keys (local canonical u << 32 | v) of a planted clique.
void clique_keys(const std::vector<uint32_t>& vs, std::vector<uint64_t>& out) {
  for (size_t i = 0; i < vs.size(); ++i)
    for (size_t j = i + 1; j < vs.size(); ++j) {
      const uint64_t a = vs[i], b = vs[j];
      out.push_back(a < b ? (a << 32 | b) : (b << 32 | a));
    }
}

}  // namespace

void BatchItem::from_mix(uint64_t index, uint64_t base_seed) {
  generated = true;
  ktg_spec s;
  ktg_mix_spec(index, base_seed, &s);
  kind = s.kind;
  scale = s.scale;
  n = s.n;
  draws = s.draws;
  seed = s.seed;
  extra.clear();
  for (uint32_t c = 0; c < s.n_cliques; ++c) {
    std::vector<uint32_t> vs(s.clique_sizes[c]);
    ktg_sample_vertices(s.seed, KTG_STREAM_CLIQUE + c, n, s.clique_sizes[c], vs.data());
    clique_keys(vs, extra);
  }
  nkeys = draws + extra.size();
}

void BatchItem::from_pairs(const uint64_t* xy, uint64_t count) {
  generated = false;
  extra.assign(xy, xy + count);
  uint64_t mx = 0;
  bool any = false;
  for (uint64_t i = 0; i < count; ++i) {
    mx = std::max<uint64_t>(mx, std::max<uint64_t>(xy[i] >> 32, (uint32_t)xy[i]));
    any = true;
  }
  n = any ? mx + 1 : 0;
  draws = 0;
  nkeys = count;
}

// Keys of one wave (union ids) into `keys`; returns the union vertex count.
static uint64_t wave_keys(Ctx* c, const std::vector<BatchItem*>& items, DBuf& keys, uint64_t& nkeys,
                          std::vector<uint64_t>& vbase) {
  const uint32_t G = (uint32_t)items.size();
  vbase.assign(G + 1, 0);
  std::vector<uint64_t> key_off(G + 1, 0);
  for (uint32_t g = 0; g < G; ++g) {
    vbase[g + 1] = vbase[g] + items[g]->n;
    key_off[g + 1] = key_off[g] + items[g]->nkeys;
  }
  nkeys = key_off[G];
  keys.alloc(c, (nkeys ? nkeys : 1) * sizeof(uint64_t));
  std::vector<GenSpec> specs;
  uint64_t gen_total = 0;
  std::vector<uint64_t> extra_all;  // clique keys, already in union ids
  for (uint32_t g = 0; g < G; ++g) {
    const BatchItem& it = *items[g];
    if (it.generated) {
      GenSpec s;
      s.seed = it.seed;
      s.n = it.n;
      s.draws = it.draws;
      s.gen_off = gen_total;
      s.key_off = key_off[g];
      s.vbase = vbase[g];
      s.kind = it.kind;
      s.scale = it.scale;
      specs.push_back(s);
      gen_total += it.draws;
    }
  }
  DBuf dspecs;
  if (!specs.empty() && gen_total) {
    dspecs.alloc(c, specs.size() * sizeof(GenSpec));
    copy_h2d(c, dspecs.get(), specs.data(), specs.size() * sizeof(GenSpec));
    const ktg_rmat_t thr = ktg_rmat_thresholds(570000, 190000, 190000);
    k_gen_draws<<<grid_for(gen_total, 256, c->num_sms * 32), 256, 0, c->stream>>>(
        dspecs.as<GenSpec>(), (uint32_t)specs.size(), gen_total, thr, keys.as<uint64_t>());
    KT_LAUNCHED(c);
  }
  // Clique keys of generated graphs and records of host graphs (canonical,
  // self-loops -> ~0), in union ids, through one staging copy.
  std::vector<uint64_t> stage_h, src, dst;
  for (uint32_t g = 0; g < G; ++g) {
    const BatchItem& it = *items[g];
    if (it.extra.empty()) continue;
    src.push_back(stage_h.size());
    dst.push_back(key_off[g] + it.draws);
    const uint64_t vb = vbase[g];
    for (uint64_t k : it.extra) {
      const uint64_t x = k >> 32, y = (uint32_t)k;
      stage_h.push_back(x == y ? ~0ULL : (x < y ? ((x + vb) << 32) | (y + vb) : ((y + vb) << 32) | (x + vb)));
    }
  }
  if (!stage_h.empty()) {
    const uint32_t ng = (uint32_t)src.size();
    DBuf stage(c, stage_h.size() * sizeof(uint64_t)), dsrc(c, ng * sizeof(uint64_t)), ddst(c, ng * sizeof(uint64_t));
    copy_h2d(c, stage.get(), stage_h.data(), stage_h.size() * sizeof(uint64_t));
    copy_h2d(c, dsrc.get(), src.data(), ng * sizeof(uint64_t));
    copy_h2d(c, ddst.get(), dst.data(), ng * sizeof(uint64_t));
    k_place_extra<<<grid_for(stage_h.size(), 256, c->num_sms * 16), 256, 0, c->stream>>>(
        stage.as<uint64_t>(), stage_h.size(), dsrc.as<uint64_t>(), ddst.as<uint64_t>(), ng, keys.as<uint64_t>());
    KT_LAUNCHED(c);
    sync(c);  // the host staging vectors go out of scope
  }
  return vbase[G];
}

// Union working graph: the vertices of graph g whose core number reaches
// need[g] (0 = none of g), grouped by graph.
static void union_sub(Ctx* c, const Graph& U, const uint32_t* dcore, const uint32_t* dgid, uint32_t G,
                      const std::vector<uint32_t>& need, Sub& s) {
  DBuf dneed(c, G * sizeof(uint32_t));
  copy_h2d(c, dneed.get(), need.data(), G * sizeof(uint32_t));
  DBuf list(c, (U.n ? U.n : 1) * sizeof(uint32_t));
  const uint64_t na = compact(c, U.n, CoreAtLeast{dcore, dgid, dneed.as<uint32_t>()}, list.as<uint32_t>());
  DBuf rem(c, (U.n ? U.n : 1) * sizeof(uint32_t)), deg(c, (U.n ? U.n : 1) * sizeof(uint32_t));
  zero(c, rem.get(), rem.bytes());
  if (na) {
    k_mark<<<grid_for(na, 256, c->num_sms * 16), 256, 0, c->stream>>>(list.as<uint32_t>(), na, rem.as<uint32_t>());
    KT_LAUNCHED(c);
    k_alive_degree<<<grid_for(na * 32, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        list.as<uint32_t>(), na, U.off.as<uint64_t>(), U.adj.as<uint32_t>(), rem.as<uint32_t>(),
        deg.as<uint32_t>());
    KT_LAUNCHED(c);
  }
  build_sub_grouped(c, U, list.as<uint32_t>(), na, deg.as<uint32_t>(), rem.as<uint32_t>(), dgid, G, s);
}

// Edges of graph thr's group with support >= thr[group] (thr 0: none).
struct GroupAtLeast {
  const uint32_t* sup;
  const uint64_t* ends;
  const uint32_t* vgid;
  const uint32_t* thr;
  __device__ bool keep(uint64_t e) const {
    const uint32_t t = thr[vgid[(uint32_t)(ends[e] >> 32)]];
    return t && sup[e] >= t;
  }
  __device__ uint64_t value(uint64_t e) const { return ends[e]; }
};

// Per-graph support histograms: hist[hoff[g] + min(sup, cap[g])] += 1.
__global__ void k_group_hist(const uint32_t* __restrict__ sup, const uint64_t* __restrict__ ends, uint64_t m,
                             const uint32_t* __restrict__ vgid, const uint32_t* __restrict__ hoff,
                             const uint32_t* __restrict__ cap, unsigned long long* __restrict__ hist) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ((m + 31) & ~31ULL);
       e += (uint64_t)gridDim.x * blockDim.x) {
    const bool ok = e < m;
    uint32_t b = 0xffffffffu;
    if (ok) {
      const uint32_t g = vgid[(uint32_t)(ends[e] >> 32)];
      b = hoff[g] + min(sup[e], cap[g]);
    }
    const unsigned peers = __match_any_sync(kFull, b);
    if (ok && lane_id() == (unsigned)(__ffs(peers) - 1)) atomicAdd(&hist[b], (unsigned long long)__popc(peers));
  }
}

// Per-graph support bounds (the single-graph rule: largest t <= cap[g] with
// t(t-1)/2 edges of support >= t-2; 0 if none) over a grouped union.
static std::vector<uint32_t> group_bounds(Ctx* c, const Sub& s, const uint32_t* sup, const std::vector<uint32_t>& cap) {
  const uint32_t G = (uint32_t)cap.size();
  std::vector<uint32_t> hoff(G + 1, 0), out(G, 0);
  for (uint32_t g = 0; g < G; ++g) hoff[g + 1] = hoff[g] + cap[g] + 1;
  if (s.m == 0) return out;
  DBuf dh(c, (uint64_t)hoff[G] * 8), doff(c, G * 4ull), dcap(c, G * 4ull);
  zero(c, dh.get(), dh.bytes());
  copy_h2d(c, doff.get(), hoff.data(), G * 4ull);
  copy_h2d(c, dcap.get(), cap.data(), G * 4ull);
  k_group_hist<<<grid_for(s.m, 256, c->num_sms * 16), 256, 0, c->stream>>>(
      sup, s.ends.as<uint64_t>(), s.m, s.vgid.as<uint32_t>(), doff.as<uint32_t>(), dcap.as<uint32_t>(),
      dh.as<unsigned long long>());
  KT_LAUNCHED(c);
  std::vector<unsigned long long> h(hoff[G]);
  copy_d2h(c, h.data(), dh.get(), h.size() * 8);
  for (uint32_t g = 0; g < G; ++g) {
    const uint32_t cp = cap[g];
    if (cp < 3) continue;
    const unsigned long long* hg = h.data() + hoff[g];
    unsigned long long at_least = hg[cp] + hg[cp - 1];
    for (uint32_t t = cp; t >= 3; --t) {
      at_least += hg[t - 2];
      if (at_least >= (unsigned long long)t * (t - 1) / 2) {
        out[g] = t;
        break;
      }
    }
  }
  return out;
}

// Survivors: the union of each graph's edges with support >= thr[g],
// rebuilt as a grouped working graph with exact supports.  When `only_if_few`
// and they are not fewer than half the edges, nothing is built (false).
static bool survivors(Ctx* c, const Sub& s, const uint32_t* sup, const std::vector<uint32_t>& thr, bool only_if_few,
                      Sub& out, DBuf& out_sup) {
  const uint32_t G = (uint32_t)thr.size();
  DBuf dthr(c, G * 4ull);
  copy_h2d(c, dthr.get(), thr.data(), G * 4ull);
  DBuf keys(c, (s.m ? s.m : 1) * sizeof(uint64_t));
  const uint64_t k = compact(c, s.m, GroupAtLeast{sup, s.ends.as<uint64_t>(), s.vgid.as<uint32_t>(),
                                                  dthr.as<uint32_t>()},
                             keys.as<uint64_t>());
  KT_LOG(c, "kt: batch survivors: %llu of %llu edges\n", (unsigned long long)k, (unsigned long long)s.m);
  if (only_if_few && k * 2 >= s.m) return false;
  build_sub_grouped_from_keys(c, keys.as<uint64_t>(), k, s.n, s.vgid.as<uint32_t>(), G, out, true);
  keys.release();
  out_sup = DBuf(c, (out.m ? out.m : 1) * sizeof(uint32_t));
  edge_support(c, out, out_sup.as<uint32_t>());
  return true;
}

// Tracked peel of a grouped union: graph g from level t0[g] with early stop
// at stop[g] edges (0: none); returns each graph's last recorded level and
// its edge count.
static void tracked_peel(Ctx* c, const Sub& s, uint32_t* sup, const std::vector<uint32_t>& t0,
                         const std::vector<uint64_t>& stop, std::vector<uint32_t>& kmax,
                         std::vector<uint64_t>& count) {
  const uint32_t G = (uint32_t)t0.size();
  kmax.assign(G, 0);
  count.assign(G, 0);
  if (s.m == 0) return;
  DBuf dk(c, G * sizeof(uint32_t)), dc(c, G * sizeof(uint64_t)), dt0(c, G * sizeof(uint32_t)),
      dstop(c, G * sizeof(uint64_t));
  zero(c, dk.get(), dk.bytes());
  zero(c, dc.get(), dc.bytes());
  copy_h2d(c, dt0.get(), t0.data(), G * sizeof(uint32_t));
  copy_h2d(c, dstop.get(), stop.data(), G * sizeof(uint64_t));
  GraphTrack tr{s.vgid.as<uint32_t>(), G, dk.as<uint32_t>(), dc.as<uint64_t>(), dt0.as<uint32_t>(),
                dstop.as<uint64_t>()};
  const PeelResult pr = truss_peel(c, s, sup, 3, 0, nullptr, 0, &tr);
  c->stats.levels += pr.levels;
  c->stats.rounds += (uint32_t)pr.rounds;
  copy_d2h(c, kmax.data(), dk.get(), G * sizeof(uint32_t));
  copy_d2h(c, count.data(), dc.get(), G * sizeof(uint64_t));
}

// One wave: the phases of the single-graph driver, each graph on its own
// levels, all graphs of the wave in each launch.
//   1. On the union of maximum cores (2-cores for the graphs whose maximum
//      core is a large part of them -- their answer is final after this
//      phase): per-graph support bounds; graph g tries
//      level min(bound, (cmax+1)/2) on its edges of support >= level-2
//      (rebuilt), halving toward 3 while that truss is empty.
//   2. On the union of (L-1)-cores of the graphs whose bound L = cmax + 1 is
//      not met: edges of support >= L-2, peeled from L with early stop at
//      phase 1's count.
void solve_wave(Ctx* c, const std::vector<BatchItem*>& items) {
  const uint32_t G = (uint32_t)items.size();
  kt_stats& st = c->stats;
  DBuf keys;
  uint64_t nkeys = 0;
  std::vector<uint64_t> vbase;
  // Input: generation (or upload) of the wave's edge keys, timed apart.
  KT_CUDA(cudaEventRecord(c->ev[4], c->stream));
  const uint64_t nv = wave_keys(c, items, keys, nkeys, vbase);
  KT_CUDA(cudaEventRecord(c->ev[5], c->stream));
  st.ms_parse += event_ms(c->ev[4], c->ev[5]);
  Timer tm(c);
  tm.start();
  Graph U;
  build_graph(c, keys.as<uint64_t>(), nkeys, nv, U);
  keys.release();
  st.ms_csr += tm.stop();
  if (G == 1) {
    // A wave of one graph takes the single-graph driver: k-core probes
    // instead of the union's full decomposition, and none of the per-graph
    // bookkeeping of a union.  Its per-solve figures add to the batch's.
    const kt_stats before = st;
    solve_graph_inner(c, U, &items[0]->kmax, &items[0]->count);
    st.core_vertices += before.core_vertices;
    st.core_edges += before.core_edges;
    st.predict_vertices += before.predict_vertices;
    st.predict_edges += before.predict_edges;
    st.cmax = before.cmax;
    st.kmax_lower_bound = before.kmax_lower_bound;
    if (items[0]->kmax < 3) {
      items[0]->kmax = 0;
      items[0]->count = 0;
    }
    return;
  }
  // Core numbers of the union and each graph's maximum core.
  tm.start();
  DBuf dcore(c, (nv ? nv : 1) * sizeof(uint32_t));
  {
    KCore kc;
    kc.init(c, U);
    kc.core_numbers(c, dcore.as<uint32_t>());
  }
  DBuf dvb(c, (G + 1) * sizeof(uint64_t)), dgid(c, (nv ? nv : 1) * sizeof(uint32_t)), dcm(c, G * sizeof(uint32_t));
  copy_h2d(c, dvb.get(), vbase.data(), (G + 1) * sizeof(uint64_t));
  zero(c, dcm.get(), dcm.bytes());
  if (nv) {
    k_group_of<<<grid_for(nv, 256, c->num_sms * 16), 256, 0, c->stream>>>(dvb.as<uint64_t>(), G, nv,
                                                                            dgid.as<uint32_t>());
    KT_LAUNCHED(c);
    k_group_max<<<grid_for(nv, 256, c->num_sms * 16), 256, 0, c->stream>>>(dcore.as<uint32_t>(), dgid.as<uint32_t>(),
                                                                             nv, dcm.as<uint32_t>());
    KT_LAUNCHED(c);
  }
  std::vector<uint32_t> cmax(G);
  copy_d2h(c, cmax.data(), dcm.get(), G * sizeof(uint32_t));
  // Graphs whose maximum core is a large part of them take one phase (the
  // single-graph driver's rule): the truss levels of their 2-core.
  std::vector<unsigned long long> in_max(G, 0), with_edge(G, 0);
  if (nv) {
    DBuf dmx(c, G * 8ull), dwe(c, G * 8ull);
    zero(c, dmx.get(), dmx.bytes());
    zero(c, dwe.get(), dwe.bytes());
    k_group_counts<<<grid_for(nv, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        dcore.as<uint32_t>(), dgid.as<uint32_t>(), nv, dcm.as<uint32_t>(), dmx.as<unsigned long long>(),
        dwe.as<unsigned long long>());
    KT_LAUNCHED(c);
    copy_d2h(c, in_max.data(), dmx.get(), G * 8ull);
    copy_d2h(c, with_edge.data(), dwe.get(), G * 8ull);
  }
  std::vector<char> single(G, 0);
  for (uint32_t g = 0; g < G; ++g) single[g] = in_max[g] * 4 >= with_edge[g];
  st.ms_kcore += tm.stop();

  // The graphs of a wave are split in two classes for each phase: those
  // whose working core fits the bitset limit (dense_max_n vertices) and the
  // others.  A union takes the bitset kernels only when every graph in it
  // fits, so each class gets a union of its own and every graph runs the
  // kernels it would run alone.
  const uint64_t dense_lim = (uint64_t)std::max<int64_t>(0, c->opt.dense_max_n);

  // Phase 1.
  std::vector<uint32_t> L(G, 0);
  std::vector<uint64_t> C(G, 0);
  std::vector<uint32_t> need1(G, 0), cap1(G, 0);
  for (uint32_t g = 0; g < G; ++g)
    if (cmax[g] >= 2) {
      need1[g] = single[g] ? 2 : cmax[g];
      cap1[g] = cmax[g] + 1;
    }
  for (int cls = 0; cls < 2; ++cls) {
    std::vector<uint32_t> need(G, 0), cap(G, 0);
    bool any1 = false;
    for (uint32_t g = 0; g < G; ++g) {
      const uint64_t nsub = single[g] ? with_edge[g] : in_max[g];
      if (need1[g] && (nsub <= dense_lim) == (cls == 0)) {
        need[g] = need1[g];
        cap[g] = cap1[g];
        any1 = true;
      }
    }
    if (!any1) continue;
    tm.start();
    Sub s1;
    union_sub(c, U, dcore.as<uint32_t>(), dgid.as<uint32_t>(), G, need, s1);
    st.predict_vertices += s1.n;
    st.predict_edges += s1.m;
    st.ms_subgraph += tm.stop();
    tm.start();
    DBuf sup1(c, (s1.m ? s1.m : 1) * sizeof(uint32_t));
    edge_support(c, s1, sup1.as<uint32_t>());
    const std::vector<uint32_t> ub = group_bounds(c, s1, sup1.as<uint32_t>(), cap);
    st.ms_support += tm.stop();
    tm.start();
    std::vector<uint32_t> level(G, 0);
    bool pending = false;
    for (uint32_t g = 0; g < G; ++g)
      if (need[g] && ub[g] >= 3) {
        level[g] = std::max<uint32_t>(3, std::min<uint32_t>(ub[g], (cmax[g] + 1) / 2));
        pending = true;
      }
    const std::vector<uint64_t> nostop(G, 0);
    uint32_t iter = 0;
    while (pending) {
      std::vector<uint32_t> thr(G, 0);
      for (uint32_t g = 0; g < G; ++g) thr[g] = level[g] ? level[g] - 2 : 0;
      Sub s;
      DBuf sup;
      const auto t_a = std::chrono::steady_clock::now();
      survivors(c, s1, sup1.as<uint32_t>(), thr, false, s, sup);
      const auto t_b = std::chrono::steady_clock::now();
      std::vector<uint32_t> km;
      std::vector<uint64_t> cn;
      const uint32_t lv0 = st.levels, rd0 = st.rounds;
      tracked_peel(c, s, sup.as<uint32_t>(), level, nostop, km, cn);
      KT_LOG(c, "kt: wave phase 1 class %d pass %u: survivors %llu edges in %.2f ms, tracked peel %u levels %u "
                "rounds in %.2f ms\n",
             cls, iter++, (unsigned long long)s.m,
             std::chrono::duration<double, std::milli>(t_b - t_a).count(), st.levels - lv0, st.rounds - rd0,
             std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_b).count());
      pending = false;
      for (uint32_t g = 0; g < G; ++g) {
        if (!level[g]) continue;
        if (km[g] >= level[g]) {
          L[g] = km[g];
          C[g] = cn[g];
          level[g] = 0;
        } else if (level[g] == 3) {
          level[g] = 0;
        } else {
          level[g] = 3 + (level[g] - 3) / 2;
          pending = true;
        }
      }
    }
    st.ms_peel += tm.stop();
  }

  // Phase 2.
  std::vector<uint32_t> need2(G, 0), t0(G, 3);
  std::vector<uint64_t> stop(G, 0);
  bool any = false;
  for (uint32_t g = 0; g < G; ++g) {
    items[g]->kmax = 0;
    items[g]->count = 0;
    if (cmax[g] < 2) continue;
    if (single[g] || (L[g] >= 3 && L[g] == cmax[g] + 1)) {
      items[g]->kmax = L[g];
      items[g]->count = C[g];
      continue;
    }
    need2[g] = L[g] >= 3 ? L[g] - 1 : 2;
    if (L[g] >= 3) {
      t0[g] = L[g];
      stop[g] = C[g];
    }
    any = true;
  }
  if (!any) return;
  // Vertices of each graph's (need2[g])-core, for the class split.
  std::vector<unsigned long long> n2(G, 0);
  {
    tm.start();
    DBuf dneed(c, G * 4ull), dcnt(c, G * 8ull);
    copy_h2d(c, dneed.get(), need2.data(), G * 4ull);
    zero(c, dcnt.get(), dcnt.bytes());
    k_group_at_least<<<grid_for(nv, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        dcore.as<uint32_t>(), dgid.as<uint32_t>(), nv, dneed.as<uint32_t>(), dcnt.as<unsigned long long>());
    KT_LAUNCHED(c);
    copy_d2h(c, n2.data(), dcnt.get(), G * 8ull);
    st.ms_subgraph += tm.stop();
  }
  for (int cls = 0; cls < 2; ++cls) {
    std::vector<uint32_t> need(G, 0);
    bool any2 = false;
    for (uint32_t g = 0; g < G; ++g)
      if (need2[g] && (n2[g] <= dense_lim) == (cls == 0)) {
        need[g] = need2[g];
        any2 = true;
      }
    if (!any2) continue;
    tm.start();
    Sub s2;
    union_sub(c, U, dcore.as<uint32_t>(), dgid.as<uint32_t>(), G, need, s2);
    st.core_vertices += s2.n;
    st.core_edges += s2.m;
    st.ms_subgraph += tm.stop();
    tm.start();
    DBuf sup2(c, (s2.m ? s2.m : 1) * sizeof(uint32_t));
    std::vector<uint32_t> thr(G, 0);
    for (uint32_t g = 0; g < G; ++g) thr[g] = need[g] ? t0[g] - 2 : 0;
    // As in the single-graph search phase: each graph's peel starts at t0[g]
    // with no jump, so supports below t0[g] - 2 only need to be known as
    // "below" (the capped dense kernel, per-graph caps).
    const bool capped = c->opt.capped_support && s2.W;
    DBuf dthr;
    if (capped) {
      dthr.alloc(c, G * sizeof(uint32_t));
      copy_h2d(c, dthr.get(), thr.data(), G * sizeof(uint32_t));
    }
    edge_support(c, s2, sup2.as<uint32_t>(), 0, capped ? dthr.as<uint32_t>() : nullptr);
    // A union rebuilt from the survivors when they are fewer than half; else
    // the union is peeled in place, capped counts and all (those of the
    // survivors are exact, the others leave in the first round).
    Sub s3;
    DBuf sup3;
    const bool rebuilt = survivors(c, s2, sup2.as<uint32_t>(), thr, true, s3, sup3);
    st.ms_support += tm.stop();
    tm.start();
    const auto t_p = std::chrono::steady_clock::now();
    const uint32_t lv0 = st.levels, rd0 = st.rounds;
    std::vector<uint32_t> km;
    std::vector<uint64_t> cn;
    std::vector<uint32_t> t0c(G, 3);
    std::vector<uint64_t> stopc(G, 0);
    for (uint32_t g = 0; g < G; ++g)
      if (need[g]) {
        t0c[g] = t0[g];
        stopc[g] = stop[g];
      }
    if (rebuilt)
      tracked_peel(c, s3, sup3.as<uint32_t>(), t0c, stopc, km, cn);
    else
      tracked_peel(c, s2, sup2.as<uint32_t>(), t0c, stopc, km, cn);
    st.ms_peel += tm.stop();
    KT_LOG(c, "kt: wave phase 2 class %d: %llu edges (%s), tracked peel %u levels %u rounds in %.2f ms\n", cls,
           (unsigned long long)(rebuilt ? s3.m : s2.m), rebuilt ? "survivors" : "whole cores", st.levels - lv0,
           st.rounds - rd0, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_p).count());
    for (uint32_t g = 0; g < G; ++g) {
      if (!need[g]) continue;
      items[g]->kmax = km[g] >= 3 ? km[g] : 0;
      items[g]->count = km[g] >= 3 ? cn[g] : 0;
    }
  }
}

namespace {

// Adds a lane context's per-run figures into the batch's context.
void merge_lane_stats(kt_stats& a, const kt_stats& b) {
  a.ms_parse += b.ms_parse;
  a.ms_csr += b.ms_csr;
  a.ms_kcore += b.ms_kcore;
  a.ms_subgraph += b.ms_subgraph;
  a.ms_support += b.ms_support;
  a.ms_peel += b.ms_peel;
  a.ms_support_kernel += b.ms_support_kernel;
  a.ms_peel_kernel += b.ms_peel_kernel;
  a.core_vertices += b.core_vertices;
  a.core_edges += b.core_edges;
  a.predict_vertices += b.predict_vertices;
  a.predict_edges += b.predict_edges;
  a.levels += b.levels;
  a.rounds += b.rounds;
  a.support_bytes += b.support_bytes;
  a.peel_bytes += b.peel_bytes;
  a.support_kernel_bytes += b.support_kernel_bytes;
  a.support_row_words += b.support_row_words;
  a.peel_recount_bytes += b.peel_recount_bytes;
  a.support_launches += b.support_launches;
  a.peel_launches += b.peel_launches;
  a.peel_decrements += b.peel_decrements;
}

// The batch driver's second lane: a context of its own on the same device
// (own stream, device words, timers), created on first use.
Ctx* aux_lane(Ctx* c) {
  if (!c->aux) {
    kt_ctx* h = nullptr;
    const kt_status st = kt_init(c->device, c->budget, &h);
    if (st != KT_OK) throw Error(st, "batch: cannot create the second lane's context");
    c->aux = h;
    KT_CUDA(cudaSetDevice(c->device));
  }
  return &c->aux->c;
}

}  // namespace

void run_batch(Ctx* c, std::vector<BatchItem>& items, BatchRun& out) {
  // Waves: consecutive graphs while the estimated footprint fits
  // wave_budget_pct (50; measured best on the batched mix with one lane:
  // 236 graphs/s vs 228 at 70 % and 232 at 35 %) of the free budget, shared
  // by the lanes in flight (keys, sort buffers, CSR, k-core state ~ 48 B per
  // key and 40 B per vertex); the union stays below 2^28 vertices and 65536
  // graphs.  Graphs are taken in ascending size, so a wave's graphs are alike
  // and its per-graph structures (support bitmaps) are sized for graphs like
  // them.
  const int lanes = (int)std::min<int64_t>(std::max<int64_t>(1, c->opt.batch_lanes), 2);
  const uint64_t budget = (c->budget > c->in_use ? c->budget - c->in_use : 0) / 100 *
                          (uint64_t)std::min<int64_t>(std::max<int64_t>(1, c->opt.wave_budget_pct), 100) / lanes;
  std::vector<size_t> order(items.size());
  std::iota(order.begin(), order.end(), size_t(0));
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    return items[a].n != items[b].n ? items[a].n < items[b].n : items[a].nkeys < items[b].nkeys;
  });
  std::vector<std::vector<BatchItem*>> waves;
  size_t i = 0;
  while (i < items.size()) {
    std::vector<BatchItem*> wave;
    uint64_t bytes = 0, verts = 0;
    while (i < items.size()) {
      const BatchItem& it = items[order[i]];
      const uint64_t b = 48 * it.nkeys + 40 * it.n;
      if (!wave.empty() && (bytes + b > budget || verts + it.n >= (1ull << 28) || wave.size() >= 65535)) break;
      if (it.n >= (1ull << 28)) throw Error(KT_ERR_LIMIT, "batch: a graph with 2^28 or more vertex ids");
      wave.push_back(&items[order[i]]);
      bytes += b;
      verts += it.n;
      ++i;
    }
    waves.push_back(std::move(wave));
  }
  out.waves = (uint32_t)waves.size();

  auto one = [](Ctx* lc, const std::vector<BatchItem*>& wave, uint32_t no) {
    const kt_stats before = lc->stats;
    solve_wave(lc, wave);
    if (lc->opt.verbose) {
      const kt_stats& a = lc->stats;
      uint64_t keys = 0, verts_w = 0;
      for (const BatchItem* it : wave) keys += it->nkeys, verts_w += it->n;
      KT_LOG(lc,
             "kt: wave %u: %zu graphs, %llu keys, %llu vertex ids: input %.2f csr %.2f kcore %.2f subgraph %.2f "
             "support %.2f peel %.2f ms, %u levels, %u rounds\n",
             no, wave.size(), (unsigned long long)keys, (unsigned long long)verts_w, a.ms_parse - before.ms_parse,
             a.ms_csr - before.ms_csr, a.ms_kcore - before.ms_kcore, a.ms_subgraph - before.ms_subgraph,
             a.ms_support - before.ms_support, a.ms_peel - before.ms_peel, a.levels - before.levels,
             a.rounds - before.rounds);
    }
  };
  if (lanes == 1 || waves.size() < 2) {
    for (uint32_t w = 0; w < waves.size(); ++w) one(c, waves[w], w);
    return;
  }

  // Two lanes: each takes the next wave as soon as it is free, on its own
  // stream; cooperative launches of the two run one at a time.
  Ctx* a = aux_lane(c);
  std::lock_guard<std::recursive_mutex> alk(a->mu);
  a->opt = c->opt;
  a->opt.batch_lanes = 1;
  std::mutex coop;
  struct Unhook {
    Ctx* c;
    Ctx* a;
    ~Unhook() { c->coop_mu = a->coop_mu = nullptr; }
  } unhook{c, a};
  c->coop_mu = a->coop_mu = &coop;
  begin_solve_stats(a);
  const uint64_t a_launches = a->launches, a_h2d = a->h2d_bytes, a_d2h = a->d2h_bytes;
  // The second lane's stream starts after the work already on the first's.
  KT_CUDA(cudaEventRecord(c->ev[7], c->stream));
  KT_CUDA(cudaStreamWaitEvent(a->stream, c->ev[7], 0));
  reset_words(a);
  std::atomic<size_t> next{0};
  std::atomic<bool> failed{false};
  std::exception_ptr err[2];
  auto lane = [&](Ctx* lc, int li) {
    try {
      KT_CUDA(cudaSetDevice(lc->device));
      for (;;) {
        const size_t w = next.fetch_add(1);
        if (w >= waves.size() || failed.load()) break;
        one(lc, waves[w], (uint32_t)w);
      }
    } catch (...) {
      err[li] = std::current_exception();
      failed = true;
    }
  };
  std::thread t;
  try {
    t = std::thread(lane, a, 1);
  } catch (...) {
    lane(c, 0);  // no second thread: one lane does every wave
  }
  if (t.joinable()) {
    lane(c, 0);
    t.join();
  }
  // The first lane's stream continues after the second's work.
  try {
    KT_CUDA(cudaEventRecord(a->ev[7], a->stream));
    KT_CUDA(cudaStreamWaitEvent(c->stream, a->ev[7], 0));
    a->timer.resolve();
  } catch (...) {
    if (!err[0] && !err[1]) throw;
  }
  merge_lane_stats(c->stats, a->stats);
  c->launches += a->launches - a_launches;
  c->h2d_bytes += a->h2d_bytes - a_h2d;
  c->d2h_bytes += a->d2h_bytes - a_d2h;
  c->peak = std::max(c->peak, c->in_use + a->peak);
  if (err[0]) std::rethrow_exception(err[0]);
  if (err[1]) std::rethrow_exception(err[1]);
}

void load_mix_graph(Ctx* c, uint64_t index, uint64_t base_seed, Graph& g) {
  BatchItem it;
  it.from_mix(index, base_seed);
  std::vector<BatchItem*> one{&it};
  DBuf keys;
  uint64_t nkeys = 0;
  std::vector<uint64_t> vbase;
  KT_CUDA(cudaEventRecord(c->ev[4], c->stream));
  const uint64_t nv = wave_keys(c, one, keys, nkeys, vbase);
  KT_CUDA(cudaEventRecord(c->ev[5], c->stream));
  build_graph(c, keys.as<uint64_t>(), nkeys, nv, g);
  KT_CUDA(cudaEventRecord(c->ev[6], c->stream));
  c->stats.ms_parse = event_ms(c->ev[4], c->ev[5]);
  c->stats.ms_csr = event_ms(c->ev[5], c->ev[6]);
}

}  // namespace kt
