// The solve driver: ingest (a, b), k-core (c), support (d), peel (e).
//
// Two phases, as in the reference (src/kc_gpu.cpp:336-341):
//   1. prediction: the maximum core's kmax-truss gives a lower bound L (a
//      subgraph's truss is a truss of the graph);
//   2. search: the (L-1)-core contains every L-truss, so the kmax-truss is
//      found by peeling that core from level L.
// Shortcuts, both exact: if L = cmax + 1 the upper bound (an edge's
// trussness is at most its ends' core number + 1) is met and phase 2 is
// skipped; if the L-truss found in phase 2 has exactly the edges of phase
// 1's L-truss, it is that same truss and nothing above it exists.
#include <algorithm>
#include <chrono>

#include "compact.cuh"
#include "solve.h"

namespace kt {
namespace {

__device__ __forceinline__ uint64_t lower_bound_u64(const uint64_t* a, uint64_t n, uint64_t x) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (a[mid] < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Scatters a per-edge value of the working graph back to the graph's
// canonical edge order.
__global__ void k_map_back(const uint64_t* __restrict__ ends, uint64_t m, const uint32_t* __restrict__ orig,
                           const uint64_t* __restrict__ gedges, uint64_t gm, const uint32_t* __restrict__ val,
                           uint32_t* __restrict__ out) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = ends[e];
    const uint32_t a = orig[(uint32_t)(k >> 32)], b = orig[(uint32_t)k];
    const uint64_t key = a < b ? (((uint64_t)a << 32) | b) : (((uint64_t)b << 32) | a);
    const uint64_t p = lower_bound_u64(gedges, gm, key);
    if (p < gm && gedges[p] == key) out[p] = val[e];
  }
}

// Vertices with at least `need` edges of support >= thr (warp per row).
__global__ void k_rows_at_least(uint32_t n, const uint64_t* __restrict__ off, const uint32_t* __restrict__ eid,
                                const uint32_t* __restrict__ sup, uint32_t thr, uint32_t need,
                                unsigned long long* __restrict__ out) {
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t x = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; x < n; x += warps) {
    uint32_t c = 0;
    for (uint64_t j = off[x] + lane_id(); j < off[x + 1]; j += 32) c += sup[eid[j]] >= thr;
    c = warp_sum(c);
    if (lane_id() == 0 && c >= need) atomicAdd(out, 1ULL);
  }
}

// Whether a g-truss can exist in s: each of its (at least g) vertices has at
// least g-1 edges of support >= g-2 within it, hence within s.
bool truss_possible(Ctx* c, const Sub& s, const uint32_t* sup, uint32_t g) {
  if (s.n == 0 || s.m == 0) return false;
  DBuf cnt(c, 8);
  zero(c, cnt.get(), 8);
  k_rows_at_least<<<grid_for((uint64_t)s.n * 32, 256, c->num_sms * 16), 256, 0, c->stream>>>(
      s.n, s.off.as<uint64_t>(), s.eid.as<uint32_t>(), sup, g - 2, g - 1, cnt.as<unsigned long long>());
  KT_LAUNCHED(c);
  return read_word<unsigned long long>(c, cnt.as<unsigned long long>()) >= g;
}

// Ends of the edges whose (capped) support reaches a threshold.
struct AtLeast {
  const uint32_t* sup;
  const uint64_t* ends;
  uint32_t thr;
  __device__ bool keep(uint64_t e) const { return sup[e] >= thr; }
  __device__ uint64_t value(uint64_t e) const { return ends[e]; }
};


}  // namespace

void begin_solve_stats(Ctx* c) {
  kt_stats& st = c->stats;
  st.ms_parse = st.ms_csr = st.ms_kcore = st.ms_subgraph = st.ms_support = st.ms_peel = st.ms_total = 0;
  st.ms_support_kernel = st.ms_peel_kernel = 0;
  st.support_bytes = st.peel_bytes = st.peel_decrements = 0;
  st.support_kernel_bytes = st.support_row_words = st.peel_recount_bytes = 0;
  st.core_vertices = st.core_edges = st.predict_vertices = st.predict_edges = 0;
  st.cmax = st.kmax_lower_bound = st.levels = st.rounds = 0;
}

void solve_graph(Ctx* c, const Graph& g, uint32_t* kmax, uint64_t* count) {
  struct Resolve {
    Ctx* c;
    ~Resolve() {
      try {
        c->timer.resolve();
      } catch (...) {
      }
    }
  } resolve{c};
  solve_graph_inner(c, g, kmax, count);
}

// kmax-truss of the maximum core s1 (exact supports sup1, core number
// cmax).  Levels g are tried from the support bound down, halving toward 3:
// the g-truss lies within the edges of support >= g-2, so while those are
// few, the g-truss and everything above it are found on a graph rebuilt from
// them alone.  When they are not few, the whole core is peeled, first
// trying level min(g, (cmax+1)/2) from a snapshot.
PeelResult predict_peel(Ctx* c, const Sub& s1, uint32_t* sup1, uint32_t cmax) {
  uint32_t g = support_bound(c, sup1, s1.m, cmax + 1);
  KT_LOG(c, "kt: predict on %u vertices, %llu edges, cmax %u: support bound %u\n", s1.n, (unsigned long long)s1.m,
         cmax, g);
  if (g < 3) return PeelResult{};  // no truss level 3: no triangle
  const uint32_t half = (cmax + 1) / 2;
  uint32_t levels = 0;
  uint64_t rounds = 0;
  for (bool tried = false; g > 3; tried = true, g = 3 + (g - 3) / 2) {
    DBuf keys(c, s1.m * sizeof(uint64_t));
    const uint64_t k = compact(c, s1.m, AtLeast{sup1, s1.ends.as<uint64_t>(), g - 2}, keys.as<uint64_t>());
    KT_LOG(c, "kt: predict level %u: %llu of %llu edges have support >= %u\n", g, (unsigned long long)k,
           (unsigned long long)s1.m, g - 2);
    if (k * 2 > s1.m) {
      if (!tried) g = std::min(g, half);
      break;
    }
    if (!truss_possible(c, s1, sup1, g)) {
      KT_LOG(c, "kt: predict level %u: fewer than %u vertices with %u such edges\n", g, g, g - 1);
      continue;
    }
    Sub s;
    build_sub_from_keys(c, keys.as<uint64_t>(), k, s1.n, s, true);
    keys.release();
    DBuf sup(c, (s.m ? s.m : 1) * sizeof(uint32_t));
    edge_support(c, s, sup.as<uint32_t>());
    PeelResult p = truss_peel(c, s, sup.as<uint32_t>(), g, 0, nullptr);
    levels += p.levels;
    rounds += p.rounds;
    if (p.kmax >= g) {
      p.levels = levels;
      p.rounds = rounds;
      return p;
    }
  }
  KT_LOG(c, "kt: predict peels the whole core, first level %u\n", g);
  PeelResult p = truss_peel(c, s1, sup1, 3, 0, nullptr, g);
  p.levels += levels;
  p.rounds += rounds;
  return p;
}

void solve_graph_inner(Ctx* c, const Graph& g, uint32_t* kmax, uint64_t* count) {
  kt_stats& st = c->stats;
  *kmax = 0;
  *count = 0;
  Timer tm(c);
  // Verbose: host time of each stage boundary since the solve began.
  const auto t_solve = std::chrono::steady_clock::now();
  auto mark = [&](const char* what) {
    KT_LOG(c, "kt: +%.2f ms %s\n",
           std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_solve).count(), what);
  };
  mark("solve start");
  tm.start();
  KCore kc;
  kc.init(c, g);
  const uint64_t n_edge_vertices = kc.n_alive;  // vertices with an edge
  const uint32_t cmax = kc.find_max_core(c);
  st.cmax = cmax;
  st.ms_kcore += tm.stop();
  mark("maximum core found");
  if (g.m == 0 || cmax < 2) return;  // a triangle needs three vertices of degree >= 2

  // One phase when the maximum core is a large part of the graph (the
  // search core would contain it anyway): the truss levels of the 2-core,
  // tried from its support bound as in the prediction phase.
  if (!c->opt.predict || kc.n_alive * 4 >= n_edge_vertices) {
    tm.start();
    kc.restore_core(c, 2);
    st.ms_kcore += tm.stop();
    tm.start();
    Sub s;
    build_sub(c, g, kc, s);
    st.core_vertices = s.n;
    st.core_edges = s.m;
    st.ms_subgraph += tm.stop();
    tm.start();
    DBuf sup(c, (s.m ? s.m : 1) * sizeof(uint32_t));
    edge_support(c, s, sup.as<uint32_t>());
    st.ms_support += tm.stop();
    tm.start();
    const PeelResult p = predict_peel(c, s, sup.as<uint32_t>(), cmax);
    st.ms_peel += tm.stop();
    st.levels += p.levels;
    st.rounds += (uint32_t)p.rounds;
    *kmax = p.kmax;
    *count = p.count;
    st.kmax_lower_bound = p.kmax;
    return;
  }

  uint32_t L = 0;
  uint64_t C = 0;
  if (c->opt.predict) {
    tm.start();
    Sub s1;
    build_sub(c, g, kc, s1);
    st.predict_vertices = s1.n;
    st.predict_edges = s1.m;
    st.ms_subgraph += tm.stop();
    mark("prediction subgraph built");
    tm.start();
    DBuf sup1(c, (s1.m ? s1.m : 1) * sizeof(uint32_t));
    edge_support(c, s1, sup1.as<uint32_t>());
    st.ms_support += tm.stop();
    mark("prediction support counted");
    tm.start();
    const PeelResult p1 = predict_peel(c, s1, sup1.as<uint32_t>(), cmax);
    st.ms_peel += tm.stop();
    mark("prediction peeled");
    st.levels += p1.levels;
    st.rounds += (uint32_t)p1.rounds;
    L = p1.kmax;
    C = p1.count;
    if (L >= 3 && L == cmax + 1) {
      *kmax = L;
      *count = C;
      st.kmax_lower_bound = L;
      return;
    }
  }
  st.kmax_lower_bound = L;
  tm.start();
  kc.restore_core(c, L >= 3 ? L - 1 : 2);
  st.ms_kcore += tm.stop();
  mark("search core restored");
  tm.start();
  Sub s2;
  build_sub(c, g, kc, s2);
  st.core_vertices = s2.n;
  st.core_edges = s2.m;
  st.ms_subgraph += tm.stop();
  mark("search subgraph built");
  tm.start();
  DBuf sup2(c, (s2.m ? s2.m : 1) * sizeof(uint32_t));
  // The search peel starts at level max(L, 3) with no jump, so supports
  // below its threshold only need to be known as "below".
  const uint32_t t2 = std::max<uint32_t>(L, 3);
  const bool capped = c->opt.capped_support && s2.W;
  edge_support(c, s2, sup2.as<uint32_t>(), capped ? t2 - 2 : 0);
  // Edges below the first threshold leave in the first round: when they are
  // most of the graph, continue on the rest (the L-truss of the survivors is
  // the L-truss of the core) instead of clearing them one by one.  When they
  // are not, the core is peeled in place even with capped counts: those of
  // the edges at or above the threshold are exact, and the others leave in
  // the first round.
  Sub s3;
  DBuf sup3;
  const Sub* sp = &s2;
  uint32_t* supp = sup2.as<uint32_t>();
  if (t2 > 3 && s2.m) {
    DBuf keys(c, s2.m * sizeof(uint64_t));
    const uint64_t k = compact(c, s2.m, AtLeast{sup2.as<uint32_t>(), s2.ends.as<uint64_t>(), t2 - 2},
                               keys.as<uint64_t>());
    KT_LOG(c, "kt: search level %u: %llu of %llu edges have support >= %u\n", t2, (unsigned long long)k,
           (unsigned long long)s2.m, t2 - 2);
    if (k * 2 < s2.m) {
      build_sub_from_keys(c, keys.as<uint64_t>(), k, s2.n, s3, true);
      sup3 = DBuf(c, (s3.m ? s3.m : 1) * sizeof(uint32_t));
      edge_support(c, s3, sup3.as<uint32_t>());
      sp = &s3;
      supp = sup3.as<uint32_t>();
    }
  }
  st.ms_support += tm.stop();
  mark("search support counted");
  tm.start();
  const PeelResult p2 = truss_peel(c, *sp, supp, t2, L >= 3 ? C : 0, nullptr);
  st.ms_peel += tm.stop();
  mark("search peeled");
  st.levels += p2.levels;
  st.rounds += (uint32_t)p2.rounds;
  *kmax = p2.kmax;
  *count = p2.count;
}

// Resolves the context's kernel timers when a stage-output call ends.
struct ResolveTimers {
  Ctx* c;
  ~ResolveTimers() {
    try {
      c->timer.resolve();
    } catch (...) {
    }
  }
};

void graph_support(Ctx* c, const Graph& g, uint32_t* dout) {
  begin_solve_stats(c);
  ResolveTimers resolve{c};
  Sub s;
  build_sub_all(c, g, s);
  DBuf sup(c, (s.m ? s.m : 1) * sizeof(uint32_t));
  edge_support(c, s, sup.as<uint32_t>());
  if (s.m) {
    k_map_back<<<grid_for(s.m, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        s.ends.as<uint64_t>(), s.m, s.orig.as<uint32_t>(), g.edges.as<uint64_t>(), g.m, sup.as<uint32_t>(), dout);
    KT_LAUNCHED(c);
  }
}

void graph_trussness(Ctx* c, const Graph& g, uint32_t* dout) {
  begin_solve_stats(c);
  ResolveTimers resolve{c};
  Sub s;
  build_sub_all(c, g, s);
  DBuf sup(c, (s.m ? s.m : 1) * sizeof(uint32_t));
  DBuf tr(c, (s.m ? s.m : 1) * sizeof(uint32_t));
  edge_support(c, s, sup.as<uint32_t>());
  truss_peel(c, s, sup.as<uint32_t>(), 3, 0, tr.as<uint32_t>());
  if (s.m) {
    k_map_back<<<grid_for(s.m, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        s.ends.as<uint64_t>(), s.m, s.orig.as<uint32_t>(), g.edges.as<uint64_t>(), g.m, tr.as<uint32_t>(), dout);
    KT_LAUNCHED(c);
  }
}

}  // namespace kt
