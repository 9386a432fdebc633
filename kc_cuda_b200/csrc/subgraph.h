// The working graph of the truss stages: an induced subgraph relabelled by
// ascending (degree, id), with sorted rows and an id per undirected edge.
#pragma once
#include <vector>

#include "kcore.h"
#include "stages.h"

namespace kt {

struct Sub {
  uint32_t n = 0;   // vertices (new ids 0..n-1, ascending degree)
  uint64_t m = 0;   // undirected edges (ids 0..m-1, sorted by (u, v), u < v)
  DBuf orig;        // uint32[n]   original id of each new id
  DBuf off;         // uint64[n+1] row offsets
  DBuf adj;         // uint32[2m]  neighbours, ascending per row
  DBuf eid;         // uint32[2m]  edge id of each entry
  DBuf up;          // uint64[n]   first entry of each row with neighbour > row
  DBuf ends;        // uint64[m]   u << 32 | v of each edge (new ids, u < v)
  uint32_t max_deg = 0;
  // Dense mode: alive adjacency as bitsets, row u = words [u*W, (u+1)*W);
  // for a grouped union, per-graph rows: row u = words [roff[u], roff[u] +
  // rw[u]) over its graph's vertices from vbase[u] (W = the longest row).
  DBuf bits;
  uint32_t W = 0;   // 0 = not built
  DBuf roff, rw;
  uint64_t bit_words = 0;  // words of all rows
  // Dense mode, when the budget allows: the rows as built (never cleared) and
  // the set bits before each of their words, so the position of neighbour v
  // in row u's sorted adjacency is a popcount away (peel intersections).
  DBuf sbits, spre;
  // Dense mode: edge ids in tile order (u >> tb, v >> tb, u, v), so that the
  // rows read by concurrently processed edges stay within two vertex blocks
  // whose bitsets fit in L2 together.
  DBuf order;
  uint32_t tile_bits = 0;
  // Batched unions of many graphs: vertices are grouped by graph (new ids of
  // one graph are contiguous), vgid[v] = its graph, vbase[v] = first new id
  // of its graph, max_group = most vertices of one graph.
  DBuf vgid, vbase;
  uint32_t max_group = 0;
  std::vector<uint32_t> group_n;  // vertices of each graph (host)
};

// Builds the subgraph induced by the k-core state's alive vertices.
void build_sub(Ctx* c, const Graph& g, const KCore& kc, Sub& s);
// Builds the whole graph as a subgraph (every vertex of degree > 0).
void build_sub_all(Ctx* c, const Graph& g, Sub& s);
// Subgraph of a list of alive vertices of a disjoint union of graphs,
// grouped by graph: group_of[v] (< 65536) is the graph of vertex v of g
// (g.n < 2^28); within a graph, ascending (degree, id).
void build_sub_grouped(Ctx* c, const Graph& g, const uint32_t* alive, uint64_t na, const uint32_t* deg,
                       const uint32_t* rem, const uint32_t* group_of, uint32_t ngroups, Sub& s);
// The same from edge keys u << 32 | v (ids below n_ids, group_of indexed by
// them; keys consumed).
void build_sub_grouped_from_keys(Ctx* c, uint64_t* keys, uint64_t m, uint32_t n_ids, const uint32_t* group_of,
                                 uint32_t ngroups, Sub& s, bool sorted = false);

// Per-graph bookkeeping of a batched peel: every graph climbs its own
// levels; after each of its levels a graph with alive edges records (its
// minimum support + 2, its alive edges).
struct GraphTrack {
  const uint32_t* vgid;  // graph of each vertex of the working graph
  uint32_t ngroups;
  uint32_t* kmax;        // device [ngroups], last recorded level (0 = none)
  uint64_t* count;       // device [ngroups]
  const uint32_t* t0 = nullptr;    // device [ngroups]: first level (null/0: the peel's t0)
  const uint64_t* stop = nullptr;  // device [ngroups]: early-stop edge count (null/0: none)
};

// support.cu: sup[e] = triangles through edge e (all edges of s).  Uses the
// bitsets when they are built.  cap > 0 (dense mode only): an edge whose
// support is below cap may get any value below cap -- enough for a peel whose
// first level removes everything below cap.  gcap (device, per graph of a
// grouped union; dense mode only): the same with graph g's cap gcap[g].
void edge_support(Ctx* c, const Sub& s, uint32_t* sup, uint32_t cap = 0, const uint32_t* gcap = nullptr);
// Upper bound on the largest non-empty truss level, from exact supports: the
// largest t <= cap with at least t(t-1)/2 edges of support >= t-2 (a
// non-empty t-truss has t or more vertices, each of degree >= t-1 in it, and
// each of its edges has support >= t-2).  0 when no t >= 3 qualifies.
uint32_t support_bound(Ctx* c, const uint32_t* sup, uint64_t m, uint32_t cap);
// Builds s.bits when the subgraph qualifies for dense mode; returns whether.
// Every build_sub* call runs it (before the lower entries' edge ids).
bool build_bits(Ctx* c, Sub& s);

// peel.cu
struct PeelResult {
  uint32_t kmax = 0;
  uint64_t count = 0;
  uint32_t levels = 0;
  uint64_t rounds = 0;
  bool stopped_early = false;
};
// Peels from truss level t0 upwards until no edge is left.  stop_count: if
// nonzero and the t0-truss has exactly that many edges, stop there.
// truss (optional, device uint32[m]) receives each edge's trussness.
// The subgraph of edge keys (u << 32 | v, ids below n_ids; consumed), with
// bitsets when it qualifies.
// sorted: the keys are canonical, ascending and distinct (a working graph's
// edges taken in edge-id order), so the graph build skips its sort.
void build_sub_from_keys(Ctx* c, uint64_t* keys, uint64_t m, uint32_t n_ids, Sub& out, bool sorted = false);
// guess (> t0, 0 = none): first level to try, undone and halved toward t0 if
// it empties the graph (only without truss output).
PeelResult truss_peel(Ctx* c, const Sub& s, uint32_t* sup, uint32_t t0, uint64_t stop_count, uint32_t* truss,
                      uint32_t guess = 0, const GraphTrack* track = nullptr);

}  // namespace kt
