// k-core peeling state over a device graph (kcore.cu).
#pragma once
#include <vector>

#include "stages.h"

namespace kt {

struct KCore {
  const Graph* base = nullptr;  // the input graph
  Graph local;                  // compacted core (valid when compacted)
  DBuf idmap;                   // uint32[local.n]: local id -> base id
  bool compacted = false;
  uint32_t local_level = 0;     // local holds the local_level-core of base
  uint64_t n = 0;               // vertices of the current graph
  DBuf deg;        // uint32[n]: alive degree of alive vertices
  DBuf rem;        // uint32[n]: kAlive, or the tag of the probe that removed it
  DBuf alive;      // uint32[n]: compact list of alive vertices (ascending)
  DBuf front[2];   // frontiers
  DBuf big;        // rows handled by whole blocks
  DBuf cnt;        // counters
  uint64_t n_alive = 0;
  uint32_t cmax = 0;
  uint64_t rounds = 0;
  uint64_t probes = 0;
  unsigned coop_grid = 0;
  std::vector<uint32_t> levels;  // levels[tag] = k of that probe
  std::vector<uint32_t> succ;    // tags of probes that were kept
  // Earlier compactions (shallowest first), kept so that a restore below
  // the current compaction's level starts from the deepest one at or below
  // it instead of from the input graph.
  struct Saved {
    Graph local;
    DBuf idmap;
    uint32_t level = 0;
  };
  std::vector<Saved> saved;

  const Graph& cur() const { return compacted ? local : *base; }
  const uint32_t* map() const { return compacted ? idmap.as<uint32_t>() : nullptr; }

  void init(Ctx* c, const Graph& gr);
  void rebuild_alive(Ctx* c);
  void recount(Ctx* c);
  // Peels the alive set to its k-core; returns the vertices left.  may_stop:
  // the peel may stop once fewer than k+1 vertices can remain, returning 0
  // with the state partial (the caller then undoes the probe).
  uint64_t probe(Ctx* c, uint32_t k, bool may_stop = false);
  // Leaves the alive set at the maximum core; returns its k.
  uint32_t find_max_core(Ctx* c);
  // Leaves the alive set at the k-core (k <= cmax after find_max_core).
  void restore_core(Ctx* c, uint32_t k);
  // member[v] (base ids) = v is alive.
  void members(Ctx* c, uint8_t* dout);
  // Full decomposition (consumes the state; never compacts).
  void core_numbers(Ctx* c, uint32_t* dcore);
  // The same in one cooperative launch (levels stepped on the device).
  void core_numbers_persistent(Ctx* c, uint32_t* dcore);

 private:
  void reset_state(Ctx* c, const Graph& gr);
  void compact_to_alive(Ctx* c, uint32_t level);
};

}  // namespace kt
