// k-core peeling state over a device graph (kcore.cu).
#pragma once
#include <vector>

#include "stages.h"

namespace kt {

struct KCore {
  const Graph* g = nullptr;
  uint64_t n = 0;
  DBuf deg;        // uint32[n]: alive degree of alive vertices
  DBuf rem;        // uint32[n]: kAlive, or the tag of the probe that removed it
  DBuf alive;      // uint32[n]: compact list of alive vertices
  DBuf front[2];   // frontiers
  DBuf big;        // rows handled by whole blocks
  DBuf cnt;        // counters
  uint64_t n_alive = 0;
  uint32_t cmax = 0;
  uint64_t rounds = 0;
  std::vector<uint32_t> levels;  // levels[tag] = k of that probe
  std::vector<uint32_t> succ;    // tags of probes that were kept

  void init(Ctx* c, const Graph& gr);
  void rebuild_alive(Ctx* c);
  void recount(Ctx* c);
  // Peels the alive set to its k-core; returns the vertices left.
  uint64_t probe(Ctx* c, uint32_t k);
  // Leaves the alive set at the maximum core; returns its k.
  uint32_t find_max_core(Ctx* c);
  // Leaves the alive set at the k-core (k <= cmax after find_max_core).
  void restore_core(Ctx* c, uint32_t k);
  void members(Ctx* c, uint8_t* dout);
  // Full decomposition (consumes the state).
  void core_numbers(Ctx* c, uint32_t* dcore);
};

}  // namespace kt
