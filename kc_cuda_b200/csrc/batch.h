// Batched solving (batch.cu).
#pragma once
#include <vector>

#include "stages.h"

namespace kt {

// One graph of a batch: generated on the device from a mix spec, or host
// records x << 32 | y.
struct BatchItem {
  bool generated = false;
  uint32_t kind = 0, scale = 0;
  uint64_t n = 0;      // vertex id range
  uint64_t draws = 0;  // generated draws
  uint64_t seed = 0;
  uint64_t nkeys = 0;  // draws + extra
  std::vector<uint64_t> extra;  // clique keys (generated) or the records (host)
  uint32_t kmax = 0;
  uint64_t count = 0;
  void from_mix(uint64_t index, uint64_t base_seed);
  void from_pairs(const uint64_t* xy, uint64_t count);
};

struct BatchRun {
  uint32_t waves = 0;
};

void solve_wave(Ctx* c, const std::vector<BatchItem*>& items);
void run_batch(Ctx* c, std::vector<BatchItem>& items, BatchRun& out);
// Graph `index` of the batched mix, generated on the device.
void load_mix_graph(Ctx* c, uint64_t index, uint64_t base_seed, Graph& g);

}  // namespace kt
