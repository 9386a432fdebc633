// Solve driver and per-graph stage outputs (solve.cu).
#pragma once
#include "subgraph.h"

namespace kt {

// Stream-ordered stage timer: stop() waits for the stage and returns its ms.
struct Timer {
  Ctx* c;
  cudaEvent_t a, b;
  explicit Timer(Ctx* cx) : c(cx) {
    KT_CUDA(cudaEventCreate(&a));
    KT_CUDA(cudaEventCreate(&b));
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
  void start() { KT_CUDA(cudaEventRecord(a, c->stream)); }
  double stop() {
    KT_CUDA(cudaEventRecord(b, c->stream));
    KT_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    KT_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
  }
};

// Clears the per-solve statistics.
void begin_solve_stats(Ctx* c);
void solve_graph(Ctx* c, const Graph& g, uint32_t* kmax, uint64_t* count);
void solve_graph_inner(Ctx* c, const Graph& g, uint32_t* kmax, uint64_t* count);
void graph_support(Ctx* c, const Graph& g, uint32_t* dout);
void graph_trussness(Ctx* c, const Graph& g, uint32_t* dout);

// ingest (api.cu): host TSV bytes / records -> Graph.
void load_tsv(Ctx* c, const char* bytes, uint64_t len, Graph& g);
// Device-resident bytes (padded to parse_padded_bytes(len)) -> Graph.
void graph_from_device_bytes(Ctx* c, const uint8_t* dbuf, uint64_t len, Graph& g);
void load_pairs(Ctx* c, const uint64_t* xy, uint64_t count, Graph& g);

}  // namespace kt
