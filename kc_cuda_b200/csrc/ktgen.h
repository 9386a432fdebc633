// Seeded synthetic graph generator (host side), C ABI.
//
// Produces the undirected simple graph of a spec (R-MAT, Erdos-Renyi or
// Chung-Lu draws, plus planted cliques and an optional dense block), and
// writes it as the TSV edge list the kmax-truss solvers read: every edge in
// both directions, rows grouped by ascending second column.  The random
// conventions live in ktgen_core.h.
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { KTG_RMAT = 0, KTG_ER = 1, KTG_CHUNGLU = 2 };

typedef struct {
  uint32_t kind;         // KTG_RMAT / KTG_ER / KTG_CHUNGLU
  uint32_t scale;        // R-MAT: draws use 2^scale row/column ids
  uint64_t n;            // vertex count (R-MAT: ids >= n are rejected; 0 = 2^scale)
  uint64_t draws;        // edge draws before cleaning
  uint64_t seed;
  uint32_t a_ppm, b_ppm, c_ppm;  // R-MAT quadrant probabilities, parts per million
  uint32_t n_cliques;
  uint32_t clique_sizes[8];
  // Chung-Lu: expected degrees w_i = min(max_w, w_min * U_i^(-1/(gamma-1)))
  double cl_gamma;
  double cl_w_min;
  double cl_w_max;
  // Dense block planted on block_size random vertices, pair probability block_p_ppm
  uint32_t block_size;
  uint32_t block_p_ppm;
} ktg_spec;

typedef struct ktg_graph ktg_graph;

// Builds the cleaned graph (self-loops and repeated edges removed).
// Returns NULL on a bad spec or allocation failure.
ktg_graph* ktg_make(const ktg_spec* spec, int threads);
void ktg_free(ktg_graph* g);
uint64_t ktg_num_vertices(const ktg_graph* g);  // max id + 1 over all ids that occur
uint64_t ktg_num_edges(const ktg_graph* g);     // undirected edges
// Sorted canonical keys u << 32 | v with u < v, ktg_num_edges of them.
const uint64_t* ktg_edges(const ktg_graph* g);

// TSV in the solvers' input form.  mode 0: both directions, grouped by the
// second column ascending, first column ascending inside a group.
// mode 1 ("messy"): shuffled rows, edges in one or both directions, repeated
// rows, self-loops, CRLF/space/comma separators -- the same cleaned graph.
uint64_t ktg_tsv_size(const ktg_graph* g, int mode, uint64_t mess_seed);
// Fills buf (ktg_tsv_size bytes).  Returns bytes written.
uint64_t ktg_tsv_fill(const ktg_graph* g, int mode, uint64_t mess_seed, char* buf, int threads);
// Writes the TSV to a file.  Returns 0 on success.
int ktg_tsv_write(const ktg_graph* g, int mode, uint64_t mess_seed, const char* path, int threads);

// Raw draws (before cleaning) as x << 32 | y, for the device generator's
// parity check.  out must hold spec->draws entries.
int ktg_raw_draws(const ktg_spec* spec, uint64_t first, uint64_t count, uint64_t* out);
// Planted clique / dense block vertices (Floyd's sampling).  out holds size ids.
int ktg_sample_vertices(uint64_t seed, uint64_t stream, uint64_t n, uint32_t size, uint32_t* out);

// Spec of graph `index` of the batched mix: n = floor(1000 * 10^(3U)) (log-
// uniform over [1e3, 1e6]); R-MAT (a/b/c/d = .57/.19/.19/.05, scale =
// ceil(log2 n), ids >= n rejected) or Erdos-Renyi with equal chance; edge
// factor uniform over 4..64 (draws = ef * n); one clique of size uniform over
// 5..60; graph seed = base_seed << 20 | index.
int ktg_mix_spec(uint64_t index, uint64_t base_seed, ktg_spec* out);

#ifdef __cplusplus
}
#endif
