/* kt.h -- C ABI of the B200 kmax-truss solver (libkt.so).
 *
 * The solver answers the question of caixiaofan/KC_CUDA: for an undirected
 * graph given as a TSV edge list, the largest k with a non-empty k-truss and
 * the number of edges in that k-truss (a k-truss is the largest subgraph in
 * which every edge lies in at least k-2 triangles of the subgraph).  A graph
 * without triangles answers kmax = 0, 0 edges, as the reference does
 * (src/kc_cpu.cpp:703-710).
 *
 * The reference exposes its GPU path as C++ functions over host arrays
 * (src/kc_gpu.h:48-69) driven by a `main -f <path>` (src/kc_gpu.cpp:209-347).
 * This header replaces them with opaque handles and status codes; each entry
 * point names the reference function(s) it stands in for.  All pointers in
 * this header are HOST pointers unless the name says `_device`.  Calls on one
 * context are serialised internally; separate contexts may be used from
 * separate threads.
 */
#ifndef KT_H
#define KT_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum kt_status {
  KT_OK = 0,
  KT_ERR_INVALID = 1,  /* bad argument or handle */
  KT_ERR_CUDA = 2,     /* CUDA runtime error; text in kt_last_error */
  KT_ERR_NOMEM = 3,    /* device memory or the context's HBM budget exhausted */
  KT_ERR_PARSE = 4,    /* a TSV line with a single number; kt_last_error names it */
  KT_ERR_IO = 5,       /* open / mmap / read failure */
  KT_ERR_TIMEOUT = 6,  /* a bounded device wait gave up (kernel returned early) */
  KT_ERR_LIMIT = 7,    /* input beyond a documented size limit */
  KT_ERR_NODEV = 8,    /* no usable CUDA device */
  KT_ERR_BUSY = 9,     /* serving: admission refused, retry later */
} kt_status;

typedef struct kt_ctx kt_ctx;
typedef struct kt_graph kt_graph;

/* Creates a context on `device` with its own stream.  hbm_budget_bytes caps
 * the device memory the context may hold (0 = 90% of free memory).
 * Replaces initGPU (src/kc.cu:30-53, src/kc_gpu.h:48). */
kt_status kt_init(int device, uint64_t hbm_budget_bytes, kt_ctx** out);
void kt_destroy(kt_ctx* ctx);
/* Text of the last error on this context ("" if none): a copy owned by the
 * calling thread, valid until that thread's next kt_last_error call.  It does
 * not wait for a serving wave that holds the context. */
const char* kt_last_error(const kt_ctx* ctx);
const char* kt_status_string(kt_status s);

/* Tunables by name; KT_ERR_INVALID for an unknown name or a value out of
 * range (every option is >= 0).
 *   predict (1)                 prediction phase (truss of the maximum core)
 *   persistent (1)              peel / k-core rounds in one cooperative launch
 *   support_bitmap_max_n (2^20) vertex-bitmap support up to this many vertices
 *   dense_max_n (65536)         adjacency bitsets up to this many vertices
 *   dense_min_fill (32)         bitsets when avg degree * this >= words per row
 *   recount_gamma (16)          recount round when frontier * thr * gamma > alive * words
 *   capped_support (1)          search phase: abandon supports below the threshold
 *   timeout_ms (20000)          bound on every device-side wait, 0..3600000; 0 makes
 *                               every bounded wait give up at once, so a solve
 *                               returns KT_ERR_TIMEOUT (a test of the error path)
 *   parse_pipeline_mb (256)     host->device chunk of file ingest, and of host TSV
 *                               bytes parsed chunk by chunk as they land (inputs of
 *                               three chunks or more)
 *   record_kernel_times (0)     events around support / peel kernels
 *   debug_checks (0)            extra host-side consistency checks
 *   verbose (0)                 stage decisions on stderr
 *   pool_reserve_mb (0)         setting it grows the device memory pool by that
 *                               much at once (allocations mid-solve then reuse it)
 *   kcore_big_row (512)         k-core rounds deal longer rows to all warps in
 *                               windows (256 entries in the maximum-core probes,
 *                               32 in the full decomposition)
 *   peel_search_ratio (16)      peel: per-lane binary search when one row is this
 *                               many times longer than the other
 *   dense_tile_mb (48)          dense support: bitset rows of two tile blocks fit
 *                               in this many MB (L2 reuse)
 *   kcore_blocks_per_sm (0)     core decomposition: resident blocks per SM of its
 *                               one cooperative launch (0 = as many as fit)
 *   kcore_window (32)           core decomposition: levels per pass over the whole
 *                               alive list (passes between read window candidates)
 *   peel_bitset (1)             peel: intersect dense rows as bitsets (AND of two
 *                               rows) when the rows are shorter than the lists
 *   wave_budget_pct (50)        batch: a wave's estimated device footprint stays
 *                               within this % of the free budget
 *   kcore_compact (4)           maximum-core search: copy the core into a compact
 *                               graph once it holds < 1/this of the current
 *                               graph's edges (0 = never)
 *   peel_split (16)             peel: a round whose frontier edges x 8-word row
 *                               chunks <= this x warps deals (edge, chunk) units
 *                               to warps instead of edges (0 = off)
 *   serve_lanes (2)             serving: waves in flight at once, 1..4
 *   serve_small_mb (128)        serving with two or more lanes: the last lane admits
 *                               only requests whose estimated footprint is at most
 *                               this many MB, the other lanes any (0: every lane any)
 *   serve_small_coop (0)        the small lane's k-core and peel rounds: 0 = host-
 *                               stepped (no cooperative launch, so it never waits for
 *                               another lane's), 1 = cooperative launches taking turns
 *                               with the other lanes'
 *   serve_partition (0)         1: the other lanes admit only requests above
 *                               serve_small_mb (0: any request)
 *   batch_lanes (2)             batch: waves in flight at once, 1..2
 *   support_rows (2)            exact dense support: edges sharing row u counted
 *                               together per shared-memory read of it (1, 2 or 4)
 *   peel_bisect_after (16)      peel: truss levels climbed one at a time before the
 *                               rest is found by bisection (0 = never) ...
 *   peel_bisect_gap (16)        ... when the support bound of the alive edges is at
 *                               least this many levels above (>= 1)
 *   coop_occupancy_pct (100)    cooperative launches use this % of the blocks the
 *                               device can hold at once (1..100) */
kt_status kt_set_option(kt_ctx* ctx, const char* name, int64_t value);
kt_status kt_get_option(const kt_ctx* ctx, const char* name, int64_t* value);

/* ---------------------------------------------------------------- ingest */

/* Parses TSV bytes on the device and builds the cleaned graph (self-loops
 * dropped, repeated and reverse-repeated edges merged).  The record grammar is
 * the reference's (src/kc_gpu.cpp:243-306): a byte is a digit when, as a
 * signed char, it is >= '0'; a line's first two digit runs are x and y; other
 * lines are skipped; a line with one digit run is KT_ERR_PARSE.  Vertex ids
 * (here and in kt_load_pairs) must be below 2^32 - 1, else KT_ERR_LIMIT.
 * Replaces the host parse and init_graph (src/kc_gpu.cpp:221-322, 38-65). */
kt_status kt_load_tsv(kt_ctx* ctx, const char* bytes, uint64_t len, kt_graph** out);
/* As kt_load_tsv, from a file (mmap, pipelined host-to-device copies).
 * Replaces MapFile + vmtouch + parse (src/mapfile.hpp:35-84,
 * src/kc_gpu.cpp:221-240). */
kt_status kt_load_tsv_file(kt_ctx* ctx, const char* path, kt_graph** out);
/* Builds the cleaned graph from records x << 32 | y (host array). */
kt_status kt_load_pairs(kt_ctx* ctx, const uint64_t* xy, uint64_t count, kt_graph** out);
kt_status kt_graph_info(const kt_graph* g, uint64_t* num_vertices, uint64_t* num_edges);
/* Sorted canonical edges u << 32 | v (u < v), num_edges of them. */
kt_status kt_graph_edges(kt_ctx* ctx, const kt_graph* g, uint64_t* keys_out);
void kt_graph_free(kt_ctx* ctx, kt_graph* g);

/* ----------------------------------------------------------------- solve */

/* kmax and the kmax-truss edge count.  Two phases as in the reference: a
 * lower bound from the truss of the maximum core, then the search on the
 * (bound-1)-core.  Replaces kmax_truss (src/kc_gpu.cpp:129-208, called twice
 * at src/kc_gpu.cpp:336,340) with kmax_core_gpu, tricount_direct,
 * kmax_truss_GPU and reconstruct_Graph (src/kc.cu:770, 584, 1140, 1059). */
kt_status kt_solve(kt_ctx* ctx, kt_graph* g, uint32_t* kmax, uint64_t* edges);
/* kt_load_tsv + kt_solve + kt_graph_free in one call (the `-f` path). */
kt_status kt_solve_tsv(kt_ctx* ctx, const char* bytes, uint64_t len, uint32_t* kmax, uint64_t* edges);

/* TSV bytes held in device memory (for callers that keep inputs resident
 * in HBM, and for timing the solve without the host-to-device copy). */
typedef struct kt_tsv kt_tsv;
/* Copies host TSV bytes into device memory owned by the context. */
kt_status kt_tsv_stage(kt_ctx* ctx, const char* bytes, uint64_t len, kt_tsv** out);
/* Parse + clean + solve from staged bytes (the device-resident form of
 * kt_solve_tsv). */
kt_status kt_solve_staged(kt_ctx* ctx, const kt_tsv* tsv, uint32_t* kmax, uint64_t* edges);
void kt_tsv_free(kt_ctx* ctx, kt_tsv* tsv);

/* ----------------------------------------------------------------- batch */

/* Many graphs solved together (no counterpart in the reference, which
 * solves one graph per process).  Graphs are packed into waves that fit the
 * context's HBM budget; each wave is one disjoint union sent once through the
 * CSR build, the core decomposition, and a shared support count and peel in
 * which every graph keeps its own answer. */
typedef struct kt_batch kt_batch;
kt_status kt_batch_create(kt_ctx* ctx, kt_batch** out);
/* Adds a graph given as records x << 32 | y (copied); *graph_id = its index. */
kt_status kt_batch_add_pairs(kt_batch* b, const uint64_t* xy, uint64_t count, uint32_t* graph_id);
/* Adds graphs first_index .. first_index+count-1 of the batched mix
 * (generated on the device at run time from their seeds). */
kt_status kt_batch_add_mix(kt_batch* b, uint64_t first_index, uint64_t count, uint64_t base_seed);
kt_status kt_batch_size(const kt_batch* b, uint64_t* graphs, uint64_t* edge_records);
/* Solves every graph of the batch.  Waves run on batch_lanes (option, 1 or 2,
 * default 2) lanes: the second lane is a context of its own on the same
 * device (own stream), created on first use and kept with this context; each
 * lane takes the next wave as soon as it is free.  kt_get_stats: ms_total =
 * the whole run on the device (generation and upload of the graphs' edges
 * included), ms_parse and the other stage times = time spent in each stage,
 * summed over the lanes, batch_waves = waves used. */
kt_status kt_batch_run(kt_batch* b);
/* kmax and kmax-truss edge count of every graph, in graph-id order. */
kt_status kt_batch_results(const kt_batch* b, uint32_t* kmax, uint64_t* edges);
void kt_batch_free(kt_batch* b);
/* Graph `index` of the batched mix, generated on the device (the per-graph
 * path's input, identical to the batch's); kt_get_stats: ms_parse = the
 * generation, ms_csr = the CSR build. */
kt_status kt_load_mix_graph(kt_ctx* ctx, uint64_t index, uint64_t base_seed, kt_graph** out);

/* ---------------------------------------------------------------- tuning */

/* Autotuner of the kernels' bin and tile thresholds (no counterpart in the
 * reference, whose thresholds are compile-time constants): the options
 * recount_gamma, dense_min_fill, dense_max_n, support_bitmap_max_n,
 * kcore_big_row, peel_search_ratio, dense_tile_mb, kcore_blocks_per_sm,
 * kcore_window, peel_bitset and peel_split.  Solves the graphs of
 * `sample` repeatedly, one candidate value at a time (coordinate descent from
 * the context's current settings, up to `passes` sweeps, device time by CUDA
 * events, a 2% margin against noise), checks that every candidate leaves
 * every answer unchanged (KT_ERR_CUDA otherwise), and leaves the fastest
 * settings on the context.  The sample should be graphs like the ones to be
 * solved, but not those graphs themselves. */
typedef struct kt_tune_result {
  int64_t recount_gamma, dense_min_fill, dense_max_n, support_bitmap_max_n;
  int64_t kcore_big_row, peel_search_ratio, dense_tile_mb, kcore_blocks_per_sm, kcore_window, peel_bitset;
  int64_t peel_split;
  double ms_first;  /* the sample's device time with the settings at entry */
  double ms_best;   /* ... with the chosen settings */
  uint32_t trials;  /* timed candidate runs */
} kt_tune_result;
kt_status kt_autotune(kt_batch* sample, uint32_t passes, kt_tune_result* out);
/* The tuned options as "name value" lines (a comment names the GPU), and
 * back; unknown names are KT_ERR_INVALID. */
kt_status kt_options_save(kt_ctx* ctx, const char* path);
kt_status kt_options_load(kt_ctx* ctx, const char* path);

/* ----------------------------------------------------------------- serve */

/* A continuous-batching serving loop (no counterpart in the reference).
 * Requests are submitted from any thread at any time and queue in arrival
 * order.  The server runs serve_lanes (option, 1..4, default 2) lanes: lane 0
 * works on the context given, each other lane on a context the server creates
 * on the same device with the same options and budget.  Whenever a lane is
 * free it admits queued requests oldest first while their estimated device
 * footprint fits its share of half of the context's free budget (and at most
 * max_wave_graphs of them, 0 = 65535) and solves them as one wave of the
 * batch path on its own stream; requests that arrive while waves run start in
 * the next free lane, so waves overlap on the device.  With two or more lanes,
 * the last lane takes only small requests (serve_small_mb), oldest first, so they
 * never wait behind a wave of large graphs: that lane launches nothing
 * cooperative, and the other lanes' cooperative launches take 75% of the
 * device's resident blocks (coop_occupancy_pct, restored on the context at
 * kt_server_destroy), so its waves run beside theirs.  A request's answer is
 * the same alone and in any mix.  Other calls on the context block while a
 * wave of lane 0 runs. */
typedef struct kt_server kt_server;
typedef struct kt_request_result {
  kt_status status;      /* KT_OK, or the error of the wave that held it */
  uint32_t kmax;
  uint64_t edges;        /* kmax-truss edge count */
  double ms_wait;        /* submission -> admission into a wave (host clock) */
  double ms_latency;     /* submission -> result available */
  uint32_t wave;         /* the wave that solved it (0, 1, ... in order of completion) */
  uint32_t wave_graphs;  /* requests solved in that wave */
  uint32_t lane;         /* the lane that ran the wave */
  uint32_t pad0;
} kt_request_result;
typedef struct kt_server_stats {
  uint64_t submitted, completed, pending, waves, max_wave_graphs;
  double ms_busy;              /* worker time inside waves */
  uint64_t device_bytes_peak;  /* the context's peak device memory */
} kt_server_stats;
kt_status kt_server_create(kt_ctx* ctx, uint32_t max_wave_graphs, kt_server** out);
/* Queues a graph given as records x << 32 | y (copied).  KT_ERR_LIMIT if its
 * footprint alone exceeds what a wave of one lane may hold. */
kt_status kt_server_submit_pairs(kt_server* s, const uint64_t* xy, uint64_t count, uint64_t* request_id);
/* Queues graph `index` of the batched mix (generated on the device). */
kt_status kt_server_submit_mix(kt_server* s, uint64_t index, uint64_t base_seed, uint64_t* request_id);
/* A request's result; waits up to timeout_ms (0 = do not wait) and returns
 * KT_ERR_TIMEOUT while it is still pending.  A result can be read any number
 * of times: the server keeps each finished request's result record (about
 * 200 host bytes; its graph's records are freed when its wave ends) until
 * kt_server_destroy. */
kt_status kt_server_wait(kt_server* s, uint64_t request_id, uint32_t timeout_ms, kt_request_result* out);
kt_status kt_server_get_stats(kt_server* s, kt_server_stats* out);
/* Finishes every queued request, stops the worker and frees the server. */
void kt_server_destroy(kt_server* s);

/* ------------------------------------------------------- stage outputs */

/* Members of the k-core (member_out[v] = 1 if v is in it) and, in cmax_out,
 * the largest k with a non-empty k-core.  Replaces kmax_core_gpu
 * (src/kc.cu:770-884).  Either output may be NULL. */
kt_status kt_kcore(kt_ctx* ctx, kt_graph* g, uint32_t k, uint8_t* member_out, uint32_t* cmax_out);
/* k-core membership for callers that cannot allocate device memory at the
 * moment they need it (inside another runtime's fully reserved pool, from
 * host callbacks where an allocating CUDA call may block, or on paths that
 * cannot afford the synchronisation an allocation may imply).  No
 * counterpart in the reference.  DEVICE pointers: d_off (n+1 row offsets)
 * and d_adj (neighbour ids; symmetric, no self-loops, any row order) in,
 * d_member (n bytes, 1 = in the k-core) out; none may be NULL (KT_ERR_INVALID).
 * stream may be NULL (default stream); otherwise it must belong to the current
 * device (KT_ERR_INVALID).  d_member is unspecified unless the call returns
 * KT_OK.  Allocates nothing: its working memory is one fixed device array
 * of about 16 MB that every GPU loading the library holds until exit, which
 * caps n at 1,048,576 (KT_ERR_LIMIT above).  The first call on a device looks
 * up that array's device address and should come before any stream capture.
 * Calls share the array, so calls that overlap on the GPU race.  Returns
 * after the stream has finished the call. */
kt_status kt_kcore_noalloc(const uint64_t* d_off, const uint32_t* d_adj, uint32_t n, uint32_t k, uint8_t* d_member,
                           void* stream);
/* Core number of every vertex (num_vertices entries). */
kt_status kt_core_numbers(kt_ctx* ctx, kt_graph* g, uint32_t* core_out);
/* Triangles through each edge, in kt_graph_edges order.  Replaces
 * tricount_direct (src/kc.cu:584-651), which stores twice this value. */
kt_status kt_edge_support(kt_ctx* ctx, kt_graph* g, uint32_t* sup_out);
/* Trussness of each edge, in kt_graph_edges order (2 = in no triangle). */
kt_status kt_edge_trussness(kt_ctx* ctx, kt_graph* g, uint32_t* truss_out);

/* ----------------------------------------------------------- statistics */

typedef struct kt_stats {
  /* Device time (CUDA events on the context's stream) of the last solve:
   * ms_total spans the whole call (kt_solve_tsv: from the first host-to-device
   * copy to the answer; kt_solve_staged: from the parse). */
  double ms_parse, ms_csr, ms_kcore, ms_subgraph, ms_support, ms_peel, ms_total;
  uint64_t kernel_launches;       /* kernels this context launched since kt_stats_reset */
  uint64_t core_vertices, core_edges;       /* search-phase subgraph */
  uint64_t predict_vertices, predict_edges; /* prediction-phase subgraph */
  uint32_t cmax, kmax_lower_bound, levels, rounds;
  uint64_t support_bytes, peel_bytes;       /* algorithmic bytes of the last solve: a merge
                                               intersection's reads (support); list reads and
                                               decrements of the deletions (peel) */
  double ms_support_kernel, ms_peel_kernel; /* summed kernel time (events) */
  uint64_t support_launches, peel_launches;
  uint64_t device_bytes_peak;
  uint64_t h2d_bytes, d2h_bytes;            /* host<->device traffic since kt_stats_reset */
  uint64_t peel_decrements;                 /* support decrements of the last solve */
  uint32_t batch_waves, batch_graphs;       /* last kt_batch_run */
  /* Bytes the support kernels that ran moved, by their own access pattern:
   * for the dense (bitset) kernels 4 per row word read (row u loads, and the
   * words of row v actually ANDed, so a capped count's abandoned segments are
   * not counted) plus 16 per edge (list entry, ends, result); for the list
   * kernels the merge model of support_bytes. */
  uint64_t support_kernel_bytes;
  uint64_t support_row_words;               /* the dense kernels' row words read */
  uint64_t peel_recount_bytes;              /* bitset rows read by the peel's recount rounds */
  uint32_t csr_grouped;  /* last graph build took the rows straight from grouped TSV lines (1) or sorted (0) */
  uint32_t pad0;
} kt_stats;
kt_status kt_get_stats(const kt_ctx* ctx, kt_stats* out);
kt_status kt_stats_reset(kt_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
