// Host-side internals shared by the solver's translation units: the context,
// device buffers charged to the context's HBM budget, error propagation and
// launch accounting.
#pragma once
#include <algorithm>
#include <cstdio>
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "kt.h"

namespace kt {

// Exceptions carry a status to the C boundary (api.cu), where they become
// return codes; nothing is thrown across extern "C".
struct Error : std::runtime_error {
  kt_status status;
  Error(kt_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line);

#define KT_CUDA(call)                                                   \
  do {                                                                  \
    cudaError_t kt_e_ = (call);                                         \
    if (kt_e_ != cudaSuccess) ::kt::throw_cuda(kt_e_, #call, __FILE__, __LINE__); \
  } while (0)

#define KT_LAUNCHED(ctx)                                                   \
  do {                                                                     \
    cudaError_t kt_e_ = cudaGetLastError();                                \
    if (kt_e_ != cudaSuccess) ::kt::throw_cuda(kt_e_, "kernel launch", __FILE__, __LINE__); \
    (ctx)->launches++;                                                     \
  } while (0)

// Tunables, settable by name through kt_set_option.
struct Options {
  int64_t predict = 1;            // run the prediction phase (truss of the max core)
  int64_t persistent = 1;         // peel / k-core rounds inside one cooperative launch
  int64_t support_bitmap_max_n = 1 << 20;  // vertex-centric bitmap support up to this many vertices
  int64_t dense_max_n = 1 << 16;  // adjacency bitsets (dense mode) up to this many vertices
  int64_t dense_min_fill = 32;    // dense mode when avg degree * this >= words per row
  int64_t recount_gamma = 16;     // recount round when |F| * thr * gamma > alive * words
  int64_t capped_support = 1;     // search phase: abandon supports that cannot reach the threshold
  int64_t timeout_ms = 20000;     // bound on any device-side wait
  int64_t parse_pipeline_mb = 256;  // host->device chunk: file ingest, and the chunked parse of host bytes
  int64_t record_kernel_times = 0;  // events around support / peel kernels
  int64_t debug_checks = 0;       // extra host-side consistency checks
  int64_t verbose = 0;            // stage decisions on stderr
  int64_t pool_reserve_mb = 0;    // setting it grows the memory pool by this much at once
  int64_t kcore_big_row = 512;    // k-core rounds: longer rows are dealt to all warps in 32-entry windows
  int64_t peel_search_ratio = 16; // peel: binary-search the long row when it is this many times longer
  int64_t dense_tile_mb = 48;     // dense support: bitset rows of two tile blocks within this many MB
  int64_t kcore_blocks_per_sm = 0;  // core decomposition: resident blocks per SM (0 = as many as fit)
  int64_t kcore_window = 32;      // core decomposition: levels per pass over the whole alive list
  int64_t peel_bitset = 1;        // peel: dense rows intersected as bitsets when shorter than the lists
  int64_t kcore_compact = 4;      // max-core search: compact once the core's edges are < 1/this of the graph's (0 = never)
  int64_t wave_budget_pct = 50;   // batch: a wave's estimated footprint within this % of the free budget
  int64_t peel_split = 16;        // peel: (edge, 8-word chunk) units when frontier x chunks <= this x warps (0 = off)
  int64_t serve_lanes = 2;        // serving: waves in flight at once (each on a stream of its own)
  int64_t serve_small_mb = 128;   // serving, two or more lanes: the last lane admits only requests this small (0: any)
  int64_t serve_small_coop = 0;   // serving: the small lane's kernels cooperative (1) or host-stepped (0)
  int64_t serve_partition = 0;    // serving: the other lanes admit only requests above serve_small_mb
  int64_t batch_lanes = 2;        // batch: waves in flight at once (each on a stream of its own)
  int64_t support_rows = 2;       // exact dense support: edges sharing row u counted per read of it (1, 2, 4)
  int64_t peel_bisect_after = 16; // peel: truss levels climbed one at a time before bisecting the rest (0 = never)
  int64_t peel_bisect_gap = 16;   // peel: ... when the support bound is at least this far above
  int64_t coop_occupancy_pct = 100;  // cooperative grids: this % of the resident blocks the device holds
};

// Range check of an option value: every option is a count, size, ratio or
// flag (no negative values); timeout_ms is at most one hour.
bool option_value_ok(const char* name, int64_t value);

// Stage decisions on stderr when the context's verbose option is set.
#define KT_LOG(c, ...)                                  \
  do {                                                  \
    if ((c)->opt.verbose) std::fprintf(stderr, __VA_ARGS__); \
  } while (0)

struct Ctx;

// Stage timers: events recorded around kernels without synchronising; the
// elapsed times are collected when the solve ends (resolve()).
struct EventTimer {
  struct Span {
    cudaEvent_t a, b;
    double* acc;
  };
  std::vector<cudaEvent_t> pool;
  std::vector<Span> open;
  size_t used = 0;
  cudaEvent_t get();
  void begin(cudaStream_t s, double* acc, cudaEvent_t* out_a);
  void end(cudaStream_t s, cudaEvent_t a, double* acc);
  void resolve();  // adds elapsed times into their accumulators
  ~EventTimer();
};

// Device buffer charged to a context's budget; freed stream-ordered.
class DBuf {
 public:
  DBuf() = default;
  DBuf(Ctx* c, size_t bytes) { alloc(c, bytes); }
  ~DBuf() { release(); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept { *this = std::move(o); }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) {
      release();
      ctx_ = o.ctx_;
      ptr_ = o.ptr_;
      bytes_ = o.bytes_;
      o.ctx_ = nullptr;
      o.ptr_ = nullptr;
      o.bytes_ = 0;
    }
    return *this;
  }
  void alloc(Ctx* c, size_t bytes);
  void release();
  // Grows (discarding contents) when smaller than `bytes`.
  void ensure(Ctx* c, size_t bytes) {
    if (bytes > bytes_) {
      release();
      alloc(c, bytes);
    }
  }
  template <typename T>
  T* as() const { return static_cast<T*>(ptr_); }
  size_t bytes() const { return bytes_; }
  void* get() const { return ptr_; }

 private:
  Ctx* ctx_ = nullptr;
  void* ptr_ = nullptr;
  size_t bytes_ = 0;
};

struct Stats {
  kt_stats s{};
};

struct Ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // host-to-device chunks of the pipelined ingest
  uint64_t budget = 0;
  uint64_t in_use = 0;
  uint64_t peak = 0;
  uint64_t launches = 0;
  uint64_t h2d_bytes = 0, d2h_bytes = 0;
  // Text of the last error.  Guarded by its own mutex, not by `mu`, so a
  // reader is never held up by a serving wave that owns the context.
  std::string last_error;
  mutable std::mutex err_mu;
  void set_error(const std::string& m) {
    std::lock_guard<std::mutex> l(err_mu);
    last_error = m;
  }
  Options opt;
  kt_stats stats{};
  mutable std::recursive_mutex mu;  // every entry point, readers included
  // Pinned host words for small device-to-host reads.
  uint64_t* pinned = nullptr;
  cudaEvent_t ev[8] = {};
  // Device word block: bounded-wait error flag, barrier state, counters.
  DBuf words;
  EventTimer timer;
  // Set while this context is a lane of a server whose lanes share the
  // device: cooperative launches of the lanes then run one at a time.
  std::mutex* coop_mu = nullptr;
  // A second context on the same device for the batch driver's second lane
  // (created on first use, destroyed with this one).
  kt_ctx* aux = nullptr;
};

// Held from a cooperative launch until the host has read its result: a
// cooperative grid takes every SM's resident-block slots, so two of them
// (from two lanes of a server) are never in flight together.
struct CoopLock {
  std::unique_lock<std::mutex> l;
  explicit CoopLock(Ctx* c) {
    if (c->coop_mu) l = std::unique_lock<std::mutex>(*c->coop_mu);
  }
};

// Graph held on the device: cleaned, symmetric CSR (rows unsorted) plus the
// sorted canonical edge list.
struct Graph {
  uint64_t n = 0;      // vertex ids 0..n-1
  uint64_t m = 0;      // undirected edges
  DBuf off;            // uint64[n + 1]
  DBuf adj;            // uint32[2m]
  DBuf edges;          // uint64[m], sorted u << 32 | v, u < v
  DBuf deg;            // uint32[n]
  uint32_t max_deg = 0;
};

// Stream-ordered helpers.
void sync(Ctx* c);
template <typename T>
T read_word(Ctx* c, const T* dptr) {
  static_assert(sizeof(T) <= 8, "word");
  c->d2h_bytes += sizeof(T);
  KT_CUDA(cudaMemcpyAsync(c->pinned, dptr, sizeof(T), cudaMemcpyDeviceToHost, c->stream));
  sync(c);
  T v;
  memcpy(&v, c->pinned, sizeof(T));
  return v;
}
void copy_d2h(Ctx* c, void* dst, const void* src, size_t bytes);
void copy_h2d(Ctx* c, void* dst, const void* src, size_t bytes);
void zero(Ctx* c, void* dptr, size_t bytes);

// Device-wide primitives (scan.cu, sort.cu).
// Exclusive scan of n uint32 values into uint64 (out may not alias in).
void scan_u32_to_u64(Ctx* c, const uint32_t* in, uint64_t* out, uint64_t n);
// Exclusive scan of n uint32 values in place-safe form into uint32 (out may alias in).
void scan_u32(Ctx* c, const uint32_t* in, uint32_t* out, uint64_t n);
// Sum of n uint32 values (device result in *dsum, also returned).
uint64_t reduce_u32(Ctx* c, const uint32_t* in, uint64_t n);
// Stable LSD radix sort of keys (and optional uint32 values) by their bits
// [lo_bit, bits) (8-bit digits from lo_bit up; a digit may also read bits at
// or above `bits`, which must then be equal in every key).  `keys`/`vals`
// hold the input and receive the output.
void radix_sort_u64(Ctx* c, uint64_t* keys, uint32_t* vals, uint64_t n, int bits, int lo_bit = 0);
// Sorted-unique compaction of keys (drops key == ~0).  Returns new count.
uint64_t unique_sorted_u64(Ctx* c, const uint64_t* in, uint64_t* out, uint64_t n);

// Lets `func` launch with up to the device's opt-in shared memory per block
// (less its static shared memory), once per device and function.  Setting the
// largest limit once, instead of each launch's own size, keeps launches from
// two lanes (threads) of one device from lowering each other's limit.
void allow_max_dynamic_smem(const void* func);

// Milliseconds between two recorded events (waits for the second).
float event_ms(cudaEvent_t a, cudaEvent_t b);

// Grid of a cooperative launch: coop_occupancy_pct of the blocks that can be
// resident at once (per_sm on each SM), at least one.  Below 100, another
// lane's kernels keep room on every SM while the launch runs.
inline unsigned coop_blocks(const Ctx* c, int per_sm) {
  const int64_t pct = std::min<int64_t>(std::max<int64_t>(1, c->opt.coop_occupancy_pct), 100);
  const int64_t all = (int64_t)std::max(1, per_sm) * c->num_sms;
  return (unsigned)std::max<int64_t>(1, all * pct / 100);
}

// Grid sizing.
inline unsigned grid_for(uint64_t work, unsigned block, unsigned cap) {
  uint64_t g = (work + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

}  // namespace kt
