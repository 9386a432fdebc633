// The C ABI (include/kt.h): handles, status codes, ingest and stage outputs.
// Every entry point catches kt::Error and std::exception and returns a
// status; nothing is thrown across the boundary.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>

#include "handles.h"
#include "solve.h"


namespace kt {

DevWords* dev_words(Ctx* c) { return c->words.as<DevWords>(); }

bool option_value_ok(const char* name, int64_t value) {
  if (value < 0) return false;
  // timeout_ms = 0 is allowed: every bounded device wait then gives up at
  // once (the error path, for tests); above an hour is refused.
  if (!std::strcmp(name, "timeout_ms")) return value <= 3600000;
  if (!std::strcmp(name, "serve_lanes")) return value >= 1 && value <= 4;
  if (!std::strcmp(name, "batch_lanes")) return value >= 1 && value <= 2;
  if (!std::strcmp(name, "support_rows")) return value == 1 || value == 2 || value == 4;
  if (!std::strcmp(name, "peel_bisect_gap")) return value >= 1;
  if (!std::strcmp(name, "serve_small_coop")) return value == 0 || value == 1;
  if (!std::strcmp(name, "serve_partition")) return value == 0 || value == 1;
  if (!std::strcmp(name, "coop_occupancy_pct")) return value >= 1 && value <= 100;
  return true;
}

void reset_words(Ctx* c) {
  KT_CUDA(cudaMemsetAsync(c->words.get(), 0, sizeof(DevWords), c->stream));
  KT_CUDA(cudaMemsetAsync(&dev_words(c)->bad_line, 0xff, sizeof(unsigned long long), c->stream));
}

void check_words(Ctx* c, const char* stage) {
  DevWords w;
  copy_d2h(c, &w, c->words.get(), sizeof(DevWords));
  if (!w.err) return;
  char buf[256];
  kt_status s = KT_ERR_CUDA;
  if (w.err & kDevErrParse) {
    std::snprintf(buf, sizeof(buf), "malformed record on line %llu: a line needs two numbers",
                  (unsigned long long)w.bad_line + 1);
    s = KT_ERR_PARSE;
  } else if (w.err & (kDevErrBarrier | kDevErrWait)) {
    std::snprintf(buf, sizeof(buf), "%s: a bounded device wait gave up (flags %u)", stage, w.err);
    s = KT_ERR_TIMEOUT;
  } else {
    std::snprintf(buf, sizeof(buf), "%s: device work list overflow (flags %u)", stage, w.err);
  }
  reset_words(c);
  throw Error(s, buf);
}

namespace {

__global__ void k_canon_pairs(uint64_t* __restrict__ xy, uint64_t n, unsigned int* __restrict__ vmax,
                              unsigned int* __restrict__ any) {
  uint32_t mx = 0;
  bool seen = false;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = xy[i];
    const uint32_t x = (uint32_t)(k >> 32), y = (uint32_t)k;
    mx = max(mx, max(x, y));
    seen = true;
    xy[i] = x == y ? ~0ULL : (x < y ? (((uint64_t)x << 32) | y) : (((uint64_t)y << 32) | x));
  }
  mx = warp_max(mx);
  const unsigned s = __ballot_sync(kFull, seen);
  if (lane_id() == 0 && s) {
    atomicMax(vmax, mx);
    atomicOr(any, 1u);
  }
}

}  // namespace

float event_ms(cudaEvent_t a, cudaEvent_t b) {
  KT_CUDA(cudaEventSynchronize(b));
  float ms = 0;
  KT_CUDA(cudaEventElapsedTime(&ms, a, b));
  return ms;
}

// Device bytes (padded) -> Graph.
void graph_from_device_bytes(Ctx* c, const uint8_t* dbuf, uint64_t len, Graph& g) {
  reset_words(c);
  KT_CUDA(cudaEventRecord(c->ev[4], c->stream));
  DBuf block_off;
  const uint64_t lines = parse_count_lines(c, dbuf, len, block_off);
  DBuf keys(c, (lines ? lines : 1) * sizeof(uint64_t));
  parse_lines(c, dbuf, len, block_off, keys.as<uint64_t>(), dev_words(c));
  check_words(c, "parse");
  DevWords w;
  copy_d2h(c, &w, c->words.get(), sizeof(DevWords));
  const uint64_t n = (w.counters[1] & 1) ? (uint64_t)(uint32_t)w.counters[0] + 1 : 0;
  reset_words(c);
  block_off.release();
  KT_CUDA(cudaEventRecord(c->ev[5], c->stream));
  build_graph(c, keys.as<uint64_t>(), lines, n, g, true);
  KT_CUDA(cudaEventRecord(c->ev[6], c->stream));
  c->stats.ms_parse = event_ms(c->ev[4], c->ev[5]);
  c->stats.ms_csr = event_ms(c->ev[5], c->ev[6]);
}

// Host TSV bytes -> Graph with the host-to-device copy overlapped with the
// parse: the bytes go over in chunks (parse_pipeline_mb, whole parse blocks)
// on the copy stream; each chunk's lines are counted as soon as it lands and
// parsed into a record buffer of its own once the next chunk -- which its
// last lines may reach into -- has landed, so only the last chunk's parse and
// the joining of the chunks' records follow the copy.  A line that needs
// bytes not yet on the device (a line longer than a chunk) makes the whole
// parse run again once every byte is there.
static void load_tsv_pipelined(Ctx* c, const char* bytes, uint64_t len, uint64_t chunk, Graph& g) {
  DBuf dbuf(c, parse_padded_bytes(len));
  zero(c, dbuf.as<uint8_t>() + len, dbuf.bytes() - len);  // the parser reads zeros past len
  reset_words(c);
  const uint64_t nch = (len + chunk - 1) / chunk;
  const uint64_t bpc = chunk / parse_block_bytes();
  const uint64_t nblk = (len + parse_block_bytes() - 1) / parse_block_bytes();
  std::vector<cudaEvent_t> landed(nch + 1, nullptr);
  struct Events {
    std::vector<cudaEvent_t>& v;
    ~Events() {
      for (cudaEvent_t e : v)
        if (e) {
          cudaEventSynchronize(e);
          cudaEventDestroy(e);
        }
    }
  } guard{landed};
  for (cudaEvent_t& e : landed) KT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  // The copy stream starts once the buffer exists (it is allocated in order on
  // the main stream).
  KT_CUDA(cudaEventRecord(landed[nch], c->stream));
  KT_CUDA(cudaStreamWaitEvent(c->copy_stream, landed[nch], 0));
  for (uint64_t i = 0; i < nch; ++i) {
    const uint64_t off = i * chunk, n = std::min(chunk, len - off);
    KT_CUDA(cudaMemcpyAsync(dbuf.as<char>() + off, bytes + off, n, cudaMemcpyHostToDevice, c->copy_stream));
    KT_CUDA(cudaEventRecord(landed[i], c->copy_stream));
    c->h2d_bytes += n;
  }
  KT_CUDA(cudaEventRecord(c->ev[4], c->stream));
  std::vector<DBuf> part(nch);
  std::vector<uint64_t> plines(nch, 0);
  uint64_t lines = 0;
  for (uint64_t i = 0; i < nch; ++i) {
    KT_CUDA(cudaStreamWaitEvent(c->stream, landed[i], 0));
    const uint64_t b0 = i * bpc, nb = std::min(bpc, nblk - b0);
    DBuf boff;
    plines[i] = parse_count_lines(c, dbuf.as<uint8_t>(), len, boff, b0, nb);
    if (i + 1 < nch) KT_CUDA(cudaStreamWaitEvent(c->stream, landed[i + 1], 0));
    const uint64_t ready = i + 1 < nch ? std::min(len, (i + 2) * chunk) : len;
    part[i].alloc(c, (plines[i] ? plines[i] : 1) * sizeof(uint64_t));
    parse_lines(c, dbuf.as<uint8_t>(), len, boff, part[i].as<uint64_t>(), dev_words(c), b0, nb, ready, lines);
    lines += plines[i];
  }
  DevWords w;
  copy_d2h(c, &w, c->words.get(), sizeof(DevWords));
  if (w.counters[2]) {
    part.clear();
    graph_from_device_bytes(c, dbuf.as<uint8_t>(), len, g);
    return;
  }
  check_words(c, "parse");
  DBuf keys(c, (lines ? lines : 1) * sizeof(uint64_t));
  uint64_t at = 0;
  for (uint64_t i = 0; i < nch; ++i) {
    if (plines[i])
      KT_CUDA(cudaMemcpyAsync(keys.as<uint64_t>() + at, part[i].get(), plines[i] * sizeof(uint64_t),
                              cudaMemcpyDeviceToDevice, c->stream));
    at += plines[i];
    part[i].release();
  }
  const uint64_t n = (w.counters[1] & 1) ? (uint64_t)(uint32_t)w.counters[0] + 1 : 0;
  reset_words(c);
  KT_CUDA(cudaEventRecord(c->ev[5], c->stream));
  build_graph(c, keys.as<uint64_t>(), lines, n, g, true);
  KT_CUDA(cudaEventRecord(c->ev[6], c->stream));
  c->stats.ms_parse = event_ms(c->ev[4], c->ev[5]);  // copy and parse, overlapped
  c->stats.ms_csr = event_ms(c->ev[5], c->ev[6]);
}

void load_tsv(Ctx* c, const char* bytes, uint64_t len, Graph& g) {
  const uint64_t blk = parse_block_bytes();
  const uint64_t chunk = std::max<uint64_t>(1, ((uint64_t)std::max<int64_t>(1, c->opt.parse_pipeline_mb) << 20) / blk) * blk;
  if (len >= 3 * chunk) {
    load_tsv_pipelined(c, bytes, len, chunk, g);
    return;
  }
  DBuf dbuf(c, parse_padded_bytes(len));
  zero(c, dbuf.as<uint8_t>() + len, dbuf.bytes() - len);  // the parser reads zeros past len
  copy_h2d(c, dbuf.get(), bytes, len);
  graph_from_device_bytes(c, dbuf.as<uint8_t>(), len, g);
}

void load_pairs(Ctx* c, const uint64_t* xy, uint64_t count, Graph& g) {
  DBuf keys(c, (count ? count : 1) * sizeof(uint64_t));
  copy_h2d(c, keys.get(), xy, count * sizeof(uint64_t));
  DBuf mx(c, 8);
  zero(c, mx.get(), 8);
  if (count) {
    k_canon_pairs<<<grid_for(count, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        keys.as<uint64_t>(), count, mx.as<unsigned int>(), mx.as<unsigned int>() + 1);
    KT_LAUNCHED(c);
  }
  uint32_t h[2];
  copy_d2h(c, h, mx.get(), 8);
  const uint64_t n = h[1] ? (uint64_t)h[0] + 1 : 0;
  build_graph(c, keys.as<uint64_t>(), count, n, g);
}

// File ingest: mmap, then copy through two pinned staging buffers so the
// host-side copy of one chunk overlaps the device copy of the previous one.
static void load_tsv_file(Ctx* c, const char* path, Graph& g) {
  const int fd = open(path, O_RDONLY);
  if (fd < 0) throw Error(KT_ERR_IO, std::string("open file error: ") + std::strerror(errno));
  struct stat sb;
  if (fstat(fd, &sb) < 0) {
    const int e = errno;
    close(fd);
    throw Error(KT_ERR_IO, std::string("get file length error: ") + std::strerror(e));
  }
  const uint64_t len = (uint64_t)sb.st_size;
  void* map = len ? mmap(nullptr, len, PROT_READ, MAP_SHARED, fd, 0) : MAP_FAILED;
  if (map == MAP_FAILED) {
    // The reference maps the file the same way and fails identically on an
    // empty file (src/mapfile.hpp:50-54).
    const int e = len ? errno : EINVAL;
    close(fd);
    throw Error(KT_ERR_IO, std::string("mmap file error: ") + std::strerror(e));
  }
  madvise(map, len, MADV_SEQUENTIAL);
  struct Unmap {
    void* p;
    uint64_t n;
    int fd;
    ~Unmap() {
      munmap(p, n);
      close(fd);
    }
  } unmap{map, len, fd};
  DBuf dbuf(c, parse_padded_bytes(len));
  zero(c, dbuf.as<uint8_t>() + len, dbuf.bytes() - len);  // the parser reads zeros past len
  const uint64_t chunk = (uint64_t)std::max<int64_t>(1, c->opt.parse_pipeline_mb) << 20;
  char* stage[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  struct Pinned {
    char** s;
    cudaEvent_t* d;
    ~Pinned() {
      for (int i = 0; i < 2; ++i) {
        if (d[i]) {
          cudaEventSynchronize(d[i]);
          cudaEventDestroy(d[i]);
        }
        if (s[i]) cudaFreeHost(s[i]);
      }
    }
  } pinned{stage, done};
  for (int i = 0; i < 2; ++i) {
    KT_CUDA(cudaHostAlloc(&stage[i], chunk, cudaHostAllocDefault));
    KT_CUDA(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming));
  }
  const char* src = static_cast<const char*>(map);
  int slot = 0;
  for (uint64_t off = 0; off < len; off += chunk, slot ^= 1) {
    const uint64_t n = std::min(chunk, len - off);
    KT_CUDA(cudaEventSynchronize(done[slot]));
#pragma omp parallel for schedule(static)
    for (int t = 0; t < 16; ++t) {
      const uint64_t a = n * t / 16, b = n * (t + 1) / 16;
      std::memcpy(stage[slot] + a, src + off + a, b - a);
    }
    KT_CUDA(cudaMemcpyAsync(dbuf.as<char>() + off, stage[slot], n, cudaMemcpyHostToDevice, c->stream));
    KT_CUDA(cudaEventRecord(done[slot], c->stream));
  }
  graph_from_device_bytes(c, dbuf.as<uint8_t>(), len, g);
}

}  // namespace kt

using kt::Error;

extern "C" {

const char* kt_status_string(kt_status s) {
  switch (s) {
    case KT_OK: return "ok";
    case KT_ERR_INVALID: return "invalid argument";
    case KT_ERR_CUDA: return "CUDA error";
    case KT_ERR_NOMEM: return "out of device memory";
    case KT_ERR_PARSE: return "malformed input";
    case KT_ERR_IO: return "I/O error";
    case KT_ERR_TIMEOUT: return "device wait timed out";
    case KT_ERR_LIMIT: return "size limit exceeded";
    case KT_ERR_NODEV: return "no CUDA device";
    case KT_ERR_BUSY: return "busy";
  }
  return "unknown status";
}

namespace {
// Contexts alive per device (the default memory pool is shared by them).
int live_contexts(int device, int delta) {
  static std::mutex mu;
  static std::map<int, int> live;
  std::lock_guard<std::mutex> lk(mu);
  return live[device] += delta;
}
}  // namespace

kt_status kt_init(int device, uint64_t budget, kt_ctx** out) {
  if (!out) return KT_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return KT_ERR_NODEV;
  }
  if (device < 0 || device >= ndev) return KT_ERR_INVALID;
  kt_ctx* h = new (std::nothrow) kt_ctx;
  if (!h) return KT_ERR_NOMEM;
  kt::Ctx& c = h->c;
  c.device = device;
  try {
    KT_CUDA(cudaSetDevice(device));
    KT_CUDA(cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, device));
    KT_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    KT_CUDA(cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking));
    size_t fr = 0, tot = 0;
    KT_CUDA(cudaMemGetInfo(&fr, &tot));
    // Keep freed blocks in the pool for reuse across calls.  Memory the pool
    // holds but no allocation uses (left by earlier contexts) counts as free.
    cudaMemPool_t pool;
    KT_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t thr = UINT64_MAX;
    KT_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    uint64_t reserved = 0, used = 0;
    KT_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
    KT_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
    c.budget = budget ? budget : (uint64_t)((fr + (reserved > used ? reserved - used : 0)) * 0.9);
    live_contexts(device, +1);
    h->counted = true;
    KT_CUDA(cudaHostAlloc(&c.pinned, 4096, cudaHostAllocDefault));
    for (auto& e : c.ev) KT_CUDA(cudaEventCreate(&e));
    c.words.alloc(&c, sizeof(kt::DevWords));
    kt::reset_words(&c);
    kt::sync(&c);
  } catch (const Error&) {
    kt_destroy(h);
    return KT_ERR_CUDA;
  }
  *out = h;
  return KT_OK;
}

void kt_destroy(kt_ctx* h) {
  if (!h) return;
  if (h->c.aux) {
    kt_destroy(h->c.aux);
    h->c.aux = nullptr;
  }
  {
    std::lock_guard<std::recursive_mutex> lk(h->c.mu);
    cudaSetDevice(h->c.device);
    h->c.words.release();
    if (h->c.stream) cudaStreamSynchronize(h->c.stream);
    for (auto& e : h->c.ev)
      if (e) cudaEventDestroy(e);
    if (h->c.pinned) cudaFreeHost(h->c.pinned);
    if (h->c.stream) cudaStreamDestroy(h->c.stream);
    if (h->c.copy_stream) cudaStreamDestroy(h->c.copy_stream);
    // The last context on the device hands the pool's cached memory back,
    // so the next one (or anything else in the process) can have it.
    if (h->counted && live_contexts(h->c.device, -1) == 0) {
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, h->c.device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
      cudaGetLastError();
    }
  }
  delete h;
}

const char* kt_last_error(const kt_ctx* h) {
  if (!h) return "null context";
  // A copy per calling thread, taken under the error text's own mutex: a
  // serving worker may overwrite the text while the caller reads it, and the
  // worker holds the context lock for a whole wave.
  static thread_local std::string copy;
  std::lock_guard<std::mutex> lk(h->c.err_mu);
  copy = h->c.last_error;
  return copy.c_str();
}

static int64_t* option_slot(kt::Options& o, const char* name) {
  if (!name) return nullptr;
  struct {
    const char* n;
    int64_t* p;
  } tab[] = {{"predict", &o.predict},
             {"persistent", &o.persistent},
             {"support_bitmap_max_n", &o.support_bitmap_max_n},
             {"dense_max_n", &o.dense_max_n},
             {"dense_min_fill", &o.dense_min_fill},
             {"recount_gamma", &o.recount_gamma},
             {"capped_support", &o.capped_support},
             {"timeout_ms", &o.timeout_ms},
             {"parse_pipeline_mb", &o.parse_pipeline_mb},
             {"record_kernel_times", &o.record_kernel_times},
             {"debug_checks", &o.debug_checks},
             {"verbose", &o.verbose},
             {"pool_reserve_mb", &o.pool_reserve_mb},
             {"kcore_big_row", &o.kcore_big_row},
             {"peel_search_ratio", &o.peel_search_ratio},
             {"dense_tile_mb", &o.dense_tile_mb},
             {"kcore_blocks_per_sm", &o.kcore_blocks_per_sm},
             {"kcore_window", &o.kcore_window},
             {"peel_bitset", &o.peel_bitset},
             {"peel_split", &o.peel_split},
             {"kcore_compact", &o.kcore_compact},
             {"wave_budget_pct", &o.wave_budget_pct},
             {"serve_lanes", &o.serve_lanes},
             {"batch_lanes", &o.batch_lanes},
             {"support_rows", &o.support_rows},
             {"serve_small_mb", &o.serve_small_mb},
             {"serve_small_coop", &o.serve_small_coop},
             {"serve_partition", &o.serve_partition},
             {"peel_bisect_after", &o.peel_bisect_after},
             {"peel_bisect_gap", &o.peel_bisect_gap},
             {"coop_occupancy_pct", &o.coop_occupancy_pct}};
  for (auto& t : tab)
    if (!std::strcmp(t.n, name)) return t.p;
  return nullptr;
}

kt_status kt_set_option(kt_ctx* h, const char* name, int64_t value) {
  if (!h) return KT_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(h->c.mu);
  int64_t* p = option_slot(h->c.opt, name);
  if (!p || !kt::option_value_ok(name, value)) return KT_ERR_INVALID;
  *p = value;
  if (!std::strcmp(name, "pool_reserve_mb") && value > 0) {
    // Grow the context's memory pool once, up front: later allocations up to
    // this size are served from it instead of mapping new memory mid-solve.
    kt::Ctx* c = &h->c;
    const uint64_t bytes = std::min<uint64_t>((uint64_t)value << 20, c->budget > c->in_use ? c->budget - c->in_use : 0);
    void* ptr = nullptr;
    if (bytes && cudaMallocAsync(&ptr, bytes, c->stream) == cudaSuccess) {
      cudaFreeAsync(ptr, c->stream);
      if (cudaStreamSynchronize(c->stream) != cudaSuccess) return KT_ERR_CUDA;
    } else if (bytes) {
      cudaGetLastError();
      return KT_ERR_NOMEM;
    }
  }
  return KT_OK;
}

kt_status kt_get_option(const kt_ctx* h, const char* name, int64_t* value) {
  if (!h || !value) return KT_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(h->c.mu);
  int64_t* p = option_slot(const_cast<kt::Options&>(h->c.opt), name);
  if (!p) return KT_ERR_INVALID;
  *value = *p;
  return KT_OK;
}

kt_status kt_load_tsv(kt_ctx* h, const char* bytes, uint64_t len, kt_graph** out) {
  if (!out || (!bytes && len)) return KT_ERR_INVALID;
  *out = nullptr;
  KT_API_BEGIN(h)
  kt_graph* g = new kt_graph;
  try {
    kt::load_tsv(&h->c, bytes, len, g->g);
  } catch (...) {
    delete g;
    throw;
  }
  *out = g;
  KT_API_END(h)
}

kt_status kt_load_tsv_file(kt_ctx* h, const char* path, kt_graph** out) {
  if (!out || !path) return KT_ERR_INVALID;
  *out = nullptr;
  KT_API_BEGIN(h)
  kt_graph* g = new kt_graph;
  try {
    kt::load_tsv_file(&h->c, path, g->g);
  } catch (...) {
    delete g;
    throw;
  }
  *out = g;
  KT_API_END(h)
}

kt_status kt_load_pairs(kt_ctx* h, const uint64_t* xy, uint64_t count, kt_graph** out) {
  if (!out || (!xy && count)) return KT_ERR_INVALID;
  *out = nullptr;
  KT_API_BEGIN(h)
  kt_graph* g = new kt_graph;
  try {
    kt::load_pairs(&h->c, xy, count, g->g);
  } catch (...) {
    delete g;
    throw;
  }
  *out = g;
  KT_API_END(h)
}

kt_status kt_graph_info(const kt_graph* g, uint64_t* nv, uint64_t* ne) {
  if (!g) return KT_ERR_INVALID;
  if (nv) *nv = g->g.n;
  if (ne) *ne = g->g.m;
  return KT_OK;
}

kt_status kt_graph_edges(kt_ctx* h, const kt_graph* g, uint64_t* keys) {
  if (!g || (!keys && g->g.m)) return KT_ERR_INVALID;
  KT_API_BEGIN(h)
  kt::copy_d2h(&h->c, keys, g->g.edges.get(), g->g.m * sizeof(uint64_t));
  KT_API_END(h)
}

void kt_graph_free(kt_ctx* h, kt_graph* g) {
  if (!g) return;
  if (h) {
    std::lock_guard<std::recursive_mutex> lk(h->c.mu);
    cudaSetDevice(h->c.device);
    delete g;
  } else {
    delete g;
  }
}

kt_status kt_solve(kt_ctx* h, kt_graph* g, uint32_t* kmax, uint64_t* edges) {
  if (!g || !kmax || !edges) return KT_ERR_INVALID;
  KT_API_BEGIN(h)
  kt::Ctx* c = &h->c;
  kt::reset_words(c);
  kt::begin_solve_stats(c);
  KT_CUDA(cudaEventRecord(c->ev[0], c->stream));
  kt::solve_graph(c, g->g, kmax, edges);
  KT_CUDA(cudaEventRecord(c->ev[1], c->stream));
  c->stats.ms_total = kt::event_ms(c->ev[0], c->ev[1]);
  KT_API_END(h)
}

kt_status kt_solve_tsv(kt_ctx* h, const char* bytes, uint64_t len, uint32_t* kmax, uint64_t* edges) {
  if (!kmax || !edges || (!bytes && len)) return KT_ERR_INVALID;
  KT_API_BEGIN(h)
  kt::Ctx* c = &h->c;
  kt::begin_solve_stats(c);
  KT_CUDA(cudaEventRecord(c->ev[0], c->stream));
  {
    kt::Graph g;
    kt::load_tsv(c, bytes, len, g);
    const double p = c->stats.ms_parse, q = c->stats.ms_csr;
    kt::solve_graph(c, g, kmax, edges);
    c->stats.ms_parse = p;
    c->stats.ms_csr = q;
  }
  KT_CUDA(cudaEventRecord(c->ev[1], c->stream));
  c->stats.ms_total = kt::event_ms(c->ev[0], c->ev[1]);
  KT_API_END(h)
}

kt_status kt_tsv_stage(kt_ctx* h, const char* bytes, uint64_t len, kt_tsv** out) {
  if (!out || (!bytes && len)) return KT_ERR_INVALID;
  *out = nullptr;
  KT_API_BEGIN(h)
  kt::Ctx* c = &h->c;
  kt_tsv* t = new kt_tsv;
  try {
    t->len = len;
    t->bytes.alloc(c, kt::parse_padded_bytes(len));
    kt::zero(c, t->bytes.as<uint8_t>() + len, t->bytes.bytes() - len);  // the parser reads zeros past len
    kt::copy_h2d(c, t->bytes.get(), bytes, len);
    kt::sync(c);
  } catch (...) {
    delete t;
    throw;
  }
  *out = t;
  KT_API_END(h)
}

kt_status kt_solve_staged(kt_ctx* h, const kt_tsv* t, uint32_t* kmax, uint64_t* edges) {
  if (!t || !kmax || !edges) return KT_ERR_INVALID;
  KT_API_BEGIN(h)
  kt::Ctx* c = &h->c;
  kt::begin_solve_stats(c);
  const auto t0 = std::chrono::steady_clock::now();
  auto host_ms = [&] { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); };
  KT_CUDA(cudaEventRecord(c->ev[0], c->stream));
  {
    kt::Graph g;
    kt::graph_from_device_bytes(c, t->bytes.as<uint8_t>(), t->len, g);
    KT_LOG(c, "kt: +%.2f ms graph built (parse %.2f, build %.2f ms)\n", host_ms(), c->stats.ms_parse,
           c->stats.ms_csr);
    const double p = c->stats.ms_parse, q = c->stats.ms_csr;
    kt::solve_graph(c, g, kmax, edges);
    c->stats.ms_parse = p;
    c->stats.ms_csr = q;
    KT_LOG(c, "kt: +%.2f ms solved\n", host_ms());
  }
  KT_CUDA(cudaEventRecord(c->ev[1], c->stream));
  c->stats.ms_total = kt::event_ms(c->ev[0], c->ev[1]);
  KT_LOG(c, "kt: +%.2f ms graph freed; device time %.2f ms\n", host_ms(), c->stats.ms_total);
  KT_API_END(h)
}

void kt_tsv_free(kt_ctx* h, kt_tsv* t) {
  if (!t) return;
  if (h) {
    std::lock_guard<std::recursive_mutex> lk(h->c.mu);
    cudaSetDevice(h->c.device);
    delete t;
  } else {
    delete t;
  }
}

kt_status kt_batch_create(kt_ctx* h, kt_batch** out) {
  if (!h || !out) return KT_ERR_INVALID;
  *out = new (std::nothrow) kt_batch;
  if (!*out) return KT_ERR_NOMEM;
  (*out)->ctx = h;
  return KT_OK;
}

kt_status kt_batch_add_pairs(kt_batch* b, const uint64_t* xy, uint64_t count, uint32_t* graph_id) {
  if (!b || (!xy && count)) return KT_ERR_INVALID;
  try {
    b->items.emplace_back();
    b->items.back().from_pairs(xy, count);
  } catch (const std::bad_alloc&) {
    return KT_ERR_NOMEM;
  }
  if (graph_id) *graph_id = (uint32_t)(b->items.size() - 1);
  return KT_OK;
}

kt_status kt_batch_add_mix(kt_batch* b, uint64_t first, uint64_t count, uint64_t base_seed) {
  if (!b) return KT_ERR_INVALID;
  try {
    for (uint64_t i = 0; i < count; ++i) {
      b->items.emplace_back();
      b->items.back().from_mix(first + i, base_seed);
    }
  } catch (const std::bad_alloc&) {
    return KT_ERR_NOMEM;
  }
  return KT_OK;
}

kt_status kt_batch_size(const kt_batch* b, uint64_t* graphs, uint64_t* records) {
  if (!b) return KT_ERR_INVALID;
  if (graphs) *graphs = b->items.size();
  if (records) {
    uint64_t s = 0;
    for (const auto& it : b->items) s += it.nkeys;
    *records = s;
  }
  return KT_OK;
}

kt_status kt_batch_run(kt_batch* b) {
  if (!b) return KT_ERR_INVALID;
  kt_ctx* h = b->ctx;
  KT_API_BEGIN(h)
  kt::Ctx* c = &h->c;
  kt::reset_words(c);
  kt::begin_solve_stats(c);
  KT_CUDA(cudaEventRecord(c->ev[0], c->stream));
  kt::BatchRun run;
  {
    struct Resolve {
      kt::Ctx* c;
      ~Resolve() {
        try {
          c->timer.resolve();
        } catch (...) {
        }
      }
    } resolve{c};
    kt::run_batch(c, b->items, run);
  }
  KT_CUDA(cudaEventRecord(c->ev[1], c->stream));
  c->stats.ms_total = kt::event_ms(c->ev[0], c->ev[1]);
  c->stats.batch_waves = run.waves;
  c->stats.batch_graphs = (uint32_t)b->items.size();
  KT_API_END(h)
}

kt_status kt_batch_results(const kt_batch* b, uint32_t* kmax, uint64_t* edges) {
  if (!b) return KT_ERR_INVALID;
  for (size_t i = 0; i < b->items.size(); ++i) {
    if (kmax) kmax[i] = b->items[i].kmax;
    if (edges) edges[i] = b->items[i].count;
  }
  return KT_OK;
}

void kt_batch_free(kt_batch* b) { delete b; }

kt_status kt_load_mix_graph(kt_ctx* h, uint64_t index, uint64_t base_seed, kt_graph** out) {
  if (!out) return KT_ERR_INVALID;
  *out = nullptr;
  KT_API_BEGIN(h)
  kt_graph* g = new kt_graph;
  try {
    kt::load_mix_graph(&h->c, index, base_seed, g->g);
  } catch (...) {
    delete g;
    throw;
  }
  *out = g;
  KT_API_END(h)
}

kt_status kt_kcore(kt_ctx* h, kt_graph* g, uint32_t k, uint8_t* member, uint32_t* cmax) {
  if (!g) return KT_ERR_INVALID;
  KT_API_BEGIN(h)
  kt::Ctx* c = &h->c;
  kt::KCore kc;
  kc.init(c, g->g);
  const uint32_t cm = kc.find_max_core(c);
  if (cmax) *cmax = cm;
  if (member && g->g.n) {
    kt::DBuf d(c, g->g.n);
    if (k == 0) {
      KT_CUDA(cudaMemsetAsync(d.get(), 1, g->g.n, c->stream));
    } else if (k > cm) {
      kt::zero(c, d.get(), g->g.n);
    } else {
      kc.restore_core(c, k);
      kc.members(c, d.as<uint8_t>());
    }
    kt::copy_d2h(c, member, d.get(), g->g.n);
  }
  KT_API_END(h)
}

kt_status kt_core_numbers(kt_ctx* h, kt_graph* g, uint32_t* core) {
  if (!g || (!core && g->g.n)) return KT_ERR_INVALID;
  KT_API_BEGIN(h)
  kt::Ctx* c = &h->c;
  kt::KCore kc;
  kc.init(c, g->g);
  kt::DBuf d(c, (g->g.n ? g->g.n : 1) * sizeof(uint32_t));
  kc.core_numbers(c, d.as<uint32_t>());
  kt::copy_d2h(c, core, d.get(), g->g.n * sizeof(uint32_t));
  KT_API_END(h)
}

kt_status kt_edge_support(kt_ctx* h, kt_graph* g, uint32_t* sup) {
  if (!g || (!sup && g->g.m)) return KT_ERR_INVALID;
  KT_API_BEGIN(h)
  kt::Ctx* c = &h->c;
  kt::DBuf d(c, (g->g.m ? g->g.m : 1) * sizeof(uint32_t));
  kt::zero(c, d.get(), d.bytes());
  kt::graph_support(c, g->g, d.as<uint32_t>());
  kt::copy_d2h(c, sup, d.get(), g->g.m * sizeof(uint32_t));
  KT_API_END(h)
}

kt_status kt_edge_trussness(kt_ctx* h, kt_graph* g, uint32_t* truss) {
  if (!g || (!truss && g->g.m)) return KT_ERR_INVALID;
  KT_API_BEGIN(h)
  kt::Ctx* c = &h->c;
  kt::DBuf d(c, (g->g.m ? g->g.m : 1) * sizeof(uint32_t));
  kt::zero(c, d.get(), d.bytes());
  kt::reset_words(c);
  kt::graph_trussness(c, g->g, d.as<uint32_t>());
  kt::copy_d2h(c, truss, d.get(), g->g.m * sizeof(uint32_t));
  KT_API_END(h)
}

kt_status kt_get_stats(const kt_ctx* h, kt_stats* out) {
  if (!h || !out) return KT_ERR_INVALID;
  // A serving worker may be writing these mid-wave: read them under the lock.
  std::lock_guard<std::recursive_mutex> lk(h->c.mu);
  *out = h->c.stats;
  out->kernel_launches = h->c.launches;
  out->device_bytes_peak = h->c.peak;
  out->h2d_bytes = h->c.h2d_bytes;
  out->d2h_bytes = h->c.d2h_bytes;
  return KT_OK;
}

kt_status kt_stats_reset(kt_ctx* h) {
  if (!h) return KT_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(h->c.mu);
  h->c.stats = kt_stats{};
  h->c.launches = 0;
  h->c.h2d_bytes = h->c.d2h_bytes = 0;
  h->c.peak = h->c.in_use;
  return KT_OK;
}

}  // extern "C"
