// Autotuner of the thresholds that pick the variants of the support, peel
// and k-core kernels: the bin thresholds (which vertex-count range gets the
// dense bitset support, which the shared-memory bitmap support; which rows
// the k-core rounds expand with whole blocks) and the tile thresholds (the
// dense support's tile-block size, the peel's switch from the 32-wide tile
// merge to per-lane binary search, the cost ratio that turns a peel round
// into an AND/popcount recount, the core decomposition's blocks per SM and
// levels per window, the peel's bitset intersection of dense rows and its
// split rounds).
//
// The tuner times a sample batch -- graphs like the ones the caller will
// solve -- under candidate values, one parameter at a time (coordinate
// descent from the context's current settings), keeps a candidate only when
// it is faster by more than the noise margin, checks that every candidate
// gives the sample's answers unchanged, and leaves the best settings on the
// context.  kt_options_save / kt_options_load keep a tuned setting in a
// plain "name value" text file, so a tuning run can be reused.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "handles.h"
#include "solve.h"

namespace kt {
namespace {

struct Param {
  const char* name;
  int64_t Options::*field;
  std::vector<int64_t> cands;
};

const std::vector<Param>& params() {
  static const std::vector<Param> p = {
      {"recount_gamma", &Options::recount_gamma, {2, 4, 8, 16, 32, 64, 128}},
      {"dense_min_fill", &Options::dense_min_fill, {4, 8, 16, 32, 64, 128}},
      {"dense_max_n", &Options::dense_max_n, {16384, 32768, 65536, 131072}},
      {"support_bitmap_max_n", &Options::support_bitmap_max_n, {1 << 17, 1 << 18, 1 << 19, 1 << 20}},
      {"kcore_big_row", &Options::kcore_big_row, {64, 128, 256, 512, 1024, 2048}},
      {"peel_search_ratio", &Options::peel_search_ratio, {4, 8, 16, 32, 64}},
      {"dense_tile_mb", &Options::dense_tile_mb, {12, 24, 48, 96}},
      {"kcore_blocks_per_sm", &Options::kcore_blocks_per_sm, {0, 1, 2, 4}},
      {"kcore_window", &Options::kcore_window, {8, 16, 32, 64, 128}},
      {"peel_bitset", &Options::peel_bitset, {0, 1}},
      {"peel_split", &Options::peel_split, {0, 4, 16, 64}},
  };
  return p;
}

// Device time of one run of the batch (the whole run, input generation
// included: with two lanes one wave's generation overlaps another's solve)
// and its answers.
double time_batch(Ctx* c, std::vector<BatchItem>& items, std::vector<uint32_t>& kmax, std::vector<uint64_t>& count) {
  reset_words(c);
  begin_solve_stats(c);
  KT_CUDA(cudaEventRecord(c->ev[0], c->stream));
  BatchRun run;
  {
    struct Resolve {
      Ctx* c;
      ~Resolve() {
        try {
          c->timer.resolve();
        } catch (...) {
        }
      }
    } resolve{c};
    run_batch(c, items, run);
  }
  KT_CUDA(cudaEventRecord(c->ev[1], c->stream));
  c->stats.ms_total = event_ms(c->ev[0], c->ev[1]);
  kmax.resize(items.size());
  count.resize(items.size());
  for (size_t i = 0; i < items.size(); ++i) {
    kmax[i] = items[i].kmax;
    count[i] = items[i].count;
  }
  return c->stats.ms_total;
}

void fill_result(const Options& o, kt_tune_result* r) {
  r->recount_gamma = o.recount_gamma;
  r->dense_min_fill = o.dense_min_fill;
  r->dense_max_n = o.dense_max_n;
  r->support_bitmap_max_n = o.support_bitmap_max_n;
  r->kcore_big_row = o.kcore_big_row;
  r->peel_search_ratio = o.peel_search_ratio;
  r->dense_tile_mb = o.dense_tile_mb;
  r->kcore_blocks_per_sm = o.kcore_blocks_per_sm;
  r->kcore_window = o.kcore_window;
  r->peel_bitset = o.peel_bitset;
  r->peel_split = o.peel_split;
}

}  // namespace

void autotune(Ctx* c, std::vector<BatchItem>& items, uint32_t passes, kt_tune_result* out) {
  std::memset(out, 0, sizeof(*out));
  std::vector<uint32_t> k0, k;
  std::vector<uint64_t> c0, cn;
  time_batch(c, items, k0, c0);  // warm-up: memory pool, module loading
  double best = time_batch(c, items, k, cn);
  if (k != k0 || cn != c0) throw Error(KT_ERR_CUDA, "autotune: two runs of the sample disagree");
  out->ms_first = best;
  // A candidate must beat the incumbent by this fraction to replace it.
  const double margin = 0.02;
  uint32_t trials = 0;
  for (uint32_t pass = 0; pass < std::max<uint32_t>(1, passes); ++pass) {
    bool changed = false;
    for (const Param& p : params()) {
      const int64_t start = c->opt.*p.field;
      int64_t keep = start;
      for (int64_t v : p.cands) {
        if (v == start) continue;
        c->opt.*p.field = v;
        double ms = 0;
        try {
          ms = time_batch(c, items, k, cn);
        } catch (const Error& e) {
          // A setting the sample cannot run with (e.g. bitsets beyond the
          // budget) is not a candidate.
          if (e.status != KT_ERR_NOMEM && e.status != KT_ERR_LIMIT) throw;
          KT_LOG(c, "kt: autotune %s=%lld: %s\n", p.name, (long long)v, e.what());
          continue;
        }
        ++trials;
        if (k != k0 || cn != c0)
          throw Error(KT_ERR_CUDA, std::string("autotune: answers changed with ") + p.name + "=" + std::to_string(v));
        KT_LOG(c, "kt: autotune %s=%lld: %.2f ms (best %.2f)\n", p.name, (long long)v, ms, best);
        if (ms < best * (1.0 - margin)) {
          best = ms;
          keep = v;
        }
      }
      c->opt.*p.field = keep;
      changed |= keep != start;
    }
    if (!changed) break;
  }
  out->ms_best = time_batch(c, items, k, cn);
  out->trials = trials;
  fill_result(c->opt, out);
}

}  // namespace kt

kt_status kt_autotune(kt_batch* b, uint32_t passes, kt_tune_result* out) {
  if (!b || !out) return KT_ERR_INVALID;
  kt_ctx* h = b->ctx;
  KT_API_BEGIN(h)
  if (b->items.empty()) throw kt::Error(KT_ERR_INVALID, "autotune: the sample batch is empty");
  kt::autotune(&h->c, b->items, passes, out);
  KT_API_END(h)
}

kt_status kt_options_save(kt_ctx* h, const char* path) {
  if (!path) return KT_ERR_INVALID;
  KT_API_BEGIN(h)
  cudaDeviceProp prop;
  KT_CUDA(cudaGetDeviceProperties(&prop, h->c.device));
  FILE* f = std::fopen(path, "w");
  if (!f) throw kt::Error(KT_ERR_IO, std::string("cannot write ") + path);
  std::fprintf(f, "# kt options, tuned on %s (%d SMs)\n", prop.name, prop.multiProcessorCount);
  for (const kt::Param& p : kt::params()) std::fprintf(f, "%s %lld\n", p.name, (long long)(h->c.opt.*p.field));
  const bool ok = std::fclose(f) == 0;
  if (!ok) throw kt::Error(KT_ERR_IO, std::string("cannot write ") + path);
  KT_API_END(h)
}

kt_status kt_options_load(kt_ctx* h, const char* path) {
  if (!path) return KT_ERR_INVALID;
  KT_API_BEGIN(h)
  FILE* f = std::fopen(path, "r");
  if (!f) throw kt::Error(KT_ERR_IO, std::string("cannot read ") + path);
  char line[256];
  kt::Options o = h->c.opt;
  while (std::fgets(line, sizeof(line), f)) {
    const char* first = line + std::strspn(line, " \t\r\n");
    if (*first == '#' || *first == '\0') continue;  // comments and blank (or CRLF) lines
    char name[128];
    long long v = 0;
    if (std::sscanf(line, "%127s %lld", name, &v) != 2) {
      std::fclose(f);
      throw kt::Error(KT_ERR_PARSE, std::string("options file: bad line: ") + line);
    }
    bool known = false;
    for (const kt::Param& p : kt::params())
      if (!std::strcmp(p.name, name)) {
        if (!kt::option_value_ok(name, v)) {
          std::fclose(f);
          throw kt::Error(KT_ERR_INVALID, std::string("options file: value out of range for ") + name);
        }
        o.*p.field = v;
        known = true;
      }
    if (!known) {
      std::fclose(f);
      throw kt::Error(KT_ERR_INVALID, std::string("options file: unknown option ") + name);
    }
  }
  std::fclose(f);
  h->c.opt = o;
  KT_API_END(h)
}
