// Host graph generator: draws, planted structure, cleaning and TSV output.
// The random conventions are in ktgen_core.h; this file only assembles them.
#include "ktgen.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ktgen_core.h"

struct ktg_graph {
  uint64_t n = 0;
  std::vector<uint64_t> edges;  // sorted unique u << 32 | v, u < v
};

namespace {

int clamp_threads(int t) {
  if (t <= 0) t = omp_get_max_threads();
  return t < 1 ? 1 : t;
}

// LSD radix sort of 64-bit keys, 8-bit digits; digits that every key shares
// are skipped.
void radix_sort_u64(std::vector<uint64_t>& a, int threads) {
  const size_t n = a.size();
  if (n < 2) return;
  std::vector<uint64_t> tmp(n);
  uint64_t* src = a.data();
  uint64_t* dst = tmp.data();
  const int T = threads;
  std::vector<size_t> hist((size_t)T * 256);
  for (int pass = 0; pass < 8; ++pass) {
    const int sh = pass * 8;
    std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(T)
    {
      const int t = omp_get_thread_num();
      const size_t lo = n * t / T, hi = n * (t + 1) / T;
      size_t* h = &hist[(size_t)t * 256];
      for (size_t i = lo; i < hi; ++i) h[(src[i] >> sh) & 255]++;
    }
    // Skip a digit that all keys share.
    size_t tot0 = 0;
    int nonzero = 0;
    for (int d = 0; d < 256; ++d) {
      size_t s = 0;
      for (int t = 0; t < T; ++t) s += hist[(size_t)t * 256 + d];
      if (s) nonzero++;
      (void)tot0;
    }
    if (nonzero <= 1) continue;
    size_t run = 0;
    for (int d = 0; d < 256; ++d)
      for (int t = 0; t < T; ++t) {
        const size_t c = hist[(size_t)t * 256 + d];
        hist[(size_t)t * 256 + d] = run;
        run += c;
      }
#pragma omp parallel num_threads(T)
    {
      const int t = omp_get_thread_num();
      const size_t lo = n * t / T, hi = n * (t + 1) / T;
      size_t* h = &hist[(size_t)t * 256];
      for (size_t i = lo; i < hi; ++i) dst[h[(src[i] >> sh) & 255]++] = src[i];
    }
    std::swap(src, dst);
  }
  if (src != a.data()) std::memcpy(a.data(), src, n * sizeof(uint64_t));
}

void add_clique(std::vector<uint64_t>& keys, const std::vector<uint32_t>& vs) {
  for (size_t i = 0; i < vs.size(); ++i)
    for (size_t j = i + 1; j < vs.size(); ++j) {
      const uint64_t a = vs[i], b = vs[j];
      keys.push_back(a < b ? (a << 32 | b) : (b << 32 | a));
    }
}

inline int ndigits(uint32_t x) {
  int d = 1;
  while (x >= 10) {
    x /= 10;
    ++d;
  }
  return d;
}

inline char* put_u32(char* p, uint32_t x) {
  char tmp[10];
  int k = 0;
  do {
    tmp[k++] = char('0' + x % 10);
    x /= 10;
  } while (x);
  while (k) *p++ = tmp[--k];
  return p;
}

// Symmetric CSR with ascending rows, from sorted canonical keys.
void build_sym_csr(const ktg_graph* g, std::vector<uint64_t>& off, std::vector<uint32_t>& col) {
  const uint64_t n = g->n;
  off.assign(n + 1, 0);
  for (uint64_t k : g->edges) {
    off[(k >> 32) + 1]++;
    off[(uint32_t)k + 1]++;
  }
  for (uint64_t i = 0; i < n; ++i) off[i + 1] += off[i];
  col.resize(off[n]);
  std::vector<uint64_t> cur(off.begin(), off.end() - 1);
  // Sorted by (u, v): row r receives its smaller neighbours (as v) before its
  // larger ones (as u), each in ascending order.
  for (uint64_t k : g->edges) {
    const uint32_t u = (uint32_t)(k >> 32), v = (uint32_t)k;
    col[cur[u]++] = v;
    col[cur[v]++] = u;
  }
}

std::string messy_text(const ktg_graph* g, uint64_t seed) {
  struct Line {
    uint64_t key;
    std::string s;
  };
  std::vector<Line> lines;
  const char* seps[] = {"\t", " ", ",", " \t", "\t\t"};
  uint64_t ctr = 0;
  auto emit = [&](uint32_t x, uint32_t y) {
    const uint64_t w = ktg_word(seed, 100, ctr++);
    std::string s = std::to_string(x);
    s += seps[ktg_below(w, 5)];
    s += std::to_string(y);
    if (((w >> 20) & 15) == 0) s += "\t1";  // an extra column
    s += (((w >> 24) & 7) == 0) ? "\r\n" : "\n";
    lines.push_back({ktg_word(seed, 101, ctr), s});
  };
  for (uint64_t i = 0; i < g->edges.size(); ++i) {
    const uint32_t u = (uint32_t)(g->edges[i] >> 32), v = (uint32_t)g->edges[i];
    const uint64_t r = ktg_below(ktg_word(seed, 102, i), 10);
    if (r < 5) {
      emit(u, v);
      emit(v, u);
    } else if (r < 7) {
      emit(u, v);
    } else if (r < 9) {
      emit(v, u);
    } else {
      emit(u, v);
      emit(v, u);
      emit(u, v);
    }
    if (ktg_below(ktg_word(seed, 103, i), 50) == 0) emit(u, u);
  }
  std::sort(lines.begin(), lines.end(), [](const Line& a, const Line& b) { return a.key < b.key; });
  std::string out;
  for (size_t i = 0; i < lines.size(); ++i) {
    if (i % 97 == 13) out += "\n";  // blank lines are skipped by the parsers
    out += lines[i].s;
  }
  return out;
}

}  // namespace

extern "C" {

int ktg_sample_vertices(uint64_t seed, uint64_t stream, uint64_t n, uint32_t size, uint32_t* out) {
  if (size > n) return -1;
  // Floyd: for j = n-size .. n-1, pick t in [0, j]; take t unless taken, else j.
  uint32_t k = 0;
  for (uint64_t j = n - size; j < n; ++j) {
    const uint64_t t = ktg_below(ktg_word(seed, stream, j - (n - size)), j + 1);
    bool seen = false;
    for (uint32_t q = 0; q < k; ++q)
      if (out[q] == t) {
        seen = true;
        break;
      }
    out[k++] = seen ? (uint32_t)j : (uint32_t)t;
  }
  return 0;
}

int ktg_mix_spec(uint64_t index, uint64_t base_seed, ktg_spec* out) {
  if (!out) return -1;
  std::memset(out, 0, sizeof(*out));
  const uint64_t w0 = ktg_word(base_seed, KTG_STREAM_MIX, 4 * index + 0);
  const uint64_t w1 = ktg_word(base_seed, KTG_STREAM_MIX, 4 * index + 1);
  const uint64_t w2 = ktg_word(base_seed, KTG_STREAM_MIX, 4 * index + 2);
  const uint64_t w3 = ktg_word(base_seed, KTG_STREAM_MIX, 4 * index + 3);
  const double u = (double)(w0 >> 11) * (1.0 / 9007199254740992.0);
  uint64_t n = (uint64_t)std::floor(1000.0 * std::pow(10.0, 3.0 * u));
  if (n < 1000) n = 1000;
  if (n > 1000000) n = 1000000;
  const uint64_t ef = 4 + ktg_below(w2, 61);
  out->kind = (w1 >> 63) ? KTG_ER : KTG_RMAT;
  out->n = n;
  uint32_t sc = 0;
  while ((1ULL << sc) < n) ++sc;
  out->scale = sc;
  out->draws = ef * n;
  out->seed = (base_seed << 20) | index;
  out->a_ppm = 570000;
  out->b_ppm = 190000;
  out->c_ppm = 190000;
  out->n_cliques = 1;
  out->clique_sizes[0] = (uint32_t)(5 + ktg_below(w3, 56));
  return 0;
}

int ktg_raw_draws(const ktg_spec* s, uint64_t first, uint64_t count, uint64_t* out) {
  if (!s) return -1;
  if (s->kind == KTG_RMAT) {
    const ktg_rmat_t t = ktg_rmat_thresholds(s->a_ppm, s->b_ppm, s->c_ppm);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)count; ++i) out[i] = ktg_rmat_draw(s->seed, t, s->scale, first + i);
    return 0;
  }
  if (s->kind == KTG_ER) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)count; ++i) out[i] = ktg_er_draw(s->seed, s->n, first + i);
    return 0;
  }
  return -1;
}

ktg_graph* ktg_make(const ktg_spec* s, int threads) {
  if (!s) return nullptr;
  const int T = clamp_threads(threads);
  uint64_t n = s->n;
  if (s->kind == KTG_RMAT) {
    if (s->scale == 0 || s->scale > 31) return nullptr;
    if (n == 0 || n > (1ULL << s->scale)) n = 1ULL << s->scale;
  }
  if (n == 0 || n > 0xffffffffULL) return nullptr;
  ktg_graph* g = new (std::nothrow) ktg_graph;
  if (!g) return nullptr;
  std::vector<uint64_t> keys;
  try {
    keys.resize(s->draws);
    if (s->kind == KTG_RMAT || s->kind == KTG_ER) {
      ktg_raw_draws(s, 0, s->draws, keys.data());
#pragma omp parallel for num_threads(T) schedule(static)
      for (int64_t i = 0; i < (int64_t)s->draws; ++i) keys[i] = ktg_canon(keys[i], n);
    } else if (s->kind == KTG_CHUNGLU) {
      // Expected degrees, then a fixed-point cumulative table; endpoints are
      // found by binary search, so host and device agree exactly.
      std::vector<uint64_t> cdf(n + 1, 0);
      const double ex = -1.0 / (s->cl_gamma - 1.0);
      for (uint64_t i = 0; i < n; ++i) {
        const uint64_t w = ktg_word(s->seed, KTG_STREAM_CL_WEIGHT, i);
        const double u = (double)((w >> 11) + 1) * (1.0 / 9007199254740992.0);
        double wt = s->cl_w_min * std::pow(u, ex);
        if (wt > s->cl_w_max) wt = s->cl_w_max;
        cdf[i + 1] = cdf[i] + (uint64_t)std::llround(wt * 1024.0);
      }
      const uint64_t tot = cdf[n];
#pragma omp parallel for num_threads(T) schedule(static)
      for (int64_t i = 0; i < (int64_t)s->draws; ++i) {
        const uint64_t a = ktg_below(ktg_word(s->seed, KTG_STREAM_CL_EDGE, 2 * i), tot);
        const uint64_t b = ktg_below(ktg_word(s->seed, KTG_STREAM_CL_EDGE, 2 * i + 1), tot);
        const uint64_t x = (uint64_t)(std::upper_bound(cdf.begin(), cdf.end(), a) - cdf.begin()) - 1;
        const uint64_t y = (uint64_t)(std::upper_bound(cdf.begin(), cdf.end(), b) - cdf.begin()) - 1;
        keys[i] = ktg_canon((x << 32) | y, n);
      }
    } else {
      delete g;
      return nullptr;
    }
    for (uint32_t c = 0; c < s->n_cliques && c < 8; ++c) {
      const uint32_t sz = s->clique_sizes[c];
      if (sz > n) {
        delete g;
        return nullptr;
      }
      std::vector<uint32_t> vs(sz);
      ktg_sample_vertices(s->seed, KTG_STREAM_CLIQUE + c, n, sz, vs.data());
      add_clique(keys, vs);
    }
    if (s->block_size) {
      if (s->block_size > n) {
        delete g;
        return nullptr;
      }
      std::vector<uint32_t> vs(s->block_size);
      ktg_sample_vertices(s->seed, KTG_STREAM_CLIQUE + 31, n, s->block_size, vs.data());
      const uint64_t thr = ((uint64_t)s->block_p_ppm << 32) / 1000000ULL;
      uint64_t pair = 0;
      for (size_t i = 0; i < vs.size(); ++i)
        for (size_t j = i + 1; j < vs.size(); ++j, ++pair) {
          if ((ktg_word(s->seed, KTG_STREAM_BLOCK, pair) & 0xffffffffULL) >= thr) continue;
          const uint64_t a = vs[i], b = vs[j];
          keys.push_back(a < b ? (a << 32 | b) : (b << 32 | a));
        }
    }
    radix_sort_u64(keys, T);
    size_t m = 0;
    for (size_t i = 0; i < keys.size(); ++i) {
      if (keys[i] == ~0ULL) break;
      if (m == 0 || keys[i] != keys[m - 1]) keys[m++] = keys[i];
    }
    keys.resize(m);
    keys.shrink_to_fit();
  } catch (...) {
    delete g;
    return nullptr;
  }
  uint64_t mx = 0;
  for (uint64_t k : keys) mx = std::max<uint64_t>(mx, (uint32_t)k);
  g->n = keys.empty() ? 0 : mx + 1;
  g->edges.swap(keys);
  return g;
}

void ktg_free(ktg_graph* g) { delete g; }
uint64_t ktg_num_vertices(const ktg_graph* g) { return g ? g->n : 0; }
uint64_t ktg_num_edges(const ktg_graph* g) { return g ? g->edges.size() : 0; }
const uint64_t* ktg_edges(const ktg_graph* g) { return g ? g->edges.data() : nullptr; }

uint64_t ktg_tsv_size(const ktg_graph* g, int mode, uint64_t mess_seed) {
  if (!g) return 0;
  if (mode == 1) return messy_text(g, mess_seed).size();
  uint64_t tot = 0;
#pragma omp parallel for reduction(+ : tot) schedule(static)
  for (int64_t i = 0; i < (int64_t)g->edges.size(); ++i) {
    const uint32_t u = (uint32_t)(g->edges[i] >> 32), v = (uint32_t)g->edges[i];
    tot += 2 * (uint64_t)(ndigits(u) + ndigits(v) + 2);
  }
  return tot;
}

uint64_t ktg_tsv_fill(const ktg_graph* g, int mode, uint64_t mess_seed, char* buf, int threads) {
  if (!g || !buf) return 0;
  if (mode == 1) {
    const std::string s = messy_text(g, mess_seed);
    std::memcpy(buf, s.data(), s.size());
    return s.size();
  }
  const int T = clamp_threads(threads);
  std::vector<uint64_t> off;
  std::vector<uint32_t> col;
  build_sym_csr(g, off, col);
  const uint64_t n = g->n;
  // Byte offset of each row group "x\ty\n" for the rows keyed by y.
  std::vector<uint64_t> boff(n + 1, 0);
#pragma omp parallel for num_threads(T) schedule(dynamic, 4096)
  for (int64_t y = 0; y < (int64_t)n; ++y) {
    uint64_t b = 0;
    const int dy = ndigits((uint32_t)y) + 2;
    for (uint64_t j = off[y]; j < off[y + 1]; ++j) b += ndigits(col[j]) + dy;
    boff[y + 1] = b;
  }
  for (uint64_t y = 0; y < n; ++y) boff[y + 1] += boff[y];
#pragma omp parallel for num_threads(T) schedule(dynamic, 4096)
  for (int64_t y = 0; y < (int64_t)n; ++y) {
    char* p = buf + boff[y];
    for (uint64_t j = off[y]; j < off[y + 1]; ++j) {
      p = put_u32(p, col[j]);
      *p++ = '\t';
      p = put_u32(p, (uint32_t)y);
      *p++ = '\n';
    }
  }
  return boff[n];
}

int ktg_tsv_write(const ktg_graph* g, int mode, uint64_t mess_seed, const char* path, int threads) {
  if (!g || !path) return -1;
  const uint64_t sz = ktg_tsv_size(g, mode, mess_seed);
  std::vector<char> buf(sz);
  const uint64_t w = ktg_tsv_fill(g, mode, mess_seed, buf.data(), threads);
  FILE* f = std::fopen(path, "wb");
  if (!f) return -2;
  const size_t put = w ? std::fwrite(buf.data(), 1, w, f) : 0;
  const int rc = std::fclose(f);
  return (put == w && rc == 0) ? 0 : -3;
}

}  // extern "C"
