/* CPU oracle for the kmax-truss path (TEST INFRASTRUCTURE ONLY; see
 * kt_oracle.h).  Serial, exact, plain C11. */
#include "kt_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ parse */

static int is_digit_byte(char b) { return (signed char)b >= '0'; }

/* kc_cpu.cpp:816-834 (x run, separators, y run, rest of line). */
int64_t kto_parse(const char* buf, uint64_t len, uint64_t* xy, uint64_t* bad_line) {
  uint64_t i = 0, line = 0;
  int64_t rec = 0;
  while (i < len) {
    uint64_t e = i;
    while (e < len && buf[e] != '\n') ++e;
    uint64_t j = i;
    while (j < e && !is_digit_byte(buf[j])) ++j;
    if (j < e) {
      uint32_t x = 0, y = 0;
      while (j < e && is_digit_byte(buf[j])) {
        x = x * 10u + (uint32_t)((int)(signed char)buf[j] - '0');
        ++j;
      }
      while (j < e && !is_digit_byte(buf[j])) ++j;
      if (j >= e) {
        if (bad_line) *bad_line = line;
        return -2;
      }
      while (j < e && is_digit_byte(buf[j])) {
        y = y * 10u + (uint32_t)((int)(signed char)buf[j] - '0');
        ++j;
      }
      if (xy) xy[rec] = ((uint64_t)x << 32) | y;
      ++rec;
    }
    i = e + 1;
    ++line;
  }
  return rec;
}

/* ------------------------------------------------------------------ clean */

static void radix_sort(uint64_t* a, uint64_t n) {
  uint64_t* tmp = (uint64_t*)malloc((n ? n : 1) * sizeof(uint64_t));
  uint64_t* src = a;
  uint64_t* dst = tmp;
  for (int pass = 0; pass < 8; ++pass) {
    uint64_t cnt[257];
    memset(cnt, 0, sizeof(cnt));
    const int sh = pass * 8;
    for (uint64_t i = 0; i < n; ++i) cnt[((src[i] >> sh) & 255) + 1]++;
    int distinct = 0;
    for (int d = 1; d <= 256; ++d) distinct += cnt[d] != 0;
    if (distinct <= 1) continue;
    for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
    for (uint64_t i = 0; i < n; ++i) dst[cnt[(src[i] >> sh) & 255]++] = src[i];
    uint64_t* t = src;
    src = dst;
    dst = t;
  }
  if (src != a) memcpy(a, src, n * sizeof(uint64_t));
  free(tmp);
}

uint64_t kto_clean(const uint64_t* xy, uint64_t count, uint64_t* out) {
  uint64_t k = 0;
  for (uint64_t i = 0; i < count; ++i) {
    const uint32_t x = (uint32_t)(xy[i] >> 32), y = (uint32_t)xy[i];
    if (x == y) continue;
    out[k++] = x < y ? (((uint64_t)x << 32) | y) : (((uint64_t)y << 32) | x);
  }
  radix_sort(out, k);
  uint64_t m = 0;
  for (uint64_t i = 0; i < k; ++i)
    if (m == 0 || out[i] != out[m - 1]) out[m++] = out[i];
  return m;
}

/* ---------------------------------------------------- symmetric CSR + ids */

typedef struct {
  uint32_t n;
  uint64_t* off; /* n + 1 */
  uint32_t* adj; /* 2m, ascending per row */
  uint64_t* eid; /* 2m, id of the undirected edge of each entry */
} csr_t;

static void csr_build(uint32_t n, const uint64_t* edges, uint64_t m, csr_t* g) {
  g->n = n;
  g->off = (uint64_t*)calloc((size_t)n + 1, sizeof(uint64_t));
  const uint64_t cap = m > 0 ? 2 * m : 1;
  g->adj = (uint32_t*)malloc(cap * sizeof(uint32_t));
  g->eid = (uint64_t*)malloc(cap * sizeof(uint64_t));
  for (uint64_t i = 0; i < m; ++i) {
    g->off[(edges[i] >> 32) + 1]++;
    g->off[(uint32_t)edges[i] + 1]++;
  }
  for (uint32_t v = 0; v < n; ++v) g->off[v + 1] += g->off[v];
  uint64_t* cur = (uint64_t*)malloc(((size_t)n + 1) * sizeof(uint64_t));
  memcpy(cur, g->off, ((size_t)n + 1) * sizeof(uint64_t));
  /* Edges sorted by (u, v): each row gets its smaller neighbours first, then
   * its larger ones, both ascending. */
  for (uint64_t i = 0; i < m; ++i) {
    const uint32_t u = (uint32_t)(edges[i] >> 32), v = (uint32_t)edges[i];
    g->adj[cur[u]] = v;
    g->eid[cur[u]++] = i;
    g->adj[cur[v]] = u;
    g->eid[cur[v]++] = i;
  }
  free(cur);
}

static void csr_free(csr_t* g) {
  free(g->off);
  free(g->adj);
  free(g->eid);
}

static uint32_t max_vertex(const uint64_t* edges, uint64_t m) {
  uint32_t mx = 0;
  for (uint64_t i = 0; i < m; ++i)
    if ((uint32_t)edges[i] > mx) mx = (uint32_t)edges[i];
  return mx;
}

/* Position of w in row u, or -1. */
static int64_t find_in_row(const csr_t* g, uint32_t u, uint32_t w) {
  uint64_t lo = g->off[u], hi = g->off[u + 1];
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo) / 2;
    if (g->adj[mid] < w)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < g->off[u + 1] && g->adj[lo] == w) ? (int64_t)lo : -1;
}

/* --------------------------------------------------------------- k-core */

void kto_core_numbers(uint32_t n, const uint64_t* edges, uint64_t m, uint32_t* core) {
  if (n == 0) return;
  csr_t g;
  csr_build(n, edges, m, &g);
  uint32_t md = 0;
  uint32_t* deg = (uint32_t*)malloc(n * sizeof(uint32_t));
  for (uint32_t v = 0; v < n; ++v) {
    deg[v] = (uint32_t)(g.off[v + 1] - g.off[v]);
    if (deg[v] > md) md = deg[v];
  }
  uint32_t* bin = (uint32_t*)calloc((size_t)md + 2, sizeof(uint32_t));
  uint32_t* pos = (uint32_t*)malloc(n * sizeof(uint32_t));
  uint32_t* vert = (uint32_t*)malloc(n * sizeof(uint32_t));
  for (uint32_t v = 0; v < n; ++v) bin[deg[v]]++;
  uint32_t start = 0;
  for (uint32_t d = 0; d <= md; ++d) {
    const uint32_t c = bin[d];
    bin[d] = start;
    start += c;
  }
  for (uint32_t v = 0; v < n; ++v) {
    pos[v] = bin[deg[v]]++;
    vert[pos[v]] = v;
  }
  for (uint32_t d = md; d >= 1; --d) bin[d] = bin[d - 1];
  bin[0] = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t v = vert[i];
    for (uint64_t j = g.off[v]; j < g.off[v + 1]; ++j) {
      const uint32_t u = g.adj[j];
      if (deg[u] > deg[v]) {
        const uint32_t du = deg[u], pu = pos[u], pw = bin[du], w = vert[pw];
        if (u != w) {
          pos[u] = pw;
          vert[pu] = w;
          pos[w] = pu;
          vert[pw] = u;
        }
        bin[du]++;
        deg[u]--;
      }
    }
  }
  memcpy(core, deg, n * sizeof(uint32_t));
  free(bin);
  free(pos);
  free(vert);
  free(deg);
  csr_free(&g);
}

/* -------------------------------------------------------------- support */

void kto_support(uint32_t n, const uint64_t* edges, uint64_t m, uint32_t* sup) {
  (void)n;
  if (m == 0) return;
  const uint32_t nv = max_vertex(edges, m) + 1;
  csr_t g;
  csr_build(nv, edges, m, &g);
  /* For each vertex u, mark N(u); every edge (u, v) whose other end v has the
   * smaller list (ties: smaller id) is counted from u by scanning N(v). */
  unsigned char* mark = (unsigned char*)calloc(nv, 1);
  for (uint32_t u = 0; u < nv; ++u) {
    const uint64_t du = g.off[u + 1] - g.off[u];
    for (uint64_t j = g.off[u]; j < g.off[u + 1]; ++j) mark[g.adj[j]] = 1;
    for (uint64_t j = g.off[u]; j < g.off[u + 1]; ++j) {
      const uint32_t v = g.adj[j];
      const uint64_t dv = g.off[v + 1] - g.off[v];
      if (dv > du || (dv == du && v > u)) continue;
      uint32_t c = 0;
      for (uint64_t q = g.off[v]; q < g.off[v + 1]; ++q) c += mark[g.adj[q]];
      sup[g.eid[j]] = c;
    }
    for (uint64_t j = g.off[u]; j < g.off[u + 1]; ++j) mark[g.adj[j]] = 0;
  }
  free(mark);
  csr_free(&g);
}

/* ---------------------------------------------------------------- truss */

void kto_trussness(uint32_t n, const uint64_t* edges, uint64_t m, uint32_t* truss) {
  (void)n;
  if (m == 0) return;
  const uint32_t nv = max_vertex(edges, m) + 1;
  csr_t g;
  csr_build(nv, edges, m, &g);
  uint32_t* sup = (uint32_t*)malloc(m * sizeof(uint32_t));
  kto_support(nv, edges, m, sup);
  uint32_t ms = 0;
  for (uint64_t e = 0; e < m; ++e)
    if (sup[e] > ms) ms = sup[e];
  /* Edges bucketed by current support (bin sort, as for the k-core). */
  uint64_t* bin = (uint64_t*)calloc((size_t)ms + 2, sizeof(uint64_t));
  uint64_t* pos = (uint64_t*)malloc(m * sizeof(uint64_t));
  uint64_t* order = (uint64_t*)malloc(m * sizeof(uint64_t));
  unsigned char* dead = (unsigned char*)calloc(m, 1);
  for (uint64_t e = 0; e < m; ++e) bin[sup[e]]++;
  uint64_t start = 0;
  for (uint32_t s = 0; s <= ms; ++s) {
    const uint64_t c = bin[s];
    bin[s] = start;
    start += c;
  }
  for (uint64_t e = 0; e < m; ++e) {
    pos[e] = bin[sup[e]]++;
    order[pos[e]] = e;
  }
  for (uint32_t s = ms; s >= 1; --s) bin[s] = bin[s - 1];
  bin[0] = 0;
  uint32_t level = 0;
  for (uint64_t i = 0; i < m; ++i) {
    const uint64_t e = order[i];
    if (sup[e] > level) level = sup[e];
    truss[e] = level + 2;
    dead[e] = 1;
    uint32_t u = (uint32_t)(edges[e] >> 32), v = (uint32_t)edges[e];
    if (g.off[u + 1] - g.off[u] > g.off[v + 1] - g.off[v]) {
      const uint32_t t = u;
      u = v;
      v = t;
    }
    for (uint64_t j = g.off[u]; j < g.off[u + 1]; ++j) {
      const uint64_t a = g.eid[j];
      if (dead[a]) continue;
      const int64_t q = find_in_row(&g, v, g.adj[j]);
      if (q < 0) continue;
      const uint64_t b = g.eid[q];
      if (dead[b]) continue;
      const uint64_t pair[2] = {a, b};
      for (int t = 0; t < 2; ++t) {
        const uint64_t x = pair[t];
        if (sup[x] > level) {
          /* Move x to the front of its bucket, then shrink the bucket. */
          const uint32_t sx = sup[x];
          const uint64_t px = pos[x], pw = bin[sx], w = order[pw];
          if (x != w) {
            pos[x] = pw;
            order[px] = w;
            pos[w] = px;
            order[pw] = x;
          }
          bin[sx]++;
          sup[x]--;
        }
      }
    }
  }
  free(bin);
  free(pos);
  free(order);
  free(dead);
  free(sup);
  csr_free(&g);
}

void kto_kmax_from_truss(const uint32_t* truss, uint64_t m, uint32_t* kmax, uint64_t* count) {
  uint32_t k = 0;
  uint64_t c = 0;
  for (uint64_t e = 0; e < m; ++e) {
    if (truss[e] > k) {
      k = truss[e];
      c = 0;
    }
    if (truss[e] == k) ++c;
  }
  if (k < 3) { /* no triangle: kc_cpu.cpp:703-710 never records a level */
    k = 0;
    c = 0;
  }
  *kmax = k;
  *count = c;
}

int kto_solve_tsv(const char* buf, uint64_t len, uint32_t* kmax, uint64_t* count) {
  uint64_t bad = 0;
  const int64_t r = kto_parse(buf, len, NULL, &bad);
  if (r < 0) return (int)r;
  uint64_t* xy = (uint64_t*)malloc((r ? r : 1) * sizeof(uint64_t));
  kto_parse(buf, len, xy, &bad);
  uint64_t* e = (uint64_t*)malloc((r ? r : 1) * sizeof(uint64_t));
  const uint64_t m = kto_clean(xy, (uint64_t)r, e);
  free(xy);
  uint32_t* t = (uint32_t*)malloc((m ? m : 1) * sizeof(uint32_t));
  kto_trussness(0, e, m, t);
  kto_kmax_from_truss(t, m, kmax, count);
  free(t);
  free(e);
  return 0;
}
