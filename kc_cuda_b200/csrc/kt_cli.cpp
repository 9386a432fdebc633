// kt_solve: the drop-in command line of the reference solvers
// (src/kc_gpu.cpp:209-347, src/kc_cpu.cpp:763-893).
//
//   kt_solve -f <edge-list.tsv>          -> "kmax = K, Edges in kmax-truss = M."
//
// Same argument check and usage text (exit 1), same result line on stdout,
// and, like the reference, "mmap file error: ..." with exit status 255 when
// the file cannot be mapped (an empty file included).  Extensions, after the
// two reference arguments: --stats (stage timings to stderr), --device N.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "kt.h"

int main(int argc, char** argv) {
  if (argc < 3 || std::strcmp(argv[1], "-f") != 0) {
    std::fprintf(stderr, "Usage: -f [data_file_path]\n");
    return 1;
  }
  const char* path = argv[2];
  bool stats = false;
  int device = 0;
  for (int i = 3; i < argc; ++i) {
    if (!std::strcmp(argv[i], "--stats")) {
      stats = true;
    } else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) {
      device = std::atoi(argv[++i]);
    } else {
      std::fprintf(stderr, "Usage: -f [data_file_path]\n");
      return 1;
    }
  }
  kt_ctx* ctx = nullptr;
  kt_status s = kt_init(device, 0, &ctx);
  if (s != KT_OK) {
    std::fprintf(stderr, "GPUassert: %s\n", kt_status_string(s));
    return (int)s;
  }
  kt_graph* g = nullptr;
  s = kt_load_tsv_file(ctx, path, &g);
  if (s != KT_OK) {
    std::fprintf(stderr, "%s\n", kt_last_error(ctx));
    kt_destroy(ctx);
    return s == KT_ERR_IO ? 255 : (int)s;
  }
  uint32_t kmax = 0;
  uint64_t edges = 0;
  s = kt_solve(ctx, g, &kmax, &edges);
  if (s != KT_OK) {
    std::fprintf(stderr, "%s\n", kt_last_error(ctx));
    kt_graph_free(ctx, g);
    kt_destroy(ctx);
    return (int)s;
  }
  std::printf("kmax = %u, Edges in kmax-truss = %llu.\n", kmax, (unsigned long long)edges);
  if (stats) {
    kt_stats st;
    kt_get_stats(ctx, &st);
    std::fprintf(stderr,
                 "cmax %u  lower bound %u  predict %llu v / %llu e  search %llu v / %llu e  levels %u rounds %u\n"
                 "ms: kcore %.3f subgraph %.3f support %.3f peel %.3f  launches %llu  peak %.1f MB\n",
                 st.cmax, st.kmax_lower_bound, (unsigned long long)st.predict_vertices,
                 (unsigned long long)st.predict_edges, (unsigned long long)st.core_vertices,
                 (unsigned long long)st.core_edges, st.levels, st.rounds, st.ms_kcore, st.ms_subgraph, st.ms_support,
                 st.ms_peel, (unsigned long long)st.kernel_launches, st.device_bytes_peak / 1048576.0);
  }
  kt_graph_free(ctx, g);
  kt_destroy(ctx);
  return 0;
}
