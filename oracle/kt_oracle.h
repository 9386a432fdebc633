/* CPU oracle for the kmax-truss path.  TEST INFRASTRUCTURE ONLY: the tests,
 * the smoke check and the CPU baseline leg of the benchmark call it to check
 * or time the GPU solver; the solver never links or calls it.
 *
 * It restates, in plain serial C, what the reference solver computes
 * (caixiaofan/KC_CUDA, src/kc_cpu.cpp and src/kc_gpu.cpp), one function per
 * stage, each citing the reference lines it follows.  Stages use textbook
 * serial algorithms (bucket k-core, merge triangle counting, bucket truss
 * peeling) so that each result is exact and easy to audit; the reference's
 * pruning and step heuristics change only its running time, not its answer.
 */
#ifndef KT_ORACLE_H
#define KT_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Record grammar of the reference parser (kc_cpu.cpp:796-859,
 * kc_gpu.cpp:243-306).  A byte is a digit when, read as a signed char, it is
 * >= '0'; its value is byte - '0' (so letters count as large digits, and
 * bytes >= 0x80 are separators).  A line (bytes up to '\n') holding at least
 * one digit is a record: x = first digit run, y = second digit run, the rest
 * of the line is ignored; arithmetic wraps modulo 2^32.  Lines without
 * digits are skipped.  A record line with a single digit run is malformed;
 * it is reported (return -2, *bad_line = 0-based line index) instead of being
 * merged with the next line as the reference's scanner would do.
 * xy receives x << 32 | y per record; pass NULL to count only. */
int64_t kto_parse(const char* buf, uint64_t len, uint64_t* xy, uint64_t* bad_line);

/* The undirected simple graph of a record list: {x, y} for x != y, repeats
 * and reverse repeats merged.  On input in the reference's form (both
 * directions, no repeats, no self-loops) this is exactly the graph the
 * reference builds in init_graph (kc_cpu.cpp:61-90).  Writes sorted keys
 * u << 32 | v (u < v) into out (capacity >= count) and returns the number of
 * edges. */
uint64_t kto_clean(const uint64_t* xy, uint64_t count, uint64_t* out);

/* Core number of every vertex 0..n-1 (Batagelj-Zaversnik bucket order).
 * The reference's kmax_core (kc_cpu.cpp:185-251) returns the largest k with a
 * non-empty k-core, minus one; here c_max = max core[v]. */
void kto_core_numbers(uint32_t n, const uint64_t* edges, uint64_t m, uint32_t* core);

/* Triangles through each edge of the sorted edge list (kc_cpu.cpp:93-118
 * count_tc and 474-488 triangle_count; the reference stores 2x this). */
void kto_support(uint32_t n, const uint64_t* edges, uint64_t m, uint32_t* sup);

/* Trussness of each edge: the largest t such that the edge lies in the
 * t-truss (every edge of the t-truss is in >= t-2 of its triangles).  Edges
 * in no triangle get 2.  Serial bucket peeling in support order. */
void kto_trussness(uint32_t n, const uint64_t* edges, uint64_t m, uint32_t* truss);

/* The reference's answer (kc_cpu.cpp:703-710, 887): kmax = the largest
 * trussness and count = edges with that trussness, except that a graph with
 * no triangle answers kmax = 0, count = 0. */
void kto_kmax_from_truss(const uint32_t* truss, uint64_t m, uint32_t* kmax, uint64_t* count);

/* End to end: parse, clean, trussness, answer.  Returns 0, or the parse
 * error. */
int kto_solve_tsv(const char* buf, uint64_t len, uint32_t* kmax, uint64_t* count);

#ifdef __cplusplus
}
#endif
#endif
