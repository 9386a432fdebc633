// Stage entry points shared between the solver's translation units.
#pragma once
#include "kt_device.cuh"
#include "kt_internal.h"

namespace kt {

void scan_u64(Ctx* c, const uint64_t* in, uint64_t* out, uint64_t n);

// parse.cu -- stage (a)
uint64_t parse_padded_bytes(uint64_t len);
// Bytes per parse block; a chunk of the input for the pipelined ingest is a
// whole number of blocks.
uint64_t parse_block_bytes();
// Lines of blocks [block0, block0 + nblocks) (~0: to the end); block_off
// receives their exclusive scan (relative to the first of them).
uint64_t parse_count_lines(Ctx* c, const uint8_t* dbuf, uint64_t len, DBuf& block_off, uint64_t block0 = 0,
                           uint64_t nblocks = ~0ULL);
// Parses those blocks' lines into keys[block_off[b] + i].  Bytes at or past
// `ready` (~0: len) are not yet on the device: a line that needs one sets
// DevWords::counters[2] (its record must be redone).  line_base numbers the
// lines for parse errors.
void parse_lines(Ctx* c, const uint8_t* dbuf, uint64_t len, const DBuf& block_off, uint64_t* keys, DevWords* words,
                 uint64_t block0 = 0, uint64_t nblocks = ~0ULL, uint64_t ready = ~0ULL, uint64_t line_base = 0);

// csr.cu -- stage (b): edge records a << 32 | b (either end first, any
// order, ~0 = none) -> Graph.  `keys` may be consumed (sorted in place).
// `lines`: the records are a TSV's lines in file order (y << 32 | x), so the
// grouped-input route is tried first.
// lines: the keys are parsed lines (tried in the grouped form first);
// sorted: the keys are canonical, ascending and distinct (checked on the
// device; the sort is skipped when they are).
void build_graph(Ctx* c, uint64_t* keys, uint64_t nkeys, uint64_t n, Graph& g, bool lines = false,
                 bool sorted = false);

DevWords* dev_words(Ctx* c);
void reset_words(Ctx* c);
// Throws the error a kernel flagged in the device words (if any).
void check_words(Ctx* c, const char* stage);

}  // namespace kt
