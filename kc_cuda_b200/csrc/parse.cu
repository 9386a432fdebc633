// Stage (a): TSV bytes on the device -> one edge record per line.
//
// The grammar is the reference parser's (src/kc_gpu.cpp:243-306): a byte is
// a digit when, read as a signed char, it is >= '0', and contributes
// byte - '0'; a line's first two digit runs are x and y and the rest of the
// line is ignored; lines without digits are skipped.  A line holding one
// digit run is an error here (the reference would silently merge it with
// the next line).
//
// Layout: each thread owns a 36-byte chunk (9 words, so the 32 chunk starts
// of a warp fall on distinct shared-memory banks); a line belongs to the
// thread whose chunk holds the '\n' before it (line 0 belongs to thread 0).
// Pass 1 counts lines per 9 KB block with 16-byte loads; after a scan, pass 2
// stages the block's bytes (plus a 1 KB overhang) in shared memory, finds the
// chunk's newlines a word at a time (__vcmpeq4), lists the block's line
// starts in shared memory, and deals the lines round-robin to the threads;
// line i of the block goes to slot block_offset + i.  A slot gets the record
// y << 32 | x (the grouping column high), or ~0 for a blank line or a
// self-loop; the CSR build reads the records in line order (grouped input)
// or canonicalises them to min << 32 | max for its sort.
#include "kt_device.cuh"
#include "kt_internal.h"
#include "stages.h"

namespace kt {
namespace {

constexpr unsigned kParseThreads = 256;
constexpr unsigned kChunk = 36;  // 9 words: chunk starts fall on distinct smem banks
constexpr unsigned kBlockBytes = kParseThreads * kChunk;  // 9216 (a multiple of 16)
constexpr unsigned kOverhang = 1024;

__device__ __forceinline__ uint32_t count_nl4(uint32_t w) { return __popc(__vcmpeq4(w, 0x0a0a0a0au)) >> 3; }

// Lines owned by a block: its '\n' bytes except one at len-1, plus line 0.
__global__ void __launch_bounds__(kParseThreads) k_count_lines(const uint8_t* __restrict__ buf, uint64_t len,
                                                               uint64_t block0, uint32_t* __restrict__ block_lines) {
  __shared__ uint32_t tmp[33];
  const uint64_t b = block0 + blockIdx.x;
  const uint64_t blo = b * kBlockBytes;
  const uint64_t bhi = min(len, blo + kBlockBytes);
  const uint64_t nvec = (bhi - blo + 15) / 16;  // the padding past len is zero
  uint32_t c = 0;
  for (uint64_t i = threadIdx.x; i < nvec; i += kParseThreads) {
    const uint4 v = reinterpret_cast<const uint4*>(buf + blo)[i];
    c += count_nl4(v.x) + count_nl4(v.y) + count_nl4(v.z) + count_nl4(v.w);
  }
  c = block_sum<uint32_t>(c, tmp);
  if (threadIdx.x == 0) {
    if (bhi == len && len > 0 && buf[len - 1] == '\n') c -= 1;
    if (b == 0 && len > 0) c += 1;
    block_lines[blockIdx.x] = c;
  }
}

__device__ __forceinline__ bool is_digit(int b) { return b >= '0' && b < 128; }

struct Bytes {
  const uint8_t* sm;  // staged bytes [lo, hi)
  const uint8_t* g;   // global buffer
  uint64_t lo, hi, len;
  uint64_t ready;     // bytes [0, ready) of the buffer are on the device
  uint32_t* deferred; // set when a line reads past `ready` (its record is then redone)
  __device__ __forceinline__ int at(uint64_t q) const {  // -1 past the end
    if (q >= len) return -1;
    if (q < hi) return sm[q - lo];
    if (q >= ready) {
      *deferred = 1u;
      return -1;
    }
    return g[q];
  }
};

// The line at `start`: ~0 for a blank line or a self-loop, y << 32 | x
// otherwise; *bad when it holds a single number.
__device__ __forceinline__ uint64_t parse_line(const Bytes& B, uint64_t p, bool* bad, uint32_t* vmax) {
  int b = B.at(p);
  while (b >= 0 && b != '\n' && !is_digit(b)) b = B.at(++p);
  if (!is_digit(b)) return ~0ull;
  uint32_t x = 0, y = 0;
  while (is_digit(b)) {
    x = x * 10u + (uint32_t)(b - '0');
    b = B.at(++p);
  }
  while (b >= 0 && b != '\n' && !is_digit(b)) b = B.at(++p);
  if (!is_digit(b)) {
    *bad = true;
    return ~0ull;
  }
  while (is_digit(b)) {
    y = y * 10u + (uint32_t)(b - '0');
    b = B.at(++p);
  }
  *vmax = max(*vmax, max(x, y));
  return x == y ? ~0ull : (((uint64_t)y << 32) | x);
}

// The same parse from the staged words held in a register window: one
// shared-memory load per 4 bytes and no per-byte range test other than
// p < lim.  Returns false (and the caller parses the line with parse_line)
// when the line's first two numbers reach past lim = min(len, staged end).
__device__ __forceinline__ bool parse_line_fast(const uint32_t* stage, uint64_t blo, uint64_t lim, uint64_t p,
                                                uint64_t* key, bool* bad, uint32_t* vmax) {
  if (p >= lim) return false;
  const uint32_t off = (uint32_t)(p - blo);
  uint32_t q = off >> 2;
  uint32_t cur = stage[q] >> (8 * (off & 3));
  uint32_t nb = 4 - (off & 3);
  uint32_t b = cur & 0xffu;
  // Next byte into b; false past lim.
#define KT_ADV()                 \
  do {                           \
    if (++p >= lim) return false; \
    if (--nb == 0) {             \
      cur = stage[++q];          \
      nb = 4;                    \
    } else {                     \
      cur >>= 8;                 \
    }                            \
    b = cur & 0xffu;             \
  } while (0)
#define KT_DIGIT(x) ((uint32_t)((x) - 0x30u) < 0x50u)  // signed char >= '0'
  while (b != '\n' && !KT_DIGIT(b)) KT_ADV();
  if (!KT_DIGIT(b)) {
    *key = ~0ull;
    return true;
  }
  uint32_t x = 0, y = 0;
  while (KT_DIGIT(b)) {
    x = x * 10u + (b - 0x30u);
    KT_ADV();
  }
  while (b != '\n' && !KT_DIGIT(b)) KT_ADV();
  if (!KT_DIGIT(b)) {
    *bad = true;
    *key = ~0ull;
    return true;
  }
  while (KT_DIGIT(b)) {
    y = y * 10u + (b - 0x30u);
    KT_ADV();
  }
#undef KT_ADV
#undef KT_DIGIT
  *vmax = max(*vmax, max(x, y));
  *key = x == y ? ~0ull : (((uint64_t)y << 32) | x);
  return true;
}

// Phase 1 finds the block's line starts (newlines a word at a time, a block
// scan, offsets into shared memory); phase 2 deals the lines round-robin to
// the threads, so the per-line work is balanced and the keys are written
// with consecutive threads on consecutive slots.
__global__ void __launch_bounds__(kParseThreads) k_parse_lines(const uint8_t* __restrict__ buf, uint64_t len,
                                                               uint64_t block0, uint64_t ready, uint64_t line_base,
                                                               const uint64_t* __restrict__ block_off,
                                                               uint64_t* __restrict__ keys, DevWords* words) {
  __shared__ __align__(16) uint32_t stage[(kBlockBytes + kOverhang) / 4];
  __shared__ uint16_t starts[kBlockBytes + 1];
  __shared__ uint32_t tmp[33];
  __shared__ __align__(8) uint64_t stage_bar;
  const uint64_t blo = (block0 + blockIdx.x) * kBlockBytes;
  const uint64_t bhi = min(len, blo + kBlockBytes + kOverhang);
  // The device buffer is padded (zeros) to whole 16-byte words past len; the
  // block's bytes come in as one bulk copy (blo is a multiple of 16).
  const uint64_t nvec = (bhi - blo + 15) / 16;
  const bool staged = bulk_load_to_shared(stage, buf + blo, (uint32_t)(nvec * 16), &stage_bar, &words->err);
  if (__syncthreads_or(!staged)) return;

  const uint64_t s = blo + (uint64_t)threadIdx.x * kChunk;
  const uint64_t e = min(len, s + kChunk);
  // Owned lines: one per '\n' in [s, e) that is not the last byte, plus line 0.
  uint32_t nlmask[kChunk / 4];
  uint32_t c = 0;
#pragma unroll
  for (uint32_t j = 0; j < kChunk / 4; ++j) {
    const uint64_t a = s + 4 * j;
    uint32_t m = 0;
    if (a < e) {
      m = __vcmpeq4(stage[(a - blo) >> 2], 0x0a0a0a0au);
      // Drop bytes at or past e, and a '\n' at len-1 (it starts no line).
      const uint64_t lim = min(e, len - 1);
      if (a + 4 > lim) m &= lim > a ? (0xffffffffu >> (8 * (4 - (uint32_t)(lim - a)))) : 0u;
    }
    nlmask[j] = m;
    c += __popc(m) >> 3;
  }
  const bool first = (s == 0 && len > 0);
  if (first) c += 1;
  uint32_t total;
  uint32_t pos = block_excl_scan<uint32_t>(c, tmp, &total);
  if (first) starts[pos++] = 0;
#pragma unroll
  for (uint32_t j = 0; j < kChunk / 4; ++j) {
    uint32_t m = nlmask[j];
    while (m) {
      const uint32_t k = (__ffs(m) - 1) >> 3;
      m &= ~(0xffu << (8 * k));
      starts[pos++] = (uint16_t)(s + 4 * j + k + 1 - blo);
    }
  }
  __syncthreads();
  const Bytes B{reinterpret_cast<const uint8_t*>(stage), buf, blo, blo + nvec * 16, len, ready,
                reinterpret_cast<uint32_t*>(&words->counters[2])};
  const uint64_t slot0 = block_off[blockIdx.x];
  uint32_t vmax = 0;
  bool any = false;
  const uint64_t lim = min(len, blo + nvec * 16);
  for (uint32_t i = threadIdx.x; i < total; i += kParseThreads) {
    bool bad = false;
    uint64_t key;
    if (!parse_line_fast(stage, blo, lim, blo + starts[i], &key, &bad, &vmax)) {
      bad = false;
      key = parse_line(B, blo + starts[i], &bad, &vmax);
    }
    if (bad) {
      atomicOr(&words->err, kDevErrParse);
      atomicMin(&words->bad_line, (unsigned long long)(line_base + slot0 + i));
    }
    any = true;
    keys[slot0 + i] = key;
  }
  vmax = warp_max(vmax);
  const unsigned anyw = __ballot_sync(kFull, any);
  if (lane_id() == 0 && anyw) {
    atomicMax(reinterpret_cast<unsigned int*>(&words->counters[0]), vmax);
    atomicOr(reinterpret_cast<unsigned int*>(&words->counters[1]), 1u);
  }
}

}  // namespace

uint64_t parse_block_bytes() { return kBlockBytes; }

uint64_t parse_count_lines(Ctx* c, const uint8_t* dbuf, uint64_t len, DBuf& block_off, uint64_t block0,
                           uint64_t nblocks) {
  const uint64_t total = (len + kBlockBytes - 1) / kBlockBytes;
  if (total > 0x7fffffffULL) throw Error(KT_ERR_LIMIT, "TSV larger than the parser's grid");
  const uint64_t blocks = nblocks == ~0ULL ? total - block0 : nblocks;
  if (blocks == 0) return 0;
  DBuf cnt(c, (blocks + 1) * sizeof(uint32_t));
  k_count_lines<<<(unsigned)blocks, kParseThreads, 0, c->stream>>>(dbuf, len, block0, cnt.as<uint32_t>());
  KT_LAUNCHED(c);
  zero(c, cnt.as<uint32_t>() + blocks, sizeof(uint32_t));
  block_off.ensure(c, (blocks + 1) * sizeof(uint64_t));
  scan_u32_to_u64(c, cnt.as<uint32_t>(), block_off.as<uint64_t>(), blocks + 1);
  return read_word<uint64_t>(c, block_off.as<uint64_t>() + blocks);
}

void parse_lines(Ctx* c, const uint8_t* dbuf, uint64_t len, const DBuf& block_off, uint64_t* keys, DevWords* words,
                 uint64_t block0, uint64_t nblocks, uint64_t ready, uint64_t line_base) {
  const uint64_t total = (len + kBlockBytes - 1) / kBlockBytes;
  const uint64_t blocks = nblocks == ~0ULL ? total - block0 : nblocks;
  if (blocks == 0) return;
  k_parse_lines<<<(unsigned)blocks, kParseThreads, 0, c->stream>>>(dbuf, len, block0, ready == ~0ULL ? len : ready,
                                                                   line_base, block_off.as<uint64_t>(), keys, words);
  KT_LAUNCHED(c);
}

uint64_t parse_padded_bytes(uint64_t len) { return ((len + 15) / 16) * 16 + kOverhang + 16; }

}  // namespace kt
