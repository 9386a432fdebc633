// Stage (a): TSV bytes on the device -> one canonical edge key per line.
//
// The grammar is the reference parser's (src/kc_gpu.cpp:243-306): a byte is
// a digit when, read as a signed char, it is >= '0', and contributes
// byte - '0'; a line's first two digit runs are x and y and the rest of the
// line is ignored; lines without digits are skipped.  A line holding one
// digit run is an error here (the reference would silently merge it with
// the next line).
//
// Layout: each thread owns a 32-byte chunk; a line belongs to the thread whose
// chunk holds the '\n' before it (line 0 belongs to thread 0).  Pass 1 counts
// lines per 8 KB block with 16-byte loads; after a scan, pass 2 stages the
// block's bytes (plus a 1 KB overhang) in shared memory, block-scans the
// per-thread line counts and parses each owned line into slot
// block_offset + thread_offset + i.  A slot gets min(x,y) << 32 | max(x,y),
// or ~0 for a blank line or a self-loop (sorted to the end, then dropped).
#include "kt_device.cuh"
#include "kt_internal.h"
#include "stages.h"

namespace kt {
namespace {

constexpr unsigned kParseThreads = 256;
constexpr unsigned kChunk = 32;
constexpr unsigned kBlockBytes = kParseThreads * kChunk;  // 8192
constexpr unsigned kOverhang = 1024;

__device__ __forceinline__ uint32_t count_nl16(uint4 v) {
  const uint32_t nl = 0x0a0a0a0au;
  return (__popc(__vcmpeq4(v.x, nl)) + __popc(__vcmpeq4(v.y, nl)) + __popc(__vcmpeq4(v.z, nl)) +
          __popc(__vcmpeq4(v.w, nl))) >> 3;
}

// Lines owned by one chunk: its '\n' bytes except one at len-1, plus line 0.
__device__ __forceinline__ uint32_t owned_lines(const uint8_t* buf, uint64_t len, uint64_t s) {
  if (s >= len) return 0;
  uint32_t c = 0;
  if (s + kChunk <= len) {
    const uint4* p = reinterpret_cast<const uint4*>(buf + s);
    c = count_nl16(p[0]) + count_nl16(p[1]);
    if (s + kChunk == len && buf[len - 1] == '\n') c -= 1;
  } else {
    for (uint64_t q = s; q < len; ++q) c += (buf[q] == '\n' && q + 1 < len);
  }
  return c + (s == 0 ? 1u : 0u);
}

__global__ void __launch_bounds__(kParseThreads) k_count_lines(const uint8_t* __restrict__ buf, uint64_t len,
                                                               uint32_t* __restrict__ block_lines) {
  __shared__ uint32_t tmp[33];
  const uint64_t s = (uint64_t)blockIdx.x * kBlockBytes + (uint64_t)threadIdx.x * kChunk;
  const uint32_t c = owned_lines(buf, len, s);
  const uint32_t t = block_sum<uint32_t>(c, tmp);
  if (threadIdx.x == 0) block_lines[blockIdx.x] = t;
}

struct ByteSrc {
  const uint8_t* sm;   // staged bytes [lo, hi)
  const uint8_t* g;    // global buffer
  uint64_t lo, hi, len;
  __device__ __forceinline__ int at(uint64_t q) const {  // -1 past the end
    if (q >= len) return -1;
    return (q >= lo && q < hi) ? sm[q - lo] : g[q];
  }
};

__device__ __forceinline__ bool is_digit(int b) { return b >= '0' && b < 128; }

__global__ void __launch_bounds__(kParseThreads) k_parse_lines(const uint8_t* __restrict__ buf, uint64_t len,
                                                               const uint64_t* __restrict__ block_off,
                                                               uint64_t* __restrict__ keys, DevWords* words) {
  __shared__ __align__(16) uint8_t stage[kBlockBytes + kOverhang];
  __shared__ uint32_t tmp[33];
  const uint64_t blo = (uint64_t)blockIdx.x * kBlockBytes;
  const uint64_t bhi = min(len, blo + kBlockBytes + kOverhang);
  // The device buffer is padded to a multiple of 16 bytes plus 16, so whole
  // 16-byte loads below bhi rounded up stay inside the allocation.
  const uint64_t nvec = (bhi - blo + 15) / 16;
  for (uint64_t i = threadIdx.x; i < nvec; i += kParseThreads)
    reinterpret_cast<uint4*>(stage)[i] = reinterpret_cast<const uint4*>(buf + blo)[i];
  __syncthreads();
  const ByteSrc src{stage, buf, blo, bhi, len};

  const uint64_t s = blo + (uint64_t)threadIdx.x * kChunk;
  // Owned-line count from the staged copy.
  uint32_t c = 0;
  if (s < len) {
    const uint64_t e = min(len, s + kChunk);
    for (uint64_t q = s; q < e; ++q) c += (stage[q - blo] == '\n' && q + 1 < len);
    c += (s == 0);
  }
  uint32_t total;
  uint64_t slot = block_off[blockIdx.x] + block_excl_scan<uint32_t>(c, tmp, &total);
  if (c == 0) return;
  uint32_t vmax = 0;
  bool any = false;
  const uint64_t e = min(len, s + kChunk);
  uint64_t q = s;
  bool first = (s == 0);
  while (true) {
    uint64_t start;
    if (first) {
      start = 0;
      first = false;
    } else {
      while (q < e && src.at(q) != '\n') ++q;
      if (q >= e) break;
      start = q + 1;
      ++q;
      if (start >= len) break;
    }
    // Parse the line at `start`.
    uint64_t p = start;
    int b = src.at(p);
    while (b >= 0 && b != '\n' && !is_digit(b)) b = src.at(++p);
    uint64_t key = ~0ULL;
    if (is_digit(b)) {
      uint32_t x = 0, y = 0;
      while (is_digit(b)) {
        x = x * 10u + (uint32_t)(b - '0');
        b = src.at(++p);
      }
      while (b >= 0 && b != '\n' && !is_digit(b)) b = src.at(++p);
      if (!is_digit(b)) {
        atomicOr(&words->err, kDevErrParse);
        atomicMin(&words->bad_line, (unsigned long long)slot);
      } else {
        while (is_digit(b)) {
          y = y * 10u + (uint32_t)(b - '0');
          b = src.at(++p);
        }
        vmax = max(vmax, max(x, y));
        any = true;
        if (x != y) key = x < y ? (((uint64_t)x << 32) | y) : (((uint64_t)y << 32) | x);
      }
    }
    keys[slot++] = key;
  }
  if (any) atomicMax(reinterpret_cast<unsigned int*>(&words->counters[0]), vmax + 0u);
  if (any) atomicOr(reinterpret_cast<unsigned int*>(&words->counters[1]), 1u);
}

}  // namespace

uint64_t parse_count_lines(Ctx* c, const uint8_t* dbuf, uint64_t len, DBuf& block_off) {
  const uint64_t blocks = (len + kBlockBytes - 1) / kBlockBytes;
  if (blocks == 0) return 0;
  if (blocks > 0x7fffffffULL) throw Error(KT_ERR_LIMIT, "TSV larger than the parser's grid");
  DBuf cnt(c, (blocks + 1) * sizeof(uint32_t));
  k_count_lines<<<(unsigned)blocks, kParseThreads, 0, c->stream>>>(dbuf, len, cnt.as<uint32_t>());
  KT_LAUNCHED(c);
  zero(c, cnt.as<uint32_t>() + blocks, sizeof(uint32_t));
  block_off.ensure(c, (blocks + 1) * sizeof(uint64_t));
  scan_u32_to_u64(c, cnt.as<uint32_t>(), block_off.as<uint64_t>(), blocks + 1);
  return read_word<uint64_t>(c, block_off.as<uint64_t>() + blocks);
}

void parse_lines(Ctx* c, const uint8_t* dbuf, uint64_t len, const DBuf& block_off, uint64_t* keys, DevWords* words) {
  const uint64_t blocks = (len + kBlockBytes - 1) / kBlockBytes;
  if (blocks == 0) return;
  k_parse_lines<<<(unsigned)blocks, kParseThreads, 0, c->stream>>>(dbuf, len, block_off.as<uint64_t>(), keys, words);
  KT_LAUNCHED(c);
}

uint64_t parse_padded_bytes(uint64_t len) { return ((len + 15) / 16) * 16 + kOverhang + 16; }

}  // namespace kt
