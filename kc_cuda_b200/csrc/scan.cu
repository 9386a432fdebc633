// Device-wide scans, reductions and the sorted-unique compaction.
//
// Scans are reduce-then-scan over tiles of 2048 items (256 threads x 8): a
// tile-sum kernel, a recursive scan of the tile sums, and a tile-scan kernel
// that adds the tile's prefix.  Tiles are staged through shared memory so
// every global access is coalesced.
#include "kt_device.cuh"
#include "kt_internal.h"

namespace kt {
namespace {

constexpr unsigned kScanThreads = 256;
constexpr unsigned kScanItems = 8;
constexpr unsigned kScanTile = kScanThreads * kScanItems;

template <typename Tin, typename Tout>
__global__ void __launch_bounds__(kScanThreads) k_tile_sum(const Tin* __restrict__ in, uint64_t n,
                                                           Tout* __restrict__ sums) {
  __shared__ Tout tmp[33];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  Tout s = 0;
#pragma unroll
  for (unsigned i = 0; i < kScanItems; ++i) {
    const uint64_t j = base + i * kScanThreads + threadIdx.x;
    if (j < n) s += (Tout)in[j];
  }
  s = block_sum<Tout>(s, tmp);
  if (threadIdx.x == 0) sums[blockIdx.x] = s;
}

// Exclusive scan of one tile plus an optional per-tile prefix.  In-place safe:
// the whole tile is read before any of it is written.
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(kScanThreads) k_tile_scan(const Tin* in, Tout* out, uint64_t n,
                                                            const Tout* __restrict__ prefix) {
  __shared__ Tout stage[kScanTile];
  __shared__ Tout tmp[33];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
#pragma unroll
  for (unsigned i = 0; i < kScanItems; ++i) {
    const uint64_t j = base + i * kScanThreads + threadIdx.x;
    stage[i * kScanThreads + threadIdx.x] = j < n ? (Tout)in[j] : Tout(0);
  }
  __syncthreads();
  Tout v[kScanItems];
  Tout run = 0;
#pragma unroll
  for (unsigned i = 0; i < kScanItems; ++i) {
    v[i] = run;
    run += stage[threadIdx.x * kScanItems + i];
  }
  Tout total;
  const Tout excl = block_excl_scan<Tout>(run, tmp, &total);
  const Tout off = (prefix ? prefix[blockIdx.x] : Tout(0)) + excl;
#pragma unroll
  for (unsigned i = 0; i < kScanItems; ++i) stage[threadIdx.x * kScanItems + i] = v[i] + off;
  __syncthreads();
#pragma unroll
  for (unsigned i = 0; i < kScanItems; ++i) {
    const uint64_t j = base + i * kScanThreads + threadIdx.x;
    if (j < n) out[j] = stage[i * kScanThreads + threadIdx.x];
  }
}

template <typename Tin, typename Tout>
void scan_impl(Ctx* c, const Tin* in, Tout* out, uint64_t n) {
  if (n == 0) return;
  const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles > 0x7fffffffULL) throw Error(KT_ERR_LIMIT, "scan: too many tiles");
  if (tiles == 1) {
    k_tile_scan<Tin, Tout><<<1, kScanThreads, 0, c->stream>>>(in, out, n, nullptr);
    KT_LAUNCHED(c);
    return;
  }
  DBuf sums(c, tiles * sizeof(Tout));
  k_tile_sum<Tin, Tout><<<(unsigned)tiles, kScanThreads, 0, c->stream>>>(in, n, sums.as<Tout>());
  KT_LAUNCHED(c);
  scan_impl<Tout, Tout>(c, sums.as<Tout>(), sums.as<Tout>(), tiles);
  k_tile_scan<Tin, Tout><<<(unsigned)tiles, kScanThreads, 0, c->stream>>>(in, out, n, sums.as<Tout>());
  KT_LAUNCHED(c);
}

__global__ void k_reduce_u32(const uint32_t* __restrict__ in, uint64_t n, unsigned long long* out) {
  __shared__ uint64_t tmp[33];
  uint64_t s = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    s += in[i];
  s = block_sum<uint64_t>(s, tmp);
  if (threadIdx.x == 0 && s) atomicAdd(out, (unsigned long long)s);
}

// ---- sorted unique: count kept keys per tile, scan, then write them.
__device__ __forceinline__ bool keep_key(const uint64_t* in, uint64_t j) {
  const uint64_t k = in[j];
  return k != ~0ULL && (j == 0 || in[j - 1] != k);
}

__global__ void __launch_bounds__(kScanThreads) k_unique_count(const uint64_t* __restrict__ in, uint64_t n,
                                                               uint64_t* __restrict__ counts) {
  __shared__ uint64_t tmp[33];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  uint64_t s = 0;
#pragma unroll
  for (unsigned i = 0; i < kScanItems; ++i) {
    const uint64_t j = base + i * kScanThreads + threadIdx.x;
    if (j < n) s += keep_key(in, j);
  }
  s = block_sum<uint64_t>(s, tmp);
  if (threadIdx.x == 0) counts[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kScanThreads) k_unique_write(const uint64_t* __restrict__ in, uint64_t n,
                                                               const uint64_t* __restrict__ offs,
                                                               uint64_t* __restrict__ out) {
  __shared__ uint64_t tmp[33];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  // Blocked ownership keeps the output in input order.
  uint32_t flags = 0;
  uint64_t keys[kScanItems];
#pragma unroll
  for (unsigned i = 0; i < kScanItems; ++i) {
    const uint64_t j = base + threadIdx.x * kScanItems + i;
    keys[i] = j < n ? in[j] : ~0ULL;
    if (j < n && keep_key(in, j)) flags |= 1u << i;
  }
  uint64_t total;
  uint64_t pos = offs[blockIdx.x] + block_excl_scan<uint64_t>((uint64_t)__popc(flags), tmp, &total);
#pragma unroll
  for (unsigned i = 0; i < kScanItems; ++i)
    if (flags & (1u << i)) out[pos++] = keys[i];
}

}  // namespace

void scan_u32_to_u64(Ctx* c, const uint32_t* in, uint64_t* out, uint64_t n) { scan_impl<uint32_t, uint64_t>(c, in, out, n); }
void scan_u32(Ctx* c, const uint32_t* in, uint32_t* out, uint64_t n) { scan_impl<uint32_t, uint32_t>(c, in, out, n); }
void scan_u64(Ctx* c, const uint64_t* in, uint64_t* out, uint64_t n) { scan_impl<uint64_t, uint64_t>(c, in, out, n); }

uint64_t reduce_u32(Ctx* c, const uint32_t* in, uint64_t n) {
  DBuf acc(c, 8);
  zero(c, acc.get(), 8);
  if (n) {
    k_reduce_u32<<<grid_for(n, 256, 4 * 148 * 8), 256, 0, c->stream>>>(in, n, acc.as<unsigned long long>());
    KT_LAUNCHED(c);
  }
  return read_word<uint64_t>(c, acc.as<uint64_t>());
}

uint64_t unique_sorted_u64(Ctx* c, const uint64_t* in, uint64_t* out, uint64_t n) {
  if (n == 0) return 0;
  const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
  DBuf counts(c, (tiles + 1) * sizeof(uint64_t));
  k_unique_count<<<(unsigned)tiles, kScanThreads, 0, c->stream>>>(in, n, counts.as<uint64_t>());
  KT_LAUNCHED(c);
  // counts[tiles] = 0 so the exclusive scan's last slot is the total.
  zero(c, counts.as<uint64_t>() + tiles, sizeof(uint64_t));
  scan_u64(c, counts.as<uint64_t>(), counts.as<uint64_t>(), tiles + 1);
  k_unique_write<<<(unsigned)tiles, kScanThreads, 0, c->stream>>>(in, n, counts.as<uint64_t>(), out);
  KT_LAUNCHED(c);
  return read_word<uint64_t>(c, counts.as<uint64_t>() + tiles);
}

}  // namespace kt
