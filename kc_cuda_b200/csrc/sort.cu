// Stable LSD radix sort of 64-bit keys (optionally carrying a 32-bit value),
// 8-bit digits.
//
// One pass = tile histograms -> digit-major exclusive scan -> stable scatter.
// A tile is 4096 keys: each of the 8 warps owns 512 consecutive keys, ranks
// them with __match_any_sync against warp-private running digit counters,
// then the block turns the per-warp counts into per-warp digit offsets,
// places the tile in shared memory sorted by digit, and writes every digit's
// run with consecutive threads on consecutive addresses.  A
// first pass histograms all eight digit positions at once so passes whose
// digit is the same for every key are skipped.
#include <algorithm>

#include "kt_device.cuh"
#include "kt_internal.h"

namespace kt {
namespace {

constexpr unsigned kSortThreads = 256;
constexpr unsigned kSortWarps = kSortThreads / 32;
constexpr unsigned kSortIpt = 16;                       // keys per lane
constexpr unsigned kWarpKeys = 32 * kSortIpt;           // 512
constexpr unsigned kSortTile = kSortWarps * kWarpKeys;  // 4096

__global__ void __launch_bounds__(kSortThreads) k_hist_all(const uint64_t* __restrict__ keys, uint64_t n,
                                                           int lo, int passes,
                                                           unsigned long long* __restrict__ hist) {
  __shared__ uint32_t h[8][256];
  for (unsigned i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&h[0][0])[i] = 0;
  __syncthreads();
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    for (int p = 0; p < passes; ++p) atomicAdd(&h[p][(k >> (lo + 8 * p)) & 255], 1u);
  }
  __syncthreads();
  for (unsigned i = threadIdx.x; i < (unsigned)passes * 256; i += blockDim.x) {
    const uint32_t v = (&h[0][0])[i];
    if (v) atomicAdd(&hist[i], (unsigned long long)v);
  }
}

__global__ void __launch_bounds__(kSortThreads) k_tile_hist(const uint64_t* __restrict__ keys, uint64_t n, int shift,
                                                            uint32_t ntiles, uint32_t* __restrict__ tile_hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
#pragma unroll 4
  for (unsigned i = 0; i < kSortTile / kSortThreads; ++i) {
    const uint64_t j = base + i * kSortThreads + threadIdx.x;
    if (j < n) atomicAdd(&h[(keys[j] >> shift) & 255], 1u);
  }
  __syncthreads();
  tile_hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Scatter of one tile: rank every key (stable), place the tile sorted by
// digit in shared memory, then write each digit's run with consecutive
// threads on consecutive addresses.
template <bool kVals>
__global__ void __launch_bounds__(kSortThreads) k_scatter(const uint64_t* __restrict__ keys,
                                                          const uint32_t* __restrict__ vals, uint64_t n, int shift,
                                                          uint32_t ntiles, const uint32_t* __restrict__ tile_off,
                                                          uint64_t* __restrict__ keys_out,
                                                          uint32_t* __restrict__ vals_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* skeys = reinterpret_cast<uint64_t*>(smem_raw);                          // kSortTile
  uint32_t* svals = reinterpret_cast<uint32_t*>(smem_raw + kSortTile * 8);          // kSortTile (kVals)
  __shared__ uint32_t wrun[kSortWarps][256];
  __shared__ uint32_t toff[256];
  __shared__ uint32_t dstart[256];
  __shared__ uint32_t tmp[33];
  const unsigned w = warp_id(), l = lane_id();
  toff[threadIdx.x] = tile_off[(uint64_t)threadIdx.x * ntiles + blockIdx.x];
#pragma unroll
  for (unsigned q = 0; q < kSortWarps; ++q) wrun[q][threadIdx.x] = 0;
  __syncthreads();

  const uint64_t tbase = (uint64_t)blockIdx.x * kSortTile;
  const uint32_t tn = (uint32_t)(n - tbase < kSortTile ? n - tbase : kSortTile);
  const uint64_t wbase = tbase + (uint64_t)w * kWarpKeys;
  uint64_t k[kSortIpt];
  uint32_t v[kSortIpt];
  uint32_t rank[kSortIpt];
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (unsigned j = 0; j < kSortIpt; ++j) {
    const uint64_t idx = wbase + j * 32 + l;
    const bool valid = idx < n;
    k[j] = valid ? keys[idx] : 0;
    if (kVals) v[j] = valid ? vals[idx] : 0;
    const uint32_t d = valid ? (uint32_t)((k[j] >> shift) & 255) : 256u;
    const unsigned peers = __match_any_sync(kFull, d);
    const uint32_t base = valid ? wrun[w][d] : 0u;
    __syncwarp();
    if (valid && l == (unsigned)(__ffs(peers) - 1)) wrun[w][d] = base + __popc(peers);
    __syncwarp();
    rank[j] = base + __popc(peers & lt);
  }
  __syncthreads();
  {
    // Per digit: warp prefixes, then the tile-local start of the digit.
    const unsigned d = threadIdx.x;
    uint32_t s = 0;
#pragma unroll
    for (unsigned q = 0; q < kSortWarps; ++q) {
      const uint32_t t = wrun[q][d];
      wrun[q][d] = s;
      s += t;
    }
    uint32_t total;
    dstart[d] = block_excl_scan<uint32_t>(s, tmp, &total);
  }
  __syncthreads();
#pragma unroll
  for (unsigned j = 0; j < kSortIpt; ++j) {
    const uint64_t idx = wbase + j * 32 + l;
    if (idx < n) {
      const uint32_t d = (uint32_t)((k[j] >> shift) & 255);
      const uint32_t p = dstart[d] + wrun[w][d] + rank[j];
      skeys[p] = k[j];
      if (kVals) svals[p] = v[j];
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < tn; i += kSortThreads) {
    const uint64_t key = skeys[i];
    const uint32_t d = (uint32_t)((key >> shift) & 255);
    const uint32_t pos = toff[d] + (i - dstart[d]);
    keys_out[pos] = key;
    if (kVals) vals_out[pos] = svals[i];
  }
}

}  // namespace

void radix_sort_u64(Ctx* c, uint64_t* keys, uint32_t* vals, uint64_t n, int bits, int lo_bit) {
  if (bits > 64) bits = 64;
  if (lo_bit < 0) lo_bit = 0;
  if (n < 2 || bits <= lo_bit) return;
  if (n >= 0xffffffffULL) throw Error(KT_ERR_LIMIT, "radix sort: more than 2^32-1 keys");
  const int passes = std::min((bits - lo_bit + 7) / 8, (64 - lo_bit + 7) / 8);
  DBuf hist(c, 8 * 256 * sizeof(unsigned long long));
  zero(c, hist.get(), hist.bytes());
  k_hist_all<<<grid_for(n, kSortThreads, c->num_sms * 8), kSortThreads, 0, c->stream>>>(
      keys, n, lo_bit, passes, hist.as<unsigned long long>());
  KT_LAUNCHED(c);
  std::vector<unsigned long long> h(8 * 256);
  copy_d2h(c, h.data(), hist.get(), h.size() * sizeof(unsigned long long));

  const uint32_t ntiles = (uint32_t)((n + kSortTile - 1) / kSortTile);
  allow_max_dynamic_smem((const void*)k_scatter<true>);
  allow_max_dynamic_smem((const void*)k_scatter<false>);
  DBuf keys_alt(c, n * sizeof(uint64_t));
  DBuf vals_alt;
  if (vals) vals_alt.alloc(c, n * sizeof(uint32_t));
  DBuf th(c, (uint64_t)ntiles * 256 * sizeof(uint32_t));
  uint64_t* ksrc = keys;
  uint64_t* kdst = keys_alt.as<uint64_t>();
  uint32_t* vsrc = vals;
  uint32_t* vdst = vals ? vals_alt.as<uint32_t>() : nullptr;
  for (int p = 0; p < passes; ++p) {
    int distinct = 0;
    for (int d = 0; d < 256; ++d) distinct += h[p * 256 + d] != 0;
    if (distinct <= 1) continue;
    const int shift = lo_bit + 8 * p;
    k_tile_hist<<<ntiles, kSortThreads, 0, c->stream>>>(ksrc, n, shift, ntiles, th.as<uint32_t>());
    KT_LAUNCHED(c);
    scan_u32(c, th.as<uint32_t>(), th.as<uint32_t>(), (uint64_t)ntiles * 256);
    if (vals)
      k_scatter<true><<<ntiles, kSortThreads, kSortTile * 12, c->stream>>>(ksrc, vsrc, n, shift, ntiles,
                                                                           th.as<uint32_t>(), kdst, vdst);
    else
      k_scatter<false><<<ntiles, kSortThreads, kSortTile * 8, c->stream>>>(ksrc, nullptr, n, shift, ntiles,
                                                                           th.as<uint32_t>(), kdst, nullptr);
    KT_LAUNCHED(c);
    std::swap(ksrc, kdst);
    std::swap(vsrc, vdst);
  }
  if (ksrc != keys) {
    KT_CUDA(cudaMemcpyAsync(keys, ksrc, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, c->stream));
    if (vals) KT_CUDA(cudaMemcpyAsync(vals, vsrc, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, c->stream));
  }
}

}  // namespace kt
