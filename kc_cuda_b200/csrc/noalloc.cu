// k-core membership without any device allocation.
//
// Some callers cannot allocate device memory at the moment they need the
// answer: code that runs inside another runtime's fully reserved memory pool,
// host callbacks and other contexts where an allocating CUDA call may block
// or deadlock, and latency-bound paths that cannot afford the device-wide
// synchronisation cudaMalloc/cudaFree may imply.  kt_kcore_noalloc serves
// them: the caller passes the graph and the output already on the device,
// and every piece of working memory (degrees, removal marks, two frontiers,
// counters and the grid-barrier words) lives in one file-scope device array
// of fixed size, so the call allocates nothing.
//
// The array is kNoAllocBytes (about 16 MB) and every GPU that loads this
// library holds it until the process exits.  It caps the graph at
// kNoAllocMaxVertices vertices.  All calls share it and it keeps the last
// call's contents, so the header words that must start at zero are cleared
// at the start of every call, and calls that overlap on the GPU (two streams,
// two threads) race on it.
//
// The kernel is the probe of kcore.cu restated for a single level k and a
// caller-owned CSR: one cooperative launch, rounds separated by the bounded
// grid barrier.
#include <mutex>

#include "kt.h"
#include "kt_device.cuh"

namespace kt {
namespace {

constexpr uint32_t kNoAllocMaxVertices = 1u << 20;
constexpr size_t kHeaderBytes = 4096;  // DevWords + counters, cleared every call
constexpr size_t kNoAllocBytes = kHeaderBytes + 4ull * kNoAllocMaxVertices * sizeof(uint32_t);
constexpr int kMaxDevices = 64;
constexpr unsigned kThreads = 256;

// The working memory of every kt_kcore_noalloc call on a device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

struct View {
  DevWords* words;
  unsigned long long* cnt;  // [0..2] rotating frontier sizes
  uint32_t* deg;
  uint32_t* rem;
  uint32_t* front[2];
};

View carve(unsigned char* base) {
  View v;
  v.words = reinterpret_cast<DevWords*>(base);
  v.cnt = reinterpret_cast<unsigned long long*>(base + 1024);
  uint32_t* arr = reinterpret_cast<uint32_t*>(base + kHeaderBytes);
  v.deg = arr;
  v.rem = arr + kNoAllocMaxVertices;
  v.front[0] = arr + 2 * kNoAllocMaxVertices;
  v.front[1] = arr + 3 * kNoAllocMaxVertices;
  return v;
}

__device__ __forceinline__ void push(bool want, uint32_t item, uint32_t* list, unsigned long long* cnt,
                                     uint32_t* err) {
  const unsigned b = __ballot_sync(kFull, want);
  if (!b) return;
  const unsigned leader = __ffs(b) - 1;
  unsigned long long base = 0;
  if (lane_id() == leader) base = atomicAdd(cnt, (unsigned long long)__popc(b));
  base = __shfl_sync(kFull, base, leader);
  if (want) {
    const unsigned long long p = base + __popc(b & lanemask_lt());
    if (p < kNoAllocMaxVertices)
      list[p] = item;
    else
      atomicOr(err, kDevErrCapacity);
  }
}

__global__ void __launch_bounds__(kThreads) k_kcore_noalloc(View S, const uint64_t* __restrict__ off,
                                                            const uint32_t* __restrict__ adj, uint32_t n,
                                                            uint32_t k, uint8_t* __restrict__ member,
                                                            unsigned long long timeout_ns) {
  const uint64_t gthreads = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t gwarps = gthreads >> 5, gwarp = gtid >> 5;
  uint32_t* err = &S.words->err;
  for (uint64_t v = gtid; v < n; v += gthreads) {
    S.deg[v] = (uint32_t)(off[v + 1] - off[v]);
    S.rem[v] = kAlive;
  }
  if (!grid_barrier(S.words, timeout_ns)) return;
  for (uint64_t v = gtid; v < ((n + 31ull) & ~31ull); v += gthreads) {
    const bool want = v < n && S.deg[v] < k;
    if (want) S.rem[v] = 1;
    push(want, (uint32_t)v, S.front[0], &S.cnt[0], err);
  }
  if (!grid_barrier(S.words, timeout_ns)) return;
  for (uint32_t i = 0;; ++i) {
    const uint64_t nf = ld_acquire_u64(&S.cnt[i % 3]);
    if (nf == 0) break;
    const uint32_t* fr = S.front[i & 1];
    uint32_t* nx = S.front[(i + 1) & 1];
    unsigned long long* nc = &S.cnt[(i + 1) % 3];
    for (uint64_t f = gwarp; f < nf; f += gwarps) {
      const uint32_t v = fr[f];
      const uint64_t b = off[v], e = off[v + 1];
      for (uint64_t j = b + lane_id(); j < b + ((e - b + 31) & ~31ull); j += 32) {
        bool want = false;
        uint32_t w = 0;
        if (j < e) {
          w = adj[j];
          if (w < n && S.rem[w] == kAlive && atomicSub(&S.deg[w], 1u) == k) {
            S.rem[w] = 1;
            want = true;
          }
        }
        push(want, w, nx, nc, err);
      }
    }
    if (gtid == 0) S.cnt[(i + 2) % 3] = 0;  // read at the start of round i-1
    if (!grid_barrier(S.words, timeout_ns)) return;
  }
  for (uint64_t v = gtid; v < n; v += gthreads) member[v] = S.rem[v] == kAlive;
}

struct DeviceSetup {
  unsigned char* base = nullptr;
  unsigned grid = 0;
};

std::mutex g_setup_mu;
DeviceSetup g_setup[kMaxDevices];

}  // namespace
}  // namespace kt

extern "C" kt_status kt_kcore_noalloc(const uint64_t* d_off, const uint32_t* d_adj, uint32_t n, uint32_t k,
                                      uint8_t* d_member, void* stream) {
  using namespace kt;
  if (n > kNoAllocMaxVertices) return KT_ERR_LIMIT;
  if (n == 0) return KT_OK;
  if (!d_off || !d_adj || !d_member) return KT_ERR_INVALID;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return KT_ERR_NODEV;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (s) {
    // The array's address is per device: a stream of another device would
    // get this device's address.  Such a call is refused.
    int sdev = -1;
    if (cudaStreamGetDevice(s, &sdev) != cudaSuccess) {
      cudaGetLastError();
      return KT_ERR_INVALID;
    }
    if (sdev != dev) return KT_ERR_INVALID;
  }
  DeviceSetup setup;
  {
    // First call on this device: find the scratch array's device address
    // (the host-side name is only a stand-in) and the cooperative grid size.
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_setup[dev].base) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
        cudaGetLastError();
        return KT_ERR_CUDA;
      }
      int per_sm = 0, sms = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_kcore_noalloc, kThreads, 0) != cudaSuccess ||
          cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        return KT_ERR_CUDA;
      }
      g_setup[dev].grid = (unsigned)(per_sm * sms);
      g_setup[dev].base = static_cast<unsigned char*>(p);
    }
    setup = g_setup[dev];
  }
  // The header (error flag, barrier words, frontier counters) must start at
  // zero; the arrays are written before they are read.
  if (cudaMemsetAsync(setup.base, 0, kHeaderBytes, s) != cudaSuccess) {
    cudaGetLastError();
    return KT_ERR_CUDA;
  }
  View view = carve(setup.base);
  unsigned long long timeout_ns = 20ull * 1000000000ull;
  void* args[] = {&view, &d_off, &d_adj, &n, &k, &d_member, &timeout_ns};
  if (cudaLaunchCooperativeKernel((const void*)k_kcore_noalloc, dim3(setup.grid), dim3(kThreads), args, 0, s) !=
      cudaSuccess) {
    cudaGetLastError();
    return KT_ERR_CUDA;
  }
  uint32_t err = 0;
  if (cudaMemcpyAsync(&err, &view.words->err, sizeof(err), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return KT_ERR_CUDA;
  }
  if (err & kDevErrBarrier) return KT_ERR_TIMEOUT;
  if (err) return KT_ERR_CUDA;
  return KT_OK;
}
