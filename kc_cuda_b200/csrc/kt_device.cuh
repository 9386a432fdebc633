// Device-side building blocks: warp/block scans and reductions, acquire /
// release word access, and the bounded grid barrier used by the persistent
// (cooperatively launched) kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace kt {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kAlive = 0xffffffffu;

// Device error bits (written to DevWords::err, read by the host).
enum : uint32_t {
  kDevErrBarrier = 1u,     // a grid barrier wait ran past its bound
  kDevErrCapacity = 2u,    // a work list overflowed (kernel returned early)
  kDevErrParse = 4u,       // malformed record (first offending line in DevWords::bad_line)
  kDevErrWait = 8u,        // another bounded wait gave up
};

// One block of device words per context (kept zeroed between launches).
struct DevWords {
  uint32_t err;
  uint32_t bar_count;
  uint32_t bar_gen;
  uint32_t pad0;
  unsigned long long bad_line;
  unsigned long long counters[16];
};

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned warp_id() { return threadIdx.x >> 5; }
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T w = __shfl_xor_sync(kFull, v, o);
    v = w < v ? w : v;
  }
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T w = __shfl_xor_sync(kFull, v, o);
    v = w > v ? w : v;
  }
  return v;
}
// Inclusive warp scan.
template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
  const unsigned l = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T w = __shfl_up_sync(kFull, v, o);
    if (l >= (unsigned)o) v += w;
  }
  return v;
}

// Block-wide exclusive scan; every thread of the block must call it.
// `tmp` holds at least 33 T in shared memory.  Returns the exclusive prefix
// and the block total in *total.
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* tmp, T* total) {
  const unsigned w = warp_id(), l = lane_id(), nw = blockDim.x >> 5;
  T inc = warp_incl_scan(v);
  if (l == 31) tmp[w] = inc;
  __syncthreads();
  if (w == 0) {
    T s = l < nw ? tmp[l] : T(0);
    T si = warp_incl_scan(s);
    if (l < nw) tmp[l] = si - s;
    if (l == 31) tmp[32] = si;
  }
  __syncthreads();
  T r = tmp[w] + inc - v;
  *total = tmp[32];
  __syncthreads();
  return r;
}

template <typename T>
__device__ __forceinline__ T block_sum(T v, T* tmp) {
  const unsigned w = warp_id(), l = lane_id(), nw = blockDim.x >> 5;
  v = warp_sum(v);
  if (l == 0) tmp[w] = v;
  __syncthreads();
  if (w == 0) {
    T s = l < nw ? tmp[l] : T(0);
    s = warp_sum(s);
    if (l == 0) tmp[32] = s;
  }
  __syncthreads();
  T r = tmp[32];
  __syncthreads();
  return r;
}

// Bounded grid barrier for kernels launched with cudaLaunchCooperativeKernel
// (which guarantees that every block is resident).  Every block must call it
// the same number of times.  A wait longer than `timeout_ns` sets
// kDevErrBarrier and returns; callers test the returned flag and leave the
// kernel, so a mismatch can never hang the device.  Returns true when no
// error is flagged.
__device__ __forceinline__ bool grid_barrier(DevWords* w, unsigned long long timeout_ns) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t gen = ld_acquire_u32(&w->bar_gen);
    __threadfence();
    const uint32_t arrived = atomicAdd(&w->bar_count, 1u);
    if (arrived == gridDim.x * gridDim.y * gridDim.z - 1) {
      atomicExch(&w->bar_count, 0u);
      __threadfence();
      atomicAdd(&w->bar_gen, 1u);
    } else {
      const unsigned long long t0 = globaltimer_ns();
      unsigned spins = 0;
      while (ld_acquire_u32(&w->bar_gen) == gen) {
        if (++spins > 32) __nanosleep(spins > 1024 ? 256 : 32);
        // The bound is checked on the first spin and every 64th after it, so
        // a bound of 0 gives up at once.
        if ((spins & 63) == 1 && globaltimer_ns() - t0 >= timeout_ns) {
          atomicOr(&w->err, kDevErrBarrier);
          break;
        }
        if ((spins & 255) == 0 && ld_volatile_u32(&w->err) != 0) break;
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ld_volatile_u32(&w->err) == 0;
}

// One bulk copy by the TMA engine (cp.async.bulk, no multicast) of `bytes`
// from global memory into this block's shared memory; both addresses 16-byte
// aligned and `bytes` a multiple of 16.  Completion is tracked by the
// mbarrier `mbar` (shared memory, 8-byte aligned, used once).  Every thread
// of the block calls it: thread 0 initialises the barrier, announces the
// bytes and issues the copy; then every thread polls the barrier's first
// phase at most `polls` times.  Returns false (with kDevErrWait in *err) in
// any thread that gave up; the staged bytes must then not be used.
__device__ __forceinline__ bool bulk_load_to_shared(void* dst, const void* src, uint32_t bytes, uint64_t* mbar,
                                                    uint32_t* err, uint32_t polls = 1u << 20) {
  const uint32_t bar = (uint32_t)__cvta_generic_to_shared(mbar);
  const uint32_t sdst = (uint32_t)__cvta_generic_to_shared(dst);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(sdst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
  }
  uint32_t done = 0;
  for (uint32_t i = 0; i < polls && !done; ++i)
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(bar)
        : "memory");
  if (!done) atomicOr(err, kDevErrWait);
  return done != 0;
}

}  // namespace kt
