// Context plumbing: device buffers charged to the HBM budget, small copies,
// and the CUDA error -> kt::Error conversion.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <set>
#include <utility>

#include "kt_internal.h"

namespace kt {

void throw_cuda(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  std::snprintf(buf, sizeof(buf), "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  cudaGetLastError();  // clear a sticky launch error where possible
  kt_status s = (e == cudaErrorMemoryAllocation) ? KT_ERR_NOMEM : KT_ERR_CUDA;
  throw Error(s, buf);
}

void DBuf::alloc(Ctx* c, size_t bytes) {
  ctx_ = c;
  bytes_ = 0;
  ptr_ = nullptr;
  if (bytes == 0) bytes = 16;
  bytes = (bytes + 255) & ~size_t(255);
  if (c->budget && c->in_use + bytes > c->budget) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "HBM budget exceeded: %zu bytes requested, %llu of %llu in use", bytes,
                  (unsigned long long)c->in_use, (unsigned long long)c->budget);
    throw Error(KT_ERR_NOMEM, buf);
  }
  cudaError_t e = cudaMallocAsync(&ptr_, bytes, c->stream);
  if (e != cudaSuccess) {
    ptr_ = nullptr;
    throw_cuda(e, "cudaMallocAsync", __FILE__, __LINE__);
  }
  bytes_ = bytes;
  c->in_use += bytes;
  if (c->in_use > c->peak) c->peak = c->in_use;
}

void DBuf::release() {
  if (ptr_ && ctx_) {
    cudaFreeAsync(ptr_, ctx_->stream);
    ctx_->in_use -= bytes_;
  }
  ptr_ = nullptr;
  bytes_ = 0;
  ctx_ = nullptr;
}

void allow_max_dynamic_smem(const void* func) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  KT_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({dev, func})) return;
  int optin = 0;
  KT_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  KT_CUDA(cudaFuncGetAttributes(&fa, func));
  KT_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               optin - (int)fa.sharedSizeBytes));
  done.insert({dev, func});
}

void sync(Ctx* c) { KT_CUDA(cudaStreamSynchronize(c->stream)); }

void copy_d2h(Ctx* c, void* dst, const void* src, size_t bytes) {
  if (!bytes) return;
  c->d2h_bytes += bytes;
  KT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
  sync(c);
}

void copy_h2d(Ctx* c, void* dst, const void* src, size_t bytes) {
  if (!bytes) return;
  c->h2d_bytes += bytes;
  KT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
}

void zero(Ctx* c, void* dptr, size_t bytes) {
  if (!bytes) return;
  KT_CUDA(cudaMemsetAsync(dptr, 0, bytes, c->stream));
}

cudaEvent_t EventTimer::get() {
  if (used == pool.size()) {
    cudaEvent_t e;
    KT_CUDA(cudaEventCreate(&e));
    pool.push_back(e);
  }
  return pool[used++];
}

void EventTimer::begin(cudaStream_t s, double* acc, cudaEvent_t* out_a) {
  (void)acc;
  *out_a = get();
  KT_CUDA(cudaEventRecord(*out_a, s));
}

void EventTimer::end(cudaStream_t s, cudaEvent_t a, double* acc) {
  cudaEvent_t b = get();
  KT_CUDA(cudaEventRecord(b, s));
  open.push_back({a, b, acc});
}

void EventTimer::resolve() {
  for (const Span& sp : open) {
    KT_CUDA(cudaEventSynchronize(sp.b));
    float ms = 0;
    KT_CUDA(cudaEventElapsedTime(&ms, sp.a, sp.b));
    *sp.acc += ms;
  }
  open.clear();
  used = 0;
}

EventTimer::~EventTimer() {
  for (cudaEvent_t e : pool) cudaEventDestroy(e);
}

}  // namespace kt
