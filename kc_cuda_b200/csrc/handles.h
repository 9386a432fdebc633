// Handle types behind the C ABI and the entry-point wrapper shared by the
// files that implement it (api.cu, serve.cu).
#pragma once
#include <mutex>
#include <new>
#include <vector>

#include "kt.h"
#include "batch.h"

struct kt_ctx {
  kt::Ctx c;
  bool counted = false;  // counted among the device's live contexts
};
struct kt_graph {
  kt::Graph g;
};
struct kt_tsv {
  kt::DBuf bytes;
  uint64_t len = 0;
};
struct kt_batch {
  kt_ctx* ctx = nullptr;
  std::vector<kt::BatchItem> items;
};

#define KT_API_BEGIN(ctx)                            \
  if (!(ctx)) return KT_ERR_INVALID;                 \
  std::lock_guard<std::recursive_mutex> lk_((ctx)->c.mu); \
  try {                                              \
    KT_CUDA(cudaSetDevice((ctx)->c.device));
#define KT_API_END(ctx)                              \
  return KT_OK;                                      \
  }                                                  \
  catch (const kt::Error& e) {                       \
    (ctx)->c.set_error(e.what());                    \
    return e.status;                                 \
  }                                                  \
  catch (const std::bad_alloc&) {                    \
    (ctx)->c.set_error("host allocation failed");    \
    return KT_ERR_NOMEM;                             \
  }                                                  \
  catch (const std::exception& e) {                  \
    (ctx)->c.set_error(e.what());                    \
    return KT_ERR_CUDA;                              \
  }

