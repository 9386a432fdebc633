// Serving: a continuous-batching request loop over the batch path.
//
// Requests (graphs) are submitted from any host thread and queue in arrival
// order.  One worker thread owns the context: whenever the device is free it
// admits queued requests, oldest first, while their estimated device
// footprint fits the context's budget (and up to a graph cap), and solves the
// admitted set as one wave -- one disjoint union through every stage, each
// graph on its own peel levels (batch.cu).  Requests that arrive while a wave
// runs are admitted into the next one, so small requests ride along with
// large ones and the device never waits for a fixed batch to fill.  The
// result of a request does not depend on which wave it joined or on its
// wave-mates: triangles never cross graphs in a union.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

#include "handles.h"
#include "solve.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Request {
  uint64_t id = 0;
  kt::BatchItem item;
  uint64_t footprint = 0;
  Clock::time_point submitted, admitted, finished;
  bool done = false;
  kt_request_result result{};
};

}  // namespace

struct kt_server {
  kt_ctx* ctx = nullptr;
  uint32_t max_wave = 0;
  uint64_t budget = 0;  // footprint a wave may hold
  std::mutex m;
  std::condition_variable work_cv, done_cv;
  std::deque<Request*> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  uint64_t next_id = 0;
  bool stopping = false;
  kt_server_stats st{};
  std::thread worker;

  // Same estimate as the batch driver's waves: keys, sort buffers, CSR and
  // core state ~ 48 B per edge record and 40 B per vertex id.
  static uint64_t footprint_of(const kt::BatchItem& it) { return 48 * it.nkeys + 40 * it.n; }

  kt_status submit(std::unique_ptr<Request> r, uint64_t* id_out) {
    r->footprint = footprint_of(r->item);
    if (r->footprint > budget) return KT_ERR_LIMIT;
    std::lock_guard<std::mutex> lk(m);
    if (stopping) return KT_ERR_INVALID;
    r->id = next_id++;
    r->submitted = Clock::now();
    if (id_out) *id_out = r->id;
    queue.push_back(r.get());
    reqs.emplace(r->id, std::move(r));
    st.submitted++;
    work_cv.notify_one();
    return KT_OK;
  }

  void run() {
    kt::Ctx* c = &ctx->c;
    cudaSetDevice(c->device);
    while (true) {
      std::vector<Request*> wave;
      {
        std::unique_lock<std::mutex> lk(m);
        work_cv.wait(lk, [&] { return stopping || !queue.empty(); });
        if (queue.empty()) break;  // stopping and drained
        // Admission: arrival order, while the footprint fits.
        uint64_t bytes = 0;
        while (!queue.empty() && wave.size() < max_wave) {
          Request* r = queue.front();
          if (!wave.empty() && bytes + r->footprint > budget) break;
          bytes += r->footprint;
          wave.push_back(r);
          queue.pop_front();
        }
      }
      const Clock::time_point t_admit = Clock::now();
      std::vector<kt::BatchItem*> items;
      items.reserve(wave.size());
      for (Request* r : wave) {
        r->admitted = t_admit;
        items.push_back(&r->item);
      }
      kt_status status = KT_OK;
      uint64_t peak = 0;
      {
        std::lock_guard<std::recursive_mutex> lk(c->mu);
        try {
          kt::reset_words(c);
          kt::solve_wave(c, items);
          kt::sync(c);
        } catch (const kt::Error& e) {
          c->set_error(e.what());
          status = e.status;
        } catch (const std::bad_alloc&) {
          c->set_error("host allocation failed");
          status = KT_ERR_NOMEM;
        } catch (const std::exception& e) {
          c->set_error(e.what());
          status = KT_ERR_CUDA;
        }
        try {
          c->timer.resolve();
        } catch (...) {
        }
        peak = c->peak;
      }
      const Clock::time_point t_done = Clock::now();
      std::lock_guard<std::mutex> lk(m);
      const uint32_t wave_no = (uint32_t)st.waves++;
      st.ms_busy += ms_between(t_admit, t_done);
      if (wave.size() > st.max_wave_graphs) st.max_wave_graphs = wave.size();
      for (Request* r : wave) {
        r->finished = t_done;
        r->done = true;
        r->result.status = status;
        r->result.kmax = status == KT_OK ? r->item.kmax : 0;
        r->result.edges = status == KT_OK ? r->item.count : 0;
        r->result.ms_wait = ms_between(r->submitted, r->admitted);
        r->result.ms_latency = ms_between(r->submitted, r->finished);
        r->result.wave = wave_no;
        r->result.wave_graphs = (uint32_t)wave.size();
        r->item.extra.clear();
        r->item.extra.shrink_to_fit();
        st.completed++;
      }
      st.device_bytes_peak = peak;
      done_cv.notify_all();
    }
  }
};

extern "C" {

kt_status kt_server_create(kt_ctx* ctx, uint32_t max_wave_graphs, kt_server** out) {
  if (!ctx || !out) return KT_ERR_INVALID;
  *out = nullptr;
  kt_server* s = new (std::nothrow) kt_server;
  if (!s) return KT_ERR_NOMEM;
  s->ctx = ctx;
  s->max_wave = max_wave_graphs ? std::min<uint32_t>(max_wave_graphs, 65535) : 65535;
  {
    std::lock_guard<std::recursive_mutex> lk(ctx->c.mu);
    const kt::Ctx& c = ctx->c;
    s->budget = (c.budget > c.in_use ? c.budget - c.in_use : 0) / 2;
  }
  try {
    s->worker = std::thread([s] { s->run(); });
  } catch (...) {
    delete s;
    return KT_ERR_NOMEM;
  }
  *out = s;
  return KT_OK;
}

kt_status kt_server_submit_pairs(kt_server* s, const uint64_t* xy, uint64_t count, uint64_t* request_id) {
  if (!s || (!xy && count)) return KT_ERR_INVALID;
  try {
    std::unique_ptr<Request> r(new Request);
    r->item.from_pairs(xy, count);
    if (r->item.n >= (1ull << 28)) return KT_ERR_LIMIT;
    return s->submit(std::move(r), request_id);
  } catch (const std::bad_alloc&) {
    return KT_ERR_NOMEM;
  }
}

kt_status kt_server_submit_mix(kt_server* s, uint64_t index, uint64_t base_seed, uint64_t* request_id) {
  if (!s) return KT_ERR_INVALID;
  try {
    std::unique_ptr<Request> r(new Request);
    r->item.from_mix(index, base_seed);
    return s->submit(std::move(r), request_id);
  } catch (const std::bad_alloc&) {
    return KT_ERR_NOMEM;
  }
}

kt_status kt_server_wait(kt_server* s, uint64_t request_id, uint32_t timeout_ms, kt_request_result* out) {
  if (!s) return KT_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->m);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) return KT_ERR_INVALID;
  Request* r = it->second.get();
  if (!r->done && timeout_ms)
    s->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->done; });
  if (!r->done) return KT_ERR_TIMEOUT;
  if (out) *out = r->result;
  return KT_OK;
}

kt_status kt_server_get_stats(kt_server* s, kt_server_stats* out) {
  if (!s || !out) return KT_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->m);
  *out = s->st;
  out->pending = s->queue.size();
  return KT_OK;
}

void kt_server_destroy(kt_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->m);
    s->stopping = true;
  }
  s->work_cv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  delete s;
}

}  // extern "C"
