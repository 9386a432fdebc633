// Serving: a continuous-batching request loop over the batch path.
//
// Requests (graphs) are submitted from any host thread and queue in arrival
// order.  The server runs `lanes` workers (option serve_lanes, default 2);
// each owns a context of its own on the device -- lane 0 the server's
// context, the others contexts the server creates with the same options --
// with its own stream, device words and budget.  Whenever a lane is free it
// admits queued requests, oldest first, while their estimated device
// footprint fits the lane's share of the budget (and up to a graph cap) --
// with two or more lanes, the last lane admits only small requests
// (footprint up to serve_small_mb), so they never queue behind a wave of
// large graphs; it launches nothing cooperative, and the other lanes'
// cooperative grids take 75% of the resident blocks, so its waves run beside
// theirs -- and
// solves the admitted set as one wave -- one disjoint union through every
// stage, each graph on its own peel levels (batch.cu).  So while one wave is
// on the device, requests that arrive meanwhile start in the next free lane
// instead of waiting for that wave to end, and the two waves' kernels
// overlap on the device.  Cooperative launches (which take every SM's
// resident-block slots) of the lanes run one at a time; everything else
// overlaps.  The result of a request does not depend on which wave or lane
// it joined or on its wave-mates: triangles never cross graphs in a union.
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
  struct Lane {
    kt_ctx* ctx = nullptr;
    bool owned = false;  // created by the server (lanes after the first)
    std::thread worker;
  };
  kt_ctx* ctx = nullptr;
  uint32_t max_wave = 0;
  uint64_t budget = 0;  // footprint one wave may hold (a lane's share)
  std::mutex m;
  std::condition_variable work_cv, done_cv;
  std::deque<Request*> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  uint64_t next_id = 0;
  bool stopping = false;
  kt_server_stats st{};
  std::vector<Lane> lanes;
  std::mutex coop;  // cooperative launches of the lanes, one at a time
  uint64_t small_bytes = 0;  // the small lane (the last) admits only requests this small (0: any)
  bool partition = false;    // ... and the other lanes only larger ones
  int64_t lane0_coop_pct = 100;  // the server's context's coop_occupancy_pct, restored at the end
  // Whether a lane admits a request: the small lane only small ones; with
  // the partition the other lanes only the others.
  bool admits(bool small_lane, const Request* r) const {
    if (!small_bytes || lanes.size() < 2) return true;
    if (small_lane) return r->footprint <= small_bytes;
    return !partition || r->footprint > small_bytes;
  }
  bool queue_has_for(bool small_lane) const {
    for (const Request* r : queue)
      if (admits(small_lane, r)) return true;
    return false;
  }

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
    work_cv.notify_all();  // every free lane looks: the small lane may not take it
    return KT_OK;
  }

  void run(kt_ctx* lane_ctx) {
    kt::Ctx* c = &lane_ctx->c;
    cudaSetDevice(c->device);
    while (true) {
      std::vector<Request*> wave;
      {
        std::unique_lock<std::mutex> lk(m);
        work_cv.wait(lk, [&] { return stopping || !queue.empty(); });
        if (queue.empty()) break;  // stopping and drained
        // Admission: arrival order, while the footprint fits.  With a small
        // lane (the last of two or more, small_bytes > 0) that lane admits only
        // requests of at most small_bytes, skipping larger ones; the other
        // lanes admit any request (with the partition, only larger ones).
        const bool small_lane = lane_ctx == lanes.back().ctx;
        uint64_t bytes = 0;
        for (auto it = queue.begin(); it != queue.end() && wave.size() < max_wave;) {
          Request* r = *it;
          if (!admits(small_lane, r)) {
            ++it;
            continue;
          }
          if (!wave.empty() && bytes + r->footprint > budget) break;
          bytes += r->footprint;
          wave.push_back(r);
          it = queue.erase(it);
        }
        if (wave.empty()) {
          // Only requests of another lane's class are queued: that lane takes
          // them; wait for one of this lane's (or the end).
          if (stopping) break;
          work_cv.wait(lk, [&] { return stopping || queue_has_for(small_lane); });
          continue;
        }
        // Others still queued: wake the other free lanes for them.
        if (!queue.empty()) work_cv.notify_all();
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
        r->result.lane = (uint32_t)lane_of(lane_ctx);
        r->item.extra.clear();
        r->item.extra.shrink_to_fit();
        st.completed++;
      }
      lane_peak[lane_of(lane_ctx)] = peak;
      uint64_t tot = 0;
      for (uint64_t p : lane_peak) tot += p;
      if (tot > st.device_bytes_peak) st.device_bytes_peak = tot;
      done_cv.notify_all();
    }
  }

  std::vector<uint64_t> lane_peak;
  size_t lane_of(kt_ctx* x) const {
    for (size_t i = 0; i < lanes.size(); ++i)
      if (lanes[i].ctx == x) return i;
    return 0;
  }

  // Stops and joins the workers, then frees the lanes' own contexts.
  void shutdown() {
    {
      std::lock_guard<std::mutex> lk(m);
      stopping = true;
    }
    work_cv.notify_all();
    for (Lane& l : lanes)
      if (l.worker.joinable()) l.worker.join();
    for (Lane& l : lanes) {
      if (l.owned) {
        kt_destroy(l.ctx);
      } else if (l.ctx) {
        std::lock_guard<std::recursive_mutex> lk(l.ctx->c.mu);
        l.ctx->c.coop_mu = nullptr;
        l.ctx->c.opt.coop_occupancy_pct = lane0_coop_pct;
      }
      l.ctx = nullptr;
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
  kt::Options opt;
  int device = 0;
  uint64_t ctx_budget = 0;
  uint32_t nlanes = 1;
  {
    std::lock_guard<std::recursive_mutex> lk(ctx->c.mu);
    const kt::Ctx& c = ctx->c;
    opt = c.opt;
    device = c.device;
    ctx_budget = c.budget;
    nlanes = (uint32_t)std::min<int64_t>(std::max<int64_t>(1, c.opt.serve_lanes), 4);
    s->small_bytes = nlanes > 1 ? (uint64_t)std::max<int64_t>(0, c.opt.serve_small_mb) << 20 : 0;
    s->partition = c.opt.serve_partition != 0;
    // Half of the free budget for the waves in flight, shared by the lanes.
    s->budget = (c.budget > c.in_use ? c.budget - c.in_use : 0) / 2 / nlanes;
  }
  s->lanes.resize(nlanes);
  s->lane_peak.assign(nlanes, 0);
  s->lanes[0].ctx = ctx;
  kt_status st = KT_OK;
  for (uint32_t i = 1; i < nlanes && st == KT_OK; ++i) {
    st = kt_init(device, ctx_budget, &s->lanes[i].ctx);
    if (st == KT_OK) {
      s->lanes[i].owned = true;
      s->lanes[i].ctx->c.opt = opt;
    }
  }
  if (st == KT_OK && nlanes > 1)
    for (size_t i = 0; i < s->lanes.size(); ++i) {
      kt::Ctx& lc = s->lanes[i].ctx->c;
      std::lock_guard<std::recursive_mutex> lk(lc.mu);
      lc.coop_mu = &s->coop;
      if (!s->small_bytes || opt.serve_small_coop) continue;
      if (i + 1 == s->lanes.size()) {
        // The small lane launches nothing cooperative (host-stepped rounds,
        // list-mode support), so it never waits for another lane's
        // cooperative grid to end ...
        lc.opt.persistent = 0;
        lc.opt.dense_max_n = 0;
      } else {
        // ... and the other lanes' cooperative grids leave it room on
        // every SM.
        if (i == 0) s->lane0_coop_pct = lc.opt.coop_occupancy_pct;
        lc.opt.coop_occupancy_pct = 75;
      }
    }
  try {
    if (st == KT_OK)
      for (auto& l : s->lanes) {
        kt_ctx* lc = l.ctx;
        l.worker = std::thread([s, lc] { s->run(lc); });
      }
  } catch (...) {
    st = KT_ERR_NOMEM;
  }
  if (st != KT_OK) {
    s->shutdown();
    delete s;
    return st;
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
  s->shutdown();
  delete s;
}

}  // extern "C"
