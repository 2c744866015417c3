// Serving loop with continuous batching.
//
// Requests arrive on a schedule (Poisson by default).  Upload threads unpack
// each arrival on the host and admit it into the device-resident pool as soon
// as the pool has room for its words (admission by free HBM); the calling
// thread dispatches: whenever a batch slot is free it takes every admitted
// event that is waiting (up to max_batch events and the slot's word capacity),
// gathers them out of the pool and launches the captured chain.  Batches on
// different slots overlap on the device; each event's latency runs from its
// arrival to the moment the host sees its batch finished.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <deque>
#include <mutex>
#include <random>
#include <thread>
#include <vector>

#include "runtime.h"

namespace pixgpu {
int poolStage(pg_ctx* c, const uint8_t* raw, size_t size, uint32_t* stager, uint32_t* nWords);
int poolCommit(pg_ctx* c, uint32_t stager, uint32_t nWords, uint32_t* handle);
void poolUnstage(pg_ctx* c, uint32_t stager);
int captureGraphFor(pg_ctx* c, Slot& s, uint32_t n);
}  // namespace pixgpu

using namespace pixgpu;

namespace {

using Clock = std::chrono::steady_clock;

struct Ready {
  uint32_t request, handle, nWords;
};

double seconds(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  // nearest rank
  size_t r = size_t(std::ceil(q * double(v.size())));
  r = std::min(std::max<size_t>(r, 1), v.size());
  return v[r - 1];
}

}  // namespace

extern "C" {

void pg_default_serve_config(pg_serve_config* s) {
  s->n_requests = 1000;
  s->rate_hz = 10000.0;
  s->seed = 1;
  s->max_batch = 0;
  s->upload_threads = 2;
}

int pg_prepare(pg_ctx* c, uint32_t maxBatch) {
  if (!c) return PG_ERR_ARG;
  if (!c->cfg.use_graphs) return PG_OK;
  cudaSetDevice(c->cfg.device);
  maxBatch = std::min(maxBatch ? maxBatch : c->cfg.max_events, c->cfg.max_events);
  for (auto& s : c->slots)
    for (uint32_t n = 1; n <= maxBatch; ++n) {
      int rc = captureGraphFor(c, s, n);
      if (rc != PG_OK) return rc;
    }
  return PG_OK;
}

int pg_serve(pg_ctx* c, uint32_t nRaw, const uint8_t* const* raws, const size_t* sizes, const pg_serve_config* cfgIn,
             const double* arrivals, const uint32_t* requestEvent, pg_serve_stats* stats, double* latencies,
             pg_result_fn fn, void* user) {
  if (!c || nRaw == 0 || !raws || !sizes || !stats) return PG_ERR_ARG;
  if (!c->pool.dWords) return fail(c, PG_ERR_ARG, "pg_serve needs a context with a pool (pool_words > 0)");
  pg_serve_config cfg;
  if (cfgIn)
    cfg = *cfgIn;
  else
    pg_default_serve_config(&cfg);
  const uint32_t N = cfg.n_requests;
  if (N == 0) return PG_ERR_ARG;
  const uint32_t maxBatch = std::min(cfg.max_batch ? cfg.max_batch : c->cfg.max_events, c->cfg.max_events);
  const uint32_t nUp = std::max(1u, std::min(cfg.upload_threads, 16u));
  for (auto& s : c->slots)
    if (s.state != SlotState::kFree) return fail(c, PG_ERR_BUSY, "pg_serve needs every slot free");
  cudaSetDevice(c->cfg.device);
  int rc = pg_prepare(c, maxBatch);
  if (rc != PG_OK) return rc;

  // schedule
  std::vector<double> arr(N);
  if (arrivals) {
    for (uint32_t i = 0; i < N; ++i) arr[i] = arrivals[i];
  } else {
    if (!(cfg.rate_hz > 0)) return PG_ERR_ARG;
    std::mt19937_64 rng(cfg.seed);
    std::exponential_distribution<double> gap(cfg.rate_hz);
    double t = 0;
    for (uint32_t i = 0; i < N; ++i) {
      arr[i] = t;
      t += gap(rng);
    }
  }
  for (uint32_t i = 1; i < N; ++i)
    if (arr[i] < arr[i - 1]) return fail(c, PG_ERR_ARG, "arrival times must not decrease");
  std::vector<uint32_t> evOf(N);
  for (uint32_t i = 0; i < N; ++i) {
    evOf[i] = requestEvent ? requestEvent[i] : i % nRaw;
    if (evOf[i] >= nRaw) return fail(c, PG_ERR_ARG, "request_event out of range");
  }

  std::vector<double> lat(N, 0.0);
  std::deque<Ready> ready;
  std::mutex readyMu;
  std::atomic<uint32_t> nextReq{0};
  std::atomic<int> abortRc{PG_OK};
  std::atomic<uint32_t> admissionWaits{0};
  std::string abortMsg;
  std::mutex abortMu;
  auto abortWith = [&](int code) {
    std::lock_guard<std::mutex> lk(abortMu);
    if (abortRc.load() == PG_OK) {
      abortMsg = lastError(c);
      abortRc.store(code);
    }
  };

  const Clock::time_point t0 = Clock::now() + std::chrono::milliseconds(2);
  auto uploader = [&]() {
    cudaSetDevice(c->cfg.device);
    for (;;) {
      uint32_t r = nextReq.fetch_add(1);
      if (r >= N || abortRc.load() != PG_OK) return;
      const Clock::time_point due = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arr[r]));
      while (Clock::now() < due) {
        if (abortRc.load() != PG_OK) return;
        std::this_thread::yield();
      }
      uint32_t st = 0, nw = 0, h = 0;
      int s;
      while ((s = poolStage(c, raws[evOf[r]], sizes[evOf[r]], &st, &nw)) == PG_ERR_BUSY) {
        if (abortRc.load() != PG_OK) return;
        std::this_thread::yield();
      }
      if (s != PG_OK) {
        abortWith(s);
        return;
      }
      if (nw > c->cfg.max_words_per_batch) {
        poolUnstage(c, st);
        fail(c, PG_ERR_CAPACITY, "event larger than a batch slot");
        abortWith(PG_ERR_CAPACITY);
        return;
      }
      bool waited = false;
      while ((s = poolCommit(c, st, nw, &h)) == PG_ERR_NOMEM) {
        waited = true;
        if (abortRc.load() != PG_OK) {
          poolUnstage(c, st);
          return;
        }
        std::this_thread::yield();
      }
      if (waited) admissionWaits.fetch_add(1);
      if (s != PG_OK) {
        poolUnstage(c, st);
        abortWith(s);
        return;
      }
      std::lock_guard<std::mutex> lk(readyMu);
      ready.push_back(Ready{r, h, nw});
    }
  };
  std::vector<std::thread> ups;
  for (uint32_t i = 0; i < nUp; ++i) ups.emplace_back(uploader);

  // dispatcher
  const size_t S = c->slots.size();
  std::vector<std::vector<uint32_t>> inflight(S);
  std::vector<uint32_t> handles;
  uint32_t completed = 0, batches = 0, maxSeen = 0;
  uint64_t batchedEvents = 0;
  Clock::time_point last = t0;
  while (completed < N && abortRc.load() == PG_OK) {
    bool progress = false;
    for (size_t k = 0; k < S; ++k) {
      if (inflight[k].empty()) continue;
      int q = pg_query(c, uint32_t(k));
      if (q == PG_ERR_BUSY) continue;
      const Clock::time_point now = Clock::now();
      if (q != PG_OK) {
        abortWith(q);
        break;
      }
      for (size_t i = 0; i < inflight[k].size(); ++i) {
        uint32_t r = inflight[k][i];
        lat[r] = seconds(t0, now) - arr[r];
        if (fn) {
          pg_result_view v;
          if (pg_result(c, uint32_t(k), uint32_t(i), &v) == PG_OK) fn(user, r, evOf[r], &v);
        }
      }
      completed += uint32_t(inflight[k].size());
      last = now;
      inflight[k].clear();
      int rr = pg_release(c, uint32_t(k));
      if (rr != PG_OK) {
        abortWith(rr);
        break;
      }
      progress = true;
    }
    for (;;) {
      int k = -1;
      for (size_t j = 0; j < S; ++j)
        if (inflight[j].empty() && c->slots[j].state == SlotState::kFree) {
          k = int(j);
          break;
        }
      if (k < 0) break;
      std::vector<uint32_t> reqs;
      handles.clear();
      {
        std::lock_guard<std::mutex> lk(readyMu);
        uint64_t words = 0;
        while (!ready.empty() && reqs.size() < maxBatch && words + ready.front().nWords <= c->cfg.max_words_per_batch) {
          words += ready.front().nWords;
          reqs.push_back(ready.front().request);
          handles.push_back(ready.front().handle);
          ready.pop_front();
        }
      }
      if (reqs.empty()) break;
      uint32_t slot = 0;
      int s = pg_submit_pooled(c, uint32_t(handles.size()), handles.data(), 0, &slot);
      if (s != PG_OK) {
        abortWith(s);
        // a refused batch leaves its events admitted: give their extents back
        for (uint32_t h : handles) pg_pool_release(c, h);
        break;
      }
      inflight[slot] = std::move(reqs);
      ++batches;
      batchedEvents += inflight[slot].size();
      maxSeen = std::max<uint32_t>(maxSeen, uint32_t(inflight[slot].size()));
      progress = true;
    }
    if (!progress) std::this_thread::yield();
  }
  if (abortRc.load() != PG_OK) nextReq.store(N);
  for (auto& t : ups) t.join();
  // drain anything still in flight after an abort, and give back the pool
  // extents of events that were admitted but never batched
  for (size_t k = 0; k < S; ++k)
    if (!inflight[k].empty()) pg_release(c, uint32_t(k));
  for (const Ready& r : ready) pg_pool_release(c, r.handle);
  ready.clear();
  if (abortRc.load() != PG_OK) return fail(c, abortRc.load(), abortMsg);

  std::vector<double> ms(N);
  double sum = 0, mx = 0;
  for (uint32_t i = 0; i < N; ++i) {
    ms[i] = lat[i] * 1e3;
    sum += ms[i];
    mx = std::max(mx, ms[i]);
    if (latencies) latencies[i] = lat[i];
  }
  stats->completed = completed;
  stats->batches = batches;
  stats->max_batch_seen = maxSeen;
  stats->admission_waits = admissionWaits.load();
  stats->wall_s = seconds(t0, last);
  stats->events_per_s = stats->wall_s > 0 ? double(completed) / stats->wall_s : 0.0;
  stats->mean_batch = batches ? double(batchedEvents) / batches : 0.0;
  stats->offered_hz = arr[N - 1] > 0 ? double(N - 1) / arr[N - 1] : 0.0;
  stats->p50_ms = percentile(ms, 0.50);
  stats->p90_ms = percentile(ms, 0.90);
  stats->p99_ms = percentile(ms, 0.99);
  stats->mean_ms = sum / N;
  stats->max_ms = mx;
  return PG_OK;
}

}  // extern "C"
