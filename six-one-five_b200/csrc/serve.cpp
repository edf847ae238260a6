// serve.cpp -- the serving loop: requests from any thread, continuous batching
// on one worker thread, admission against the context's HBM budget.
//
// The reference runs one campaign per process (fourcore_cls5_gpu_v4.cu:412-563,
// solve_617_v1.cu:1907-1970) and has no serving mode; this is the engine's
// own request loop around the same batch calls (s615_prepare / s615_run_batch /
// s615_batch_results / s615_verify).
//
//  * s615_submit copies the caller's units into a pending request and returns
//    a ticket at once.
//  * The worker takes every pending request for the same (table, flags), up
//    to max_batch_units units, as one batch: requests that arrive while
//    others run join the next batch, and a batch is launched as soon as one of
//    `slots` streams is free and its device buffers fit the HBM budget.
//    Batches on different streams overlap on the device (a new persistent
//    grid fills SMs as the previous one drains).
//  * When a batch's event completes, its hits are verified and split back
//    per request (unit indices rebased to the request); results wait for
//    s615_poll and stay readable until s615_release.
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "engine.hpp"

namespace s615 {

namespace {

using Clock = std::chrono::steady_clock;

thread_local bool t_worker = false;

struct Req {
  uint64_t ticket = 0;
  int table = 0;
  unsigned flags = 0;
  std::vector<s615_unit> units;
  Clock::time_point t_submit, t_start;
};

struct Done {
  s615_result r{};
  std::vector<s615_hit> hits;
  std::vector<s615_solution> sols;
};

struct Flight {
  Clock::time_point t_take, t_launched;
  double prep_ms = 0;
  std::vector<Req> reqs;
  std::vector<s615_unit> all;
  s615_batch* b = nullptr;
  int table = 0;
  unsigned flags = 0;
  int slot = 0;
  cudaEvent_t ev = nullptr;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct Server {
  s615_ctx* ctx = nullptr;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req> pending;
  std::map<uint64_t, Done> done;
  std::deque<uint64_t> ready;
  bool stop = false, running = false;
  int slots = 1;
  size_t max_units = 1u << 20;
  uint64_t next_ticket = 1;
  std::vector<cudaStream_t> streams;
  std::vector<bool> busy;
  std::vector<s615_batch*> slot_batch;   // one reused batch per stream slot
  std::thread th;
  bool trace = std::getenv("S615_TRACE") != nullptr;   // per-batch phase times on stderr

  void complete(std::vector<Req>& reqs, int status, const Flight* f,
                const std::vector<s615_hit>* hits, const std::vector<s615_solution>* sols,
                const s615_counters* ctr) {
    const auto now = Clock::now();
    std::vector<std::pair<uint64_t, Done>> out;
    size_t off = 0;
    for (Req& q : reqs) {
      Done d;
      d.r.ticket = q.ticket;
      d.r.status = status;
      d.r.table_id = q.table;
      d.r.n_units = q.units.size();
      d.r.batch_requests = (uint32_t)reqs.size();
      if (ctr) d.r.counters = *ctr;
      const size_t lo = off, hi = off + q.units.size();
      if (status == S615_OK && hits && sols) {
        for (const s615_hit& h : *hits)
          if (h.unit >= lo && h.unit < hi) {
            s615_hit x = h;
            x.unit -= (uint32_t)lo;
            d.hits.push_back(x);
          }
        for (const s615_solution& s : *sols)
          if (s.unit >= lo && s.unit < hi) {
            s615_solution x = s;
            x.unit -= (uint32_t)lo;
            d.sols.push_back(x);
          }
      }
      off = hi;
      d.r.queued_ms = f ? ms_between(q.t_submit, q.t_start) : ms_between(q.t_submit, now);
      d.r.latency_ms = ms_between(q.t_submit, now);
      out.emplace_back(q.ticket, std::move(d));
    }
    std::lock_guard<std::mutex> lk(mu);
    for (auto& kv : out) {
      Done& d = done[kv.first] = std::move(kv.second);
      d.r.n_hits = d.hits.size();
      d.r.n_solutions = d.sols.size();
      d.r.hits = d.hits.empty() ? nullptr : d.hits.data();
      d.r.solutions = d.sols.empty() ? nullptr : d.sols.data();
      ready.push_back(kv.first);
    }
    cv_done.notify_all();
  }

  // Download, verify and split one finished batch.
  void finish(Flight& f, int status) {
    NvtxRange nvtx("serve: results + verify");
    const auto t_done = Clock::now();
    std::vector<s615_hit> hits;
    std::vector<s615_solution> sols;
    s615_counters ctr{};
    if (status == S615_OK) {   // counters first, then exactly the hits there are
      size_t nh = 0;
      status = s615_batch_results(ctx, f.b, nullptr, 0, &nh, &ctr);
      if (status == S615_E_OVERFLOW && nh <= f.b->hit_cap) {
        hits.resize(nh);
        status = s615_batch_results(ctx, f.b, hits.data(), nh, &nh, &ctr);
      }
    }
    if (status == S615_OK && !hits.empty()) {
      const DevTable* t = nullptr;
      auto it = ctx->tables.find(f.table);
      if (it != ctx->tables.end()) t = &it->second;
      if (!t) {
        status = S615_E_NOTABLE;
      } else {
        sols.resize(4 * hits.size() + 64);
        size_t ns = 0;
        status = s615_verify(ctx, f.all.data(), f.all.size(), hits.data(), hits.size(),
                             (int)t->hdr.N, sols.data(), sols.size(), &ns);
        sols.resize(std::min(ns, sols.size()));
      }
    }
    const auto t_verified = Clock::now();
    if (trace)
      std::fprintf(stderr,
                   "[s615 serve] batch of %zu requests / %zu units: prepare %.2f ms, "
                   "device %.2f ms, results+verify %.2f ms, free %.2f ms\n",
                   f.reqs.size(), f.all.size(), f.prep_ms, ms_between(f.t_launched, t_done),
                   ms_between(t_done, t_verified), ms_between(t_verified, Clock::now()));
    if (f.ev) cudaEventDestroy(f.ev);
    f.ev = nullptr;
    busy[f.slot] = false;
    complete(f.reqs, status, &f, &hits, &sols, &ctr);
  }

  // Pending requests of the front request's (table, flags), in order.
  bool take_batch(Flight& f) {
    std::lock_guard<std::mutex> lk(mu);
    if (pending.empty()) return false;
    f.table = pending.front().table;
    f.flags = pending.front().flags;
    size_t units = 0;
    for (auto it = pending.begin(); it != pending.end();) {
      if (it->table == f.table && it->flags == f.flags &&
          (f.reqs.empty() || units + it->units.size() <= max_units)) {
        units += it->units.size();
        f.reqs.push_back(std::move(*it));
        it = pending.erase(it);
      } else {
        ++it;
      }
    }
    return true;
  }

  void put_back(Flight& f) {
    std::lock_guard<std::mutex> lk(mu);
    for (auto it = f.reqs.rbegin(); it != f.reqs.rend(); ++it) pending.push_front(std::move(*it));
    f.reqs.clear();
  }

  void loop() {
    t_worker = true;
    cudaSetDevice(ctx->device);
    std::vector<Flight> flights;
    for (;;) {
      // 1. batches whose work is done
      for (size_t i = 0; i < flights.size();) {
        const cudaError_t e = cudaEventQuery(flights[i].ev);
        if (e == cudaErrorNotReady) { ++i; continue; }
        finish(flights[i], e == cudaSuccess ? S615_OK : cuda_status(e));
        flights.erase(flights.begin() + i);
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        if (stop && pending.empty() && flights.empty()) break;
      }
      // 2. admit while a stream is free and the batch fits the budget
      while ((int)flights.size() < slots) {
        Flight f;
        if (!take_batch(f)) break;
        for (const Req& q : f.reqs) f.all.insert(f.all.end(), q.units.begin(), q.units.end());
        int slot = 0;
        while (busy[slot]) ++slot;
        if (!slot_batch[slot]) slot_batch[slot] = new s615_batch();
        f.t_take = Clock::now();
        f.b = slot_batch[slot];
        nvtxRangePushA("serve: prepare batch");
        int s = fill_batch(ctx, f.all.data(), f.all.size(), f.b);
        nvtxRangePop();
        f.prep_ms = ms_between(f.t_take, Clock::now());
        if (s == S615_E_OOM && !flights.empty()) {   // wait for memory to free up
          put_back(f);
          break;
        }
        if (s != S615_OK) {
          complete(f.reqs, s, nullptr, nullptr, nullptr, nullptr);
          continue;
        }
        f.slot = slot;
        busy[slot] = true;
        const auto now = Clock::now();
        for (Req& q : f.reqs) q.t_start = now;
        s = s615_run_batch(ctx, f.table, f.b, f.flags, streams[slot]);
        if (s == S615_OK && cudaEventCreateWithFlags(&f.ev, cudaEventDisableTiming) != cudaSuccess)
          s = S615_E_DEVICE;
        if (s == S615_OK && cudaEventRecord(f.ev, streams[slot]) != cudaSuccess) s = S615_E_DEVICE;
        f.t_launched = Clock::now();
        if (s != S615_OK) {
          cudaStreamSynchronize(streams[slot]);
          finish(f, s);
          continue;
        }
        flights.push_back(std::move(f));
      }
      // 3. wait for work or for the device
      if (flights.empty()) {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait_for(lk, std::chrono::milliseconds(50), [&] { return stop || !pending.empty(); });
      } else {
        std::this_thread::sleep_for(std::chrono::microseconds(50));
      }
    }
  }
};

bool serving_blocks(s615_ctx* ctx) { return ctx && ctx->server && ctx->server->running && !t_worker; }

void server_destroy(s615_ctx* ctx) {
  if (!ctx || !ctx->server) return;
  s615_serve_stop(ctx);
  for (s615_batch* b : ctx->server->slot_batch)
    if (b) s615_batch_free(ctx, b);
  for (cudaStream_t s : ctx->server->streams) cudaStreamDestroy(s);
  delete ctx->server;
  ctx->server = nullptr;
}

}  // namespace s615

using namespace s615;

extern "C" {

int s615_serve_start(s615_ctx* ctx, int slots, size_t max_batch_units) {
  if (!ctx || slots < 1 || slots > 16) return S615_E_ARG;
  if (ctx->server && ctx->server->running) return S615_E_BUSY;
  server_destroy(ctx);
  cudaSetDevice(ctx->device);
  auto* sv = new Server();
  sv->ctx = ctx;
  sv->slots = slots;
  sv->max_units = max_batch_units ? std::min<size_t>(max_batch_units, kMaxBatchUnits) : (1u << 20);
  sv->busy.assign(slots, false);
  sv->slot_batch.assign(slots, nullptr);
  for (int i = 0; i < slots; ++i) {
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      for (cudaStream_t x : sv->streams) cudaStreamDestroy(x);
      delete sv;
      return S615_E_DEVICE;
    }
    sv->streams.push_back(s);
  }
  sv->running = true;
  ctx->server = sv;
  sv->th = std::thread([sv] { sv->loop(); });
  return S615_OK;
}

int s615_submit(s615_ctx* ctx, int table_id, const s615_unit* units, size_t n, unsigned flags,
                uint64_t* ticket) {
  if (!ctx || !ticket || (n && !units) || n > kMaxBatchUnits) return S615_E_ARG;
  Server* sv = ctx->server;
  if (!sv || !sv->running) return S615_E_ARG;
  Req q;
  q.table = table_id;
  q.flags = flags & ~S615_F_PLAIN;
  q.units.assign(units, units + n);
  q.t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) return S615_E_ARG;
    q.ticket = sv->next_ticket++;
    *ticket = q.ticket;
    sv->pending.push_back(std::move(q));
  }
  sv->cv_work.notify_one();
  return S615_OK;
}

int s615_poll(s615_ctx* ctx, s615_result* out, size_t cap, size_t* n, int wait_ms) {
  if (!ctx || !n || (cap && !out)) return S615_E_ARG;
  *n = 0;
  Server* sv = ctx->server;
  if (!sv) return S615_E_ARG;
  std::unique_lock<std::mutex> lk(sv->mu);
  if (sv->ready.empty() && wait_ms > 0)
    sv->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !sv->ready.empty(); });
  while (*n < cap && !sv->ready.empty()) {
    const uint64_t t = sv->ready.front();
    sv->ready.pop_front();
    out[(*n)++] = sv->done[t].r;
  }
  return S615_OK;
}

int s615_release(s615_ctx* ctx, uint64_t ticket) {
  if (!ctx || !ctx->server) return S615_E_ARG;
  std::lock_guard<std::mutex> lk(ctx->server->mu);
  return ctx->server->done.erase(ticket) ? S615_OK : S615_E_ARG;
}

int s615_serve_stop(s615_ctx* ctx) {
  if (!ctx || !ctx->server) return S615_E_ARG;
  Server* sv = ctx->server;
  if (!sv->running) return S615_OK;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  if (sv->th.joinable()) sv->th.join();
  sv->running = false;
  return S615_OK;
}

}  // extern "C"
