// Request loop for G0W0 solves (continuous batching).
//
// Worker threads each own a library context (stream, plan cache, a share of the
// HBM budget).  Requests are admitted by their fused device footprint into two
// lanes: large (footprint above 1/kLargeShare of a worker's share) and small.
// A free worker takes the requests of one lane waiting at that moment, in
// arrival order, as long as their footprints fit its share (a single request
// larger than the share is split into frequency chunks by the scheduler), and
// runs them as one batch.  Small requests go first; at most one large request
// runs at a time, and it starts when no small request waits or when the oldest
// large request has waited kLargeAgeNs (so neither lane starves).  With two or
// more workers, worker 0 takes only small batches and runs on high-priority
// streams, the others on low-priority ones.  A large batch
// that finds no memory while other workers hold theirs goes back to the front of
// its lane; no new small batch starts until it is taken again, which happens as
// soon as another batch completes.  Requests
// that arrive meanwhile wait for the next free worker; batches of different
// workers run concurrently on the GPU on their own streams.  Waits are bounded
// by the caller's timeout.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.cuh"

namespace rigw {

struct Request {
  uint64_t ticket = 0;
  rigw_problem prob{};
  rigw_result* res = nullptr;
  size_t bytes = 0;
  bool large = false;
  bool done = false;
  int64_t t_submit_ns = 0, t_done_ns = 0;   // steady (monotonic) clock
  int status = RIGW_OK;
  std::string err;
};

inline int64_t steady_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

inline int lane_of(const std::vector<std::shared_ptr<Request>>& batch) { return batch.front()->large ? 1 : 0; }

struct Server {
  int device = 0;
  int max_batch = 64;
  size_t share = 0;
  bool small_lane_worker = false;   // worker 0 takes only small batches (two or more workers)
  std::vector<std::unique_ptr<Context>> ctx;
  std::vector<std::thread> threads;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  static constexpr int kLargeShare = 8;
  static constexpr int64_t kLargeAgeNs = 5000000000ll;
  int large_busy = 0;           // large batches running (under mu)
  std::deque<std::shared_ptr<Request>> queue[2];   // [0] small, [1] large
  std::unordered_map<uint64_t, std::shared_ptr<Request>> live;
  uint64_t next_ticket = 1;
  bool stop = false;
  std::atomic<long long> completed{0}, batches{0};
  int busy = 0;                 // workers running a batch (under mu)
  rigw_server_stats st{};       // counters (under mu)
  int64_t hold_since = 0;
  bool hold_small = false;      // a large request waits for memory: no new small batches

  void worker(int w) {
    cudaSetDevice(device);
    Context& c = *ctx[w];
    for (;;) {
      std::vector<std::shared_ptr<Request>> batch;
      {
        std::unique_lock<std::mutex> lock(mu);
        // lane this worker takes now: -1 none
        auto pick = [&]() -> int {
          const bool large_ready = !queue[1].empty() && large_busy == 0;
          const bool large_aged = large_ready && steady_ns() - queue[1].front()->t_submit_ns > kLargeAgeNs;
          if (w == 0 && small_lane_worker) return (hold_small || queue[0].empty()) ? -1 : 0;
          // a large request sent back for memory goes next: the small lane holds for it
          if (large_ready && (large_aged || queue[0].empty() || hold_small)) return 1;
          if (hold_small) return -1;
          return queue[0].empty() ? -1 : 0;
        };
        int lane = -1;
        // timed waits: a large request can become due by age without any event
        while (!((lane = pick()) >= 0 || stop)) cv_work.wait_for(lock, std::chrono::milliseconds(50));
        if (lane < 0) return;   // stop requested and nothing left for this worker
        std::deque<std::shared_ptr<Request>>& q = queue[lane];
        size_t used = 0;
        while (!q.empty() && int(batch.size()) < max_batch) {
          auto& r = q.front();
          if (!batch.empty() && used + r->bytes > share) break;
          used += r->bytes;
          batch.push_back(r);
          q.pop_front();
        }
        ++busy;
        if (lane == 1) {
          ++large_busy;
          if (hold_small) {   // the large request is on its way: small batches may start again
            hold_small = false;
            st.hold_ns += steady_ns() - hold_since;
          }
        }
        st.batches[lane]++;
      }
      const int64_t t_start = steady_ns();
      std::vector<rigw_problem> probs(batch.size());
      std::vector<rigw_result> res(batch.size());
      for (size_t k = 0; k < batch.size(); ++k) {
        probs[k] = batch[k]->prob;
        res[k] = *batch[k]->res;
      }
      const double b0 = c.host_build_ms, c0 = c.host_capture_ms, a0 = c.host_alloc_ms;
      Status s = solve_batch(c, int(batch.size()), probs.data(), res.data());
      {
        std::lock_guard<std::mutex> lock(mu);
        st.build_ms[lane_of(batch)] += c.host_build_ms - b0;
        st.capture_ms[lane_of(batch)] += c.host_capture_ms - c0;
        st.alloc_ms[lane_of(batch)] += c.host_alloc_ms - a0;
      }
      {
        // out of memory while other workers hold device memory: the batch goes
        // back to the front of its lane and runs after one of them finishes
        std::unique_lock<std::mutex> lock(mu);
        if (s.code == RIGW_ERR_NOMEM && busy > 1 && !stop) {
          --busy;
          if (batch.front()->large) --large_busy;
          st.requeued[batch.front()->large ? 1 : 0]++;
          if (w < RIGW_SERVER_MAX_WORKERS) st.busy_ns[w] += steady_ns() - t_start;
          const long long seen = completed.load();
          if (batch.front()->large && !hold_small) {
            hold_small = true;
            hold_since = steady_ns();
          }
          auto& q = queue[batch.front()->large ? 1 : 0];
          for (auto it = batch.rbegin(); it != batch.rend(); ++it) q.push_front(*it);
          cv_done.wait(lock, [&] { return stop || completed.load() != seen || busy == 0; });
          cv_work.notify_all();
          continue;
        }
      }
      batches++;
      {
        std::lock_guard<std::mutex> lock(mu);
        --busy;
        if (batch.front()->large) --large_busy;
        const int64_t now = steady_ns();
        if (batch.front()->large && hold_small) {
          hold_small = false;
          st.hold_ns += now - hold_since;
        }
        st.completed[batch.front()->large ? 1 : 0] += (long long)batch.size();
        st.device_ms[batch.front()->large ? 1 : 0] += c.last_stats.total_ms;
        if (s.code != RIGW_OK) st.failed += (long long)batch.size();
        if (w < RIGW_SERVER_MAX_WORKERS) st.busy_ns[w] += now - t_start;
        for (size_t k = 0; k < batch.size(); ++k) {
          *batch[k]->res = res[k];
          batch[k]->status = s.code;
          batch[k]->err = s.msg;
          batch[k]->done = true;
          batch[k]->t_done_ns = now;
        }
        completed += (long long)batch.size();
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }
};

}  // namespace rigw

struct rigw_server {
  rigw::Server impl;
};

extern "C" {

RIGW_API int rigw_server_create(rigw_server** srv, int device, size_t hbm_budget_bytes, int workers,
                                int max_batch) {
  if (!srv || workers < 1 || workers > 16 || max_batch < 1) return RIGW_ERR_ARG;
  *srv = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return RIGW_ERR_CUDA;
  size_t budget = hbm_budget_bytes;
  if (!budget) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return RIGW_ERR_CUDA;
    // memory reserved by the stream-ordered pool but unused is free for the loop
    cudaMemPool_t pool;
    uint64_t reserved = 0, used = 0;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
    }
    cudaGetLastError();
    free_b += size_t(reserved > used ? reserved - used : 0);
    budget = size_t(double(free_b) * 0.85);
  }
  auto* s = new (std::nothrow) rigw_server();
  if (!s) return RIGW_ERR_NOMEM;
  rigw::Server& S = s->impl;
  S.device = device;
  S.max_batch = max_batch;
  S.share = budget / size_t(workers);
  S.small_lane_worker = workers > 1;
  for (int w = 0; w < workers; ++w) {
    S.ctx.emplace_back(new rigw::Context());
    // with two or more workers, worker 0 serves the small lane on high-priority streams
    // and the others run on low-priority ones: the block scheduler then hands free SM
    // slots to small batches first, so a large request's long kernels do not hold them up
    const int priority = workers > 1 ? (w == 0 ? 1 : -1) : 0;
    rigw::Status st = S.ctx.back()->init(device, S.share, priority, /*blocking_waits=*/true);
    // the worker's device memory is reserved once: batch plans take their arena
    // from it, so no batch waits for the memory pool to grow
    if (st.good() && S.share > (size_t(2) << 30)) st = S.ctx.back()->reserve(S.share - (size_t(1) << 30));
    if (!st.good()) {
      delete s;
      return st.code;
    }
  }
  for (int w = 0; w < workers; ++w) S.threads.emplace_back([&S, w] { S.worker(w); });
  *srv = s;
  return RIGW_OK;
}

RIGW_API int rigw_server_submit(rigw_server* srv, const rigw_problem* prob, rigw_result* result,
                                uint64_t* ticket) {
  if (!srv || !prob || !result || !ticket) return RIGW_ERR_ARG;
  rigw::Shape sh;
  rigw::Status st = rigw::make_shape(*prob, &sh);
  if (!st.good()) return st.code;
  auto r = std::make_shared<rigw::Request>();
  r->prob = *prob;
  r->res = result;
  r->bytes = rigw::Plan::measure({sh}, rigw::kPlanFused);
  r->large = r->bytes > srv->impl.share / rigw::Server::kLargeShare;
  {
    std::lock_guard<std::mutex> lock(srv->impl.mu);
    if (srv->impl.stop) return RIGW_ERR_ARG;
    r->ticket = srv->impl.next_ticket++;
    r->t_submit_ns = rigw::steady_ns();
    srv->impl.live[r->ticket] = r;
    srv->impl.queue[r->large ? 1 : 0].push_back(r);
    *ticket = r->ticket;
  }
  srv->impl.cv_work.notify_all();
  return RIGW_OK;
}

RIGW_API int rigw_server_poll(rigw_server* srv, uint64_t ticket, int* done) {
  if (!srv || !done) return RIGW_ERR_ARG;
  std::lock_guard<std::mutex> lock(srv->impl.mu);
  auto it = srv->impl.live.find(ticket);
  if (it == srv->impl.live.end()) return RIGW_ERR_ARG;
  *done = it->second->done ? 1 : 0;
  return RIGW_OK;
}

RIGW_API int rigw_server_info(rigw_server* srv, uint64_t ticket, int* done, int64_t* submit_ns, int64_t* done_ns) {
  if (!srv || !done) return RIGW_ERR_ARG;
  std::lock_guard<std::mutex> lock(srv->impl.mu);
  auto it = srv->impl.live.find(ticket);
  if (it == srv->impl.live.end()) return RIGW_ERR_ARG;
  *done = it->second->done ? 1 : 0;
  if (submit_ns) *submit_ns = it->second->t_submit_ns;
  if (done_ns) *done_ns = it->second->t_done_ns;
  return RIGW_OK;
}

RIGW_API int rigw_server_wait(rigw_server* srv, uint64_t ticket, int64_t timeout_ns, char* errbuf,
                              size_t errlen) {
  if (!srv) return RIGW_ERR_ARG;
  std::unique_lock<std::mutex> lock(srv->impl.mu);
  auto it = srv->impl.live.find(ticket);
  if (it == srv->impl.live.end()) return RIGW_ERR_ARG;
  std::shared_ptr<rigw::Request> r = it->second;
  const bool ok = srv->impl.cv_done.wait_for(lock, std::chrono::nanoseconds(timeout_ns), [&] { return r->done; });
  if (!ok) return RIGW_ERR_TIMEOUT;
  srv->impl.live.erase(ticket);
  if (errbuf && errlen) {
    std::strncpy(errbuf, r->err.c_str(), errlen - 1);
    errbuf[errlen - 1] = '\0';
  }
  return r->status;
}

RIGW_API int rigw_server_counters(rigw_server* srv, long long* completed, long long* batches, long long* queued) {
  if (!srv) return RIGW_ERR_ARG;
  std::lock_guard<std::mutex> lock(srv->impl.mu);
  if (completed) *completed = srv->impl.completed.load();
  if (batches) *batches = srv->impl.batches.load();
  if (queued) *queued = (long long)(srv->impl.queue[0].size() + srv->impl.queue[1].size());
  return RIGW_OK;
}

RIGW_API int rigw_server_stats_get(rigw_server* srv, rigw_server_stats* out) {
  if (!srv || !out) return RIGW_ERR_ARG;
  std::lock_guard<std::mutex> lock(srv->impl.mu);
  *out = srv->impl.st;
  out->queued[0] = (long long)srv->impl.queue[0].size();
  out->queued[1] = (long long)srv->impl.queue[1].size();
  out->workers = int(srv->impl.ctx.size());
  return RIGW_OK;
}

RIGW_API int rigw_server_destroy(rigw_server* srv) {
  if (!srv) return RIGW_ERR_ARG;
  {
    // queued requests are cancelled; batches already on the GPU finish
    std::lock_guard<std::mutex> lock(srv->impl.mu);
    srv->impl.stop = true;
    for (auto& q : srv->impl.queue) {
      for (auto& r : q) {
        r->status = RIGW_ERR_CANCELLED;
        r->err = "cancelled: the request loop was destroyed before this request ran";
        r->done = true;
      }
      q.clear();
    }
  }
  srv->impl.cv_work.notify_all();
  srv->impl.cv_done.notify_all();
  for (auto& t : srv->impl.threads) t.join();
  delete srv;
  return RIGW_OK;
}

}  // extern "C"
