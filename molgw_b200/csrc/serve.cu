// Request loop for G0W0 solves (continuous batching).
//
// Worker threads each own a library context (stream, plan cache, a share of the
// HBM budget).  A free worker takes the requests waiting at that moment, in
// arrival order, as long as their fused footprints fit its share (a single
// request larger than the share is split into frequency chunks by the
// scheduler), and runs them as one batch.  Requests that arrive meanwhile wait
// for the next free worker; batches of different workers run concurrently on
// the GPU on their own streams.  Waits are bounded by the caller's timeout.
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
  bool done = false;
  int status = RIGW_OK;
  std::string err;
};

struct Server {
  int device = 0;
  int max_batch = 64;
  size_t share = 0;
  std::vector<std::unique_ptr<Context>> ctx;
  std::vector<std::thread> threads;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> live;
  uint64_t next_ticket = 1;
  bool stop = false;
  std::atomic<long long> completed{0}, batches{0};

  void worker(int w) {
    cudaSetDevice(device);
    Context& c = *ctx[w];
    for (;;) {
      std::vector<std::shared_ptr<Request>> batch;
      {
        std::unique_lock<std::mutex> lock(mu);
        cv_work.wait(lock, [&] { return stop || !queue.empty(); });
        if (queue.empty()) return;   // stop requested and nothing left
        size_t used = 0;
        while (!queue.empty() && int(batch.size()) < max_batch) {
          auto& r = queue.front();
          if (!batch.empty() && used + r->bytes > share) break;
          used += r->bytes;
          batch.push_back(r);
          queue.pop_front();
        }
      }
      std::vector<rigw_problem> probs(batch.size());
      std::vector<rigw_result> res(batch.size());
      for (size_t k = 0; k < batch.size(); ++k) {
        probs[k] = batch[k]->prob;
        res[k] = *batch[k]->res;
      }
      Status s = solve_batch(c, int(batch.size()), probs.data(), res.data());
      batches++;
      {
        std::lock_guard<std::mutex> lock(mu);
        for (size_t k = 0; k < batch.size(); ++k) {
          *batch[k]->res = res[k];
          batch[k]->status = s.code;
          batch[k]->err = s.msg;
          batch[k]->done = true;
        }
        completed += (long long)batch.size();
      }
      cv_done.notify_all();
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
    budget = size_t(double(free_b) * 0.85);
  }
  auto* s = new (std::nothrow) rigw_server();
  if (!s) return RIGW_ERR_NOMEM;
  rigw::Server& S = s->impl;
  S.device = device;
  S.max_batch = max_batch;
  S.share = budget / size_t(workers);
  for (int w = 0; w < workers; ++w) {
    S.ctx.emplace_back(new rigw::Context());
    rigw::Status st = S.ctx.back()->init(device, S.share);
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
  {
    std::lock_guard<std::mutex> lock(srv->impl.mu);
    if (srv->impl.stop) return RIGW_ERR_ARG;
    r->ticket = srv->impl.next_ticket++;
    srv->impl.live[r->ticket] = r;
    srv->impl.queue.push_back(r);
    *ticket = r->ticket;
  }
  srv->impl.cv_work.notify_one();
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
  if (queued) *queued = (long long)srv->impl.queue.size();
  return RIGW_OK;
}

RIGW_API int rigw_server_destroy(rigw_server* srv) {
  if (!srv) return RIGW_ERR_ARG;
  {
    std::lock_guard<std::mutex> lock(srv->impl.mu);
    srv->impl.stop = true;
  }
  srv->impl.cv_work.notify_all();
  for (auto& t : srv->impl.threads) t.join();
  delete srv;
  return RIGW_OK;
}

}  // extern "C"
