// Serving loop of the engine: a worker thread that drains the request queue
// with continuous batching (no counterpart in the reference, whose main loop
// serves one query and one batch at a time, main.cu:152-347).
//
// Batches queued back to back run as one device batch.  That is exact: the
// batch pipeline gives every update the graph state after (insert) or before
// (delete) it in array order, so concatenating requests changes no update's
// result; only the device work per launch grows.  Registrations and
// retirements are barriers between device batches.  Lock order: mu (engine
// state, device work) before rmu (results) or qmu (queue); the worker never
// holds qmu while it takes mu.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>

#include "../host/par.h"
#include "engine_internal.h"

namespace dsm {

namespace {
double ms_between(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}
}  // namespace

int Engine::serve_start(uint32_t max_merge) {
  std::lock_guard<std::mutex> q(srv.qmu);
  if (srv.running) return fail(DSM_ERR_STATE, "the serving loop is already running");
  srv.max_merge = max_merge ? max_merge : 65536;
  srv.stopping = false;
  srv.running = true;
  srv.worker = std::thread([this] { worker_loop(); });
  return DSM_OK;
}

int Engine::serve_stop() {
  {
    std::lock_guard<std::mutex> q(srv.qmu);
    if (!srv.running) return DSM_OK;
    srv.stopping = true;
    srv.work_cv.notify_all();
  }
  srv.worker.join();
  std::lock_guard<std::mutex> q(srv.qmu);
  for (Request &r : srv.pending) post_outcome(r.id, Outcome{DSM_ERR_OOM, 0, "serving stopped before admission"});
  srv.pending.clear();
  srv.running = false;
  srv.stopping = false;
  srv.done_cv.notify_all();
  return DSM_OK;
}

int Engine::register_async(const uint32_t *qoff, const uint32_t *qnbr, const uint32_t *qlab, uint32_t nq,
                           uint64_t *ticket) {
  Request r;
  r.kind = kReqRegister;
  std::string err;
  if (int rc = plan_query(nq, qoff, qnbr, qlab, r.plan, err)) return fail(rc, err);
  r.t_submit = std::chrono::steady_clock::now();
  std::lock_guard<std::mutex> q(srv.qmu);
  if (!srv.running || srv.stopping) return fail(DSM_ERR_STATE, "the serving loop is not running");
  r.id = *ticket = srv.next_ticket++;
  srv.open_tickets.insert(r.id);
  srv.queue.push_back(std::move(r));
  srv.work_cv.notify_one();
  return DSM_OK;
}

int Engine::retire_async(uint32_t qid, uint64_t *ticket) {
  Request r;
  r.kind = kReqRetire;
  r.qid = qid;
  r.t_submit = std::chrono::steady_clock::now();
  std::lock_guard<std::mutex> q(srv.qmu);
  if (!srv.running || srv.stopping) return fail(DSM_ERR_STATE, "the serving loop is not running");
  r.id = *ticket = srv.next_ticket++;
  srv.open_tickets.insert(r.id);
  srv.queue.push_back(std::move(r));
  srv.work_cv.notify_one();
  return DSM_OK;
}

void Engine::post_outcome(uint64_t ticket, const Outcome &o) {
  srv.tickets[ticket] = o;
  srv.open_tickets.erase(ticket);
}

// Each outcome is reported once: afterwards the ticket is forgotten and a
// second call for it returns DSM_ERR_NOT_FOUND.
int Engine::admission(uint64_t ticket, int64_t timeout_ms, uint32_t *qid) {
  std::unique_lock<std::mutex> q(srv.qmu);
  if (ticket == 0 || ticket >= srv.next_ticket) return fail(DSM_ERR_NOT_FOUND, "no such ticket");
  auto ready = [&] { return srv.tickets.count(ticket) != 0 || srv.open_tickets.count(ticket) == 0; };
  if (timeout_ms < 0) srv.done_cv.wait(q, ready);
  else if (!srv.done_cv.wait_for(q, std::chrono::milliseconds(timeout_ms), ready))
    return DSM_ERR_TIMEOUT;
  auto it = srv.tickets.find(ticket);
  if (it == srv.tickets.end()) return fail(DSM_ERR_NOT_FOUND, "ticket outcome already reported");
  const Outcome o = it->second;
  srv.tickets.erase(it);
  if (o.rc) {
    set_error(o.msg);
    return o.rc;
  }
  *qid = o.qid;
  return DSM_OK;
}

// Registrations that wait for memory, first come first served (mu held).
void Engine::admit_pending() {
  for (;;) {
    Request r;
    {
      std::lock_guard<std::mutex> q(srv.qmu);
      if (srv.pending.empty()) return;
      r = std::move(srv.pending.front());
      srv.pending.pop_front();
    }
    uint32_t qid = 0;
    bool later = false;
    const int rc = admit(r.plan, &qid, &later);
    std::lock_guard<std::mutex> q(srv.qmu);
    if (rc == DSM_ERR_OOM && later) {  // still does not fit: keep its place
      srv.pending.push_front(std::move(r));
      return;
    }
    post_outcome(r.id, Outcome{rc, qid, rc ? error_text() : std::string()});
    srv.done_cv.notify_all();
  }
}

Outcome Engine::handle_control(Request &r) {
  std::lock_guard<std::mutex> lk(mu);
  Outcome o;
  if (r.kind == kReqRetire) {
    o.rc = retire_locked(r.qid);
    o.qid = r.qid;
    if (o.rc) o.msg = error_text();
    admit_pending();
    return o;
  }
  // a registration queues behind earlier ones still waiting for memory
  bool behind;
  {
    std::lock_guard<std::mutex> q(srv.qmu);
    behind = !srv.pending.empty();
  }
  bool later = true;
  o.rc = behind ? DSM_ERR_OOM : admit(r.plan, &o.qid, &later);
  if (behind) later = query_footprint(r.plan) + (bytes_in_use - std::min(bytes_in_use, query_bytes_allocated())) <=
                      budget;
  if (o.rc == DSM_ERR_OOM && later) {
    std::lock_guard<std::mutex> q(srv.qmu);
    srv.pending.push_back(std::move(r));
    o.rc = -1;  // no outcome yet
    return o;
  }
  if (o.rc) o.msg = behind ? "query admission: footprint exceeds the budget" : error_text();
  return o;
}

// The worker overlaps host and device work: while the device runs batch
// k + 1 (its union insert, filters and matcher), the host assembles batch
// k's results (copies, canonical sort) and hands them out.  A device batch's
// host preparation (key sorting) happens as the previous batch's deletions
// finish.  Control requests wait until the batch in flight is assembled.
struct InFlight {
  bool live = false;
  std::vector<Request> reqs;
  std::vector<dsm_update> all;
  std::vector<uint32_t> start;
  Staged S;
  std::chrono::steady_clock::time_point t0;
};

void Engine::worker_loop() {
  cudaSetDevice(device);
  InFlight cur, prev;
  int slot = 0;
  std::unique_lock<std::mutex> q(srv.qmu);
  for (;;) {
    if (prev.live && srv.queue.empty()) {  // nothing to overlap with: hand the last batch out
      q.unlock();
      post_batch(prev);
      q.lock();
      continue;
    }
    srv.work_cv.wait(q, [&] { return !srv.queue.empty() || srv.stopping; });
    if (srv.queue.empty()) break;  // stopping, and everything queued was served
    if (srv.queue.front().kind != kReqBatch) {
      Request r = std::move(srv.queue.front());
      srv.queue.pop_front();
      q.unlock();
      if (prev.live) post_batch(prev);
      Outcome o = handle_control(r);
      q.lock();
      if (o.rc != -1) post_outcome(r.id, o);
      srv.done_cv.notify_all();
      continue;
    }
    cur = InFlight();
    size_t total = 0;
    while (!srv.queue.empty() && srv.queue.front().kind == kReqBatch &&
           (cur.reqs.empty() || total + srv.queue.front().ups.size() <= srv.max_merge)) {
      total += srv.queue.front().ups.size();
      cur.reqs.push_back(std::move(srv.queue.front()));
      srv.queue.pop_front();
    }
    q.unlock();
    cur.start.assign(cur.reqs.size() + 1, 0);
    for (size_t k = 0; k < cur.reqs.size(); ++k) {
      cur.all.insert(cur.all.end(), cur.reqs[k].ups.begin(), cur.reqs[k].ups.end());
      cur.start[k + 1] = (uint32_t)cur.all.size();
    }
    cur.live = true;
    slot ^= 1;
    int rc;
    {
      std::lock_guard<std::mutex> lk(mu);
      cur.t0 = std::chrono::steady_clock::now();
      cudaSetDevice(device);
      rc = prepare(cur.all.data(), (uint32_t)cur.all.size(), cur.S, slot);
      if (!rc) rc = launch_front(cur.S);
    }
    if (prev.live) post_batch(prev);  // host work of batch k while the device runs batch k + 1
    if (!rc) {
      std::lock_guard<std::mutex> lk(mu);
      rc = finish_or_retry(cur.S);
    }
    if (rc) {
      fail_batch(cur, rc);
    } else {
      prev = std::move(cur);
    }
    q.lock();
    srv.done_cv.notify_all();
  }
  q.unlock();
  if (prev.live) post_batch(prev);
}

void Engine::fail_batch(InFlight &b, int rc) {
  const std::string msg = error_text();
  std::lock_guard<std::mutex> q(srv.qmu);
  for (Request &r : b.reqs) {
    srv.failed[r.id] = Outcome{rc, 0, msg};
    srv.inflight.erase(r.id);
  }
  b.live = false;
  srv.done_cv.notify_all();
}

// Assembles an in-flight device batch and gives each request its own result
// (its updates' slice of every per-(query, update) array).
void Engine::post_batch(InFlight &b) {
  BatchResult R;
  const int rc = assemble(b.S, R);
  if (rc) {
    fail_batch(b, rc);
    return;
  }
  const uint32_t N = (uint32_t)b.all.size();
  const uint32_t nql = (uint32_t)R.qids.size();
  std::vector<std::unique_ptr<BatchResult>> outs(b.reqs.size());
  if (b.reqs.size() == 1) {  // one request: its result is the batch's, moved
    auto o = std::make_unique<BatchResult>(std::move(R));
    o->id = b.reqs[0].id;
    o->merged_requests = 1;
    o->merged_updates = N;
    outs[0] = std::move(o);
  }
  // merged requests: each request's slice of every per-(query, update) array,
  // the requests on host threads
  parallel_chunks(b.reqs.size() == 1 ? 0 : b.reqs.size(), [&](size_t k) {
    const uint32_t s = b.start[k], n = b.start[k + 1] - s;
    auto o = std::make_unique<BatchResult>();
    o->id = b.reqs[k].id;
    o->n = n;
    o->qids = R.qids;
    o->widths = R.widths;
    o->qlisted = R.qlisted;
    o->listed = R.listed;
    o->signs.assign(R.signs.begin() + s, R.signs.begin() + s + n);
    o->counts.resize((size_t)nql * n);
    o->offsets.assign((size_t)nql * n + 1, 0);
    for (uint32_t ql = 0; ql < nql; ++ql)
      for (uint32_t i = 0; i < n; ++i) {
        const size_t src = (size_t)ql * N + s + i, dst = (size_t)ql * n + i;
        o->counts[dst] = R.counts[src];
        o->offsets[dst + 1] = o->offsets[dst] + (R.offsets[src + 1] - R.offsets[src]);
      }
    if (R.listed) {
      o->tuples.resize(o->offsets.back());
      for (uint32_t ql = 0; ql < nql; ++ql) {  // each query's slice is contiguous
        const size_t a = R.offsets[(size_t)ql * N + s], e = R.offsets[(size_t)ql * N + s + n];
        std::copy(R.tuples.begin() + a, R.tuples.begin() + e, o->tuples.begin() + o->offsets[(size_t)ql * n]);
      }
    }
    o->device_ms = R.device_ms;
    o->match_ms = R.match_ms;
    o->merged_requests = (uint32_t)b.reqs.size();
    o->merged_updates = N;
    outs[k] = std::move(o);
  });
  const auto t1 = std::chrono::steady_clock::now();
  {
    std::lock_guard<std::mutex> r(rmu);
    for (size_t k = 0; k < b.reqs.size(); ++k) {
      outs[k]->queue_ms = ms_between(b.reqs[k].t_submit, b.t0);
      outs[k]->service_ms = ms_between(b.t0, t1);
      outs[k]->total_ms = ms_between(b.reqs[k].t_submit, t1);
      results[b.reqs[k].id] = std::move(outs[k]);
    }
  }
  std::lock_guard<std::mutex> q(srv.qmu);
  for (Request &r : b.reqs) srv.inflight.erase(r.id);
  b.live = false;
  srv.done_cv.notify_all();
}

}  // namespace dsm
