// Engine object and the C ABI (include/dsm.h).
//
// One engine owns one CUDA stream on one device.  A batch runs as
//   upload -> edge state -> union insert -> seeds -> matcher
//   -> (regrow + rerun on result overflow) -> delete -> clear marks -> download
// with the data graph, query descriptors and scratch resident in HBM.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include <thread>
#include <atomic>

#include "../../../include/dsm.h"
#include "../host/dsm_host.h"
#include "../host/par.h"
#include "../host/query_plan.h"
#include "engine_internal.h"
#include "filter.cuh"
#include "kernels.cuh"

namespace dsm {

const char *status_string(int s) {
  switch (s) {
    case DSM_OK: return "ok";
    case DSM_ERR_PARSE: return "parse error";
    case DSM_ERR_OOM: return "out of device memory budget";
    case DSM_ERR_OVERFLOW: return "capacity overflow";
    case DSM_ERR_TIMEOUT: return "bounded device wait timed out";
    case DSM_ERR_LIMIT: return "input beyond supported limits";
    case DSM_ERR_ARG: return "bad argument";
    case DSM_ERR_CUDA: return "CUDA error";
    case DSM_ERR_STATE: return "invalid state";
    case DSM_ERR_NOT_FOUND: return "not found";
  }
  return "unknown status";
}

int Engine::fail(int code, const std::string &msg) {
  set_error(msg);
  return code;
}

int Engine::cuda_fail(cudaError_t e, const char *where) {
  set_error(std::string(where) + ": " + cudaGetErrorString(e));
  return DSM_ERR_CUDA;
}

#define CK(call)                                    \
  do {                                              \
    cudaError_t _e = (call);                        \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

int Engine::dalloc(DevBuf &b, size_t bytes) {
  if (b.bytes >= bytes && b.ptr) return DSM_OK;
  size_t grow = std::max(bytes, b.bytes + b.bytes / 2);
  grow = (grow + 255) & ~(size_t)255;
  if (bytes_in_use - b.bytes + grow > budget) {
    grow = bytes;
    if (bytes_in_use - b.bytes + grow > budget)
      return fail(DSM_ERR_OOM, "device memory budget exhausted (" + std::to_string(bytes) + " bytes requested)");
  }
  if (b.ptr) {
    cudaFree(b.ptr);
    bytes_in_use -= b.bytes;
    b.ptr = nullptr;
    b.bytes = 0;
  }
  cudaError_t e = cudaMalloc(&b.ptr, grow);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(DSM_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  b.bytes = grow;
  bytes_in_use += grow;
  return DSM_OK;
}

void Engine::dfree(DevBuf &b) {
  if (b.ptr) {
    cudaFree(b.ptr);
    bytes_in_use -= b.bytes;
  }
  b.ptr = nullptr;
  b.bytes = 0;
}

int Engine::halloc(HostBuf &b, size_t bytes) {
  if (b.bytes >= bytes && b.ptr) return DSM_OK;
  size_t grow = std::max(bytes, b.bytes + b.bytes / 2);
  if (b.ptr) cudaFreeHost(b.ptr);
  b.ptr = nullptr;
  b.bytes = 0;
  CK(cudaMallocHost(&b.ptr, grow));
  b.bytes = grow;
  return DSM_OK;
}

Engine::~Engine() {
  serve_stop();
  cudaSetDevice(device);
  if (stream) cudaStreamSynchronize(stream);
  for (auto &x : gexec)
    if (x) cudaGraphExecDestroy(x);
  for (DevBuf *b : all_dev_bufs()) dfree(*b);
  for (HostBuf *b : {&h_sched, &h_qlisted})
    if (b->ptr) cudaFreeHost(b->ptr);
  for (HostOut &H : hout) {
    for (HostBuf *b : {&H.stage, &H.hdr, &H.segcnt, &H.vtp, &H.out_seg, &H.out_tup, &H.misc})
      if (b->ptr) cudaFreeHost(b->ptr);
    if (H.ev0) cudaEventDestroy(H.ev0);
    if (H.ev_end) cudaEventDestroy(H.ev_end);
  }
  for (auto &ev : ev_pool)
    if (ev) cudaEventDestroy(ev);
  if (stream) cudaStreamDestroy(stream);
}

std::vector<DevBuf *> Engine::all_dev_bufs() {
  std::vector<DevBuf *> v = {&d_lab, &d_adj, &d_cap, &d_arena, &d_arena_top, &d_loff, &d_qd, &d_orders,
                             &d_pair_off, &d_pair_ent, &d_upd, &d_bkey, &d_bidx, &d_binfo, &d_gflag,
                             &d_vtp, &d_dkey, &d_dhead, &d_dsel, &d_seeds, &d_sched, &d_jobs,
                             &d_job_seq, &d_out_seg, &d_out_tup, &d_segcnt, &d_misc, &d_hdr, &d_qlisted, &d_segwork,
                             &d_rinfo, &d_rmark, &d_rlist, &d_rprev, &d_rows};
  for (auto &q : slots) v.push_back(&q.bitmap);
  for (auto &q : slots) v.push_back(&q.filter_scratch);
  for (auto &q : slots) v.push_back(&q.filter_plan);
  return v;
}

int Engine::init(int dev, size_t mem_budget) {
  device = dev;
  int n = 0;
  CK(cudaGetDeviceCount(&n));
  if (dev < 0 || dev >= n) return fail(DSM_ERR_ARG, "no such CUDA device");
  CK(cudaSetDevice(dev));
  CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, dev));
  num_sms = prop.multiProcessorCount;
  int clk_khz = 0;
  cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, dev);
  clock_khz = clk_khz > 0 ? clk_khz : 1965000;
  size_t freeb = 0, totalb = 0;
  CK(cudaMemGetInfo(&freeb, &totalb));
  budget = mem_budget ? mem_budget : (freeb > (1ull << 30) ? freeb - (1ull << 30) : freeb / 2);
  list_limit_bytes = std::min<uint64_t>(list_limit_bytes, budget / 4);
  ev_pool.resize(8, nullptr);
  for (auto &ev : ev_pool) CK(cudaEventCreate(&ev));
  int per_sm = match_max_blocks_per_sm();
  match_blocks_per_sm = std::max(1, std::min(per_sm, 8));
  // small fixed buffers
  if (int rc = dalloc(d_sched, sizeof(Sched))) return rc;
  if (int rc = dalloc(d_arena_top, 256)) return rc;
  if (int rc = dalloc(d_misc, 256)) return rc;
  if (int rc = dalloc(d_hdr, 256)) return rc;
  if (int rc = halloc(h_sched, sizeof(Sched) + 64)) return rc;
  return DSM_OK;
}

// ---------------------------------------------------------------------------
// Graph
// ---------------------------------------------------------------------------
int Engine::load_graph(uint32_t nv_, const uint32_t *labels, std::vector<uint64_t> &keys) {
  std::lock_guard<std::mutex> lk(mu);
  CK(cudaSetDevice(device));
  CK(cudaStreamSynchronize(stream));
  if (nv_ > kMaxVertices) return fail(DSM_ERR_LIMIT, "more than 2^27 vertices");
  uint32_t max_label = 0;
  for (uint32_t v = 0; v < nv_; ++v) {
    if (labels[v] & kTouchBit) return fail(DSM_ERR_LIMIT, "vertex label >= 2^31");
    max_label = std::max(max_label, labels[v]);
  }
  const uint32_t nlt_ = nv_ ? label_slot(max_label) + 1 : 1;
  // canonical, deduplicated undirected edges
  parallel_sort(keys);
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  std::vector<uint32_t> deg(nv_, 0);
  for (uint64_t k : keys) {
    deg[k >> 32]++;
    deg[(uint32_t)k]++;
  }
  // slack: capacity = deg + deg/8 + 4, rounded to 16 bytes
  std::vector<uint32_t> cap(nv_);
  std::vector<uint2> adj(nv_);
  uint64_t off16 = 0;
  for (uint32_t v = 0; v < nv_; ++v) {
    cap[v] = (deg[v] + deg[v] / 8 + 4 + 3) & ~3u;
    adj[v] = make_uint2((uint32_t)off16, 0);
    off16 += cap[v] / 4;
  }
  if (off16 > 0xFFFFFFFFull) return fail(DSM_ERR_LIMIT, "graph too large for 32-bit run offsets");
  uint64_t used_words = off16 * 4;
  uint64_t arena_words = used_words + used_words / 4 + std::min<uint64_t>(used_words, 1u << 20);
  arena_words = (arena_words + 3) & ~3ull;
  // fill runs on the host (pinned) and upload once
  HostBuf stage;
  if (int rc = halloc(stage, used_words * 4)) return rc;
  uint32_t *h_arena = (uint32_t *)stage.ptr;
  // label-major runs: entries sorted by (label slot, id), and each vertex's
  // slot offsets
  std::vector<uint32_t> fill(nv_, 0);
  for (uint64_t k : keys) {
    uint32_t a = (uint32_t)(k >> 32), b = (uint32_t)k;
    h_arena[(uint64_t)adj[a].x * 4 + fill[a]++] = pack_entry(labels[b], b);
    h_arena[(uint64_t)adj[b].x * 4 + fill[b]++] = pack_entry(labels[a], a);
  }
  const size_t stride = nlt_ + 1;
  std::vector<uint32_t> loff((size_t)nv_ * stride);
  parallel_for(nv_, 1u << 14, [&](size_t lo, size_t hi) {
    for (size_t v = lo; v < hi; ++v) {
      uint32_t *run = h_arena + (uint64_t)adj[v].x * 4;
      std::sort(run, run + deg[v]);
      for (uint32_t i = deg[v]; i < cap[v]; ++i) run[i] = 0xFFFFFFFFu;
      adj[v].y = deg[v];
      uint32_t *t = loff.data() + v * stride;
      for (uint32_t sl = 0, i = 0; sl <= nlt_; ++sl) {
        while (i < deg[v] && (run[i] >> kIdBits) < sl) ++i;
        t[sl] = sl == nlt_ ? deg[v] : i;
      }
    }
  });
  int rc;
  if ((rc = dalloc(d_lab, (size_t)nv_ * 4)) || (rc = dalloc(d_adj, (size_t)nv_ * 8)) ||
      (rc = dalloc(d_cap, (size_t)nv_ * 4)) || (rc = dalloc(d_loff, loff.size() * 4)) ||
      (rc = dalloc(d_arena, arena_words * 4))) {
    cudaFreeHost(stage.ptr);
    return rc;
  }
  CK(cudaMemcpyAsync(d_loff.ptr, loff.data(), loff.size() * 4, cudaMemcpyHostToDevice, stream));
  CK(cudaMemcpyAsync(d_lab.ptr, labels, (size_t)nv_ * 4, cudaMemcpyHostToDevice, stream));
  CK(cudaMemcpyAsync(d_adj.ptr, adj.data(), (size_t)nv_ * 8, cudaMemcpyHostToDevice, stream));
  CK(cudaMemcpyAsync(d_cap.ptr, cap.data(), (size_t)nv_ * 4, cudaMemcpyHostToDevice, stream));
  CK(cudaMemcpyAsync(d_arena.ptr, h_arena, used_words * 4, cudaMemcpyHostToDevice, stream));
  unsigned long long top = off16;
  CK(cudaMemcpyAsync(d_arena_top.ptr, &top, 8, cudaMemcpyHostToDevice, stream));
  CK(cudaStreamSynchronize(stream));
  cudaFreeHost(stage.ptr);
  nv = nv_;
  nlt = nlt_;
  this->arena_words = arena_words;
  arena_used16 = off16;
  graph_entries = 2 * keys.size();
  graph_loaded = true;
  label_host.assign(labels, labels + nv_);
  for (auto &q : slots) q.filter_dirty = true;
  return region_init();
}

// The incremental filter's region buffers for a new graph: marks cleared,
// nothing kept from a previous batch, the next filtered batch recomputes
// every query in full.  List capacity: a quarter of the vertices (at least
// 2^16); beyond it a region run costs about as much as a full one.
int Engine::region_init() {
  const uint32_t cap = std::max<uint32_t>(nv / 4, std::min<uint32_t>(nv, 1u << 16));
  const uint32_t prev_cap = 1u << 18;
  int rc;
  if ((rc = dalloc(d_rinfo, sizeof(RegionInfo))) || (rc = dalloc(d_rmark, (size_t)std::max<uint32_t>(nv, 1) * 4)) ||
      (rc = dalloc(d_rlist, (size_t)std::max<uint32_t>(cap, 1) * 4)) || (rc = dalloc(d_rprev, (size_t)prev_cap * 4)))
    return rc;
  RegionInfo I;
  std::memset(&I, 0, sizeof(I));
  I.stale = 1;
  I.cap = cap;
  I.prev_cap = prev_cap;
  I.ov_round = 64;
  CK(cudaMemsetAsync(d_rmark.ptr, 0, (size_t)std::max<uint32_t>(nv, 1) * 4, stream));
  CK(cudaMemcpyAsync(d_rinfo.ptr, &I, sizeof(I), cudaMemcpyHostToDevice, stream));
  CK(cudaStreamSynchronize(stream));  // `I` is stack memory
  region_batches = 0;
  return DSM_OK;
}

RegionDevice Engine::region_dev() {
  RegionDevice r;
  r.info = (RegionInfo *)d_rinfo.ptr;
  r.mark = (uint32_t *)d_rmark.ptr;
  r.list = (uint32_t *)d_rlist.ptr;
  r.prev = (uint32_t *)d_rprev.ptr;
  return r;
}

DevGraph Engine::dev_graph() {
  DevGraph g;
  g.nv = nv;
  g.lab = (uint32_t *)d_lab.ptr;
  g.adj = (uint2 *)d_adj.ptr;
  g.cap = (uint32_t *)d_cap.ptr;
  g.arena = (uint32_t *)d_arena.ptr;
  g.loff = (uint32_t *)d_loff.ptr;
  g.nlt = nlt;
  g.arena_words = arena_words;
  g.arena_top = (unsigned long long *)d_arena_top.ptr;
  return g;
}

int Engine::export_graph(uint32_t *offsets, uint32_t *nbrs, uint64_t *num_entries) {
  std::lock_guard<std::mutex> lk(mu);
  return export_graph_locked(offsets, nbrs, num_entries);
}

int Engine::export_graph_locked(uint32_t *offsets, uint32_t *nbrs, uint64_t *num_entries) {
  if (!graph_loaded) return fail(DSM_ERR_STATE, "no graph loaded");
  CK(cudaSetDevice(device));
  CK(cudaStreamSynchronize(stream));
  std::vector<uint2> adj(nv);
  CK(cudaMemcpy(adj.data(), d_adj.ptr, (size_t)nv * 8, cudaMemcpyDeviceToHost));
  uint64_t total = 0;
  for (uint32_t v = 0; v < nv; ++v) total += adj[v].y;
  if (num_entries) *num_entries = total;
  if (offsets) {
    uint64_t k = 0;
    for (uint32_t v = 0; v < nv; ++v) {
      offsets[v] = (uint32_t)k;
      k += adj[v].y;
    }
    offsets[nv] = (uint32_t)k;
  }
  if (nbrs) {
    // one copy of the arena's used part, then per run: ids, ascending
    unsigned long long top16 = 0;
    CK(cudaMemcpy(&top16, d_arena_top.ptr, 8, cudaMemcpyDeviceToHost));
    std::vector<uint32_t> arena(top16 * 4);
    if (!arena.empty())
      CK(cudaMemcpy(arena.data(), d_arena.ptr, arena.size() * 4, cudaMemcpyDeviceToHost));
    uint64_t k = 0;
    for (uint32_t v = 0; v < nv; ++v) {
      const uint32_t *run = arena.data() + (uint64_t)adj[v].x * 4;
      for (uint32_t i = 0; i < adj[v].y; ++i) nbrs[k + i] = run[i] & kIdMask;
      std::sort(nbrs + k, nbrs + k + adj[v].y);
      k += adj[v].y;
    }
  }
  return DSM_OK;
}

// ---------------------------------------------------------------------------
// Queries
// ---------------------------------------------------------------------------
// Device bytes a query is charged at admission: its descriptor and orders,
// and (for the candidate filter) bitmaps, LDF/NLF masks and encodings.
size_t Engine::query_footprint(const QueryPlan &p) const {
  size_t foot = sizeof(QDev) + p.orders.size() * sizeof(OrderRec);
  if (graph_loaded)
    foot += (size_t)p.nq * ((nv + 31) / 32) * 4 + (size_t)nv * (8 + 4 * std::max<uint32_t>(p.enc_words, 1));
  return foot;
}

size_t Engine::query_bytes_allocated() const {
  size_t b = 0;
  for (const Slot &q : slots) b += q.bitmap.bytes + q.filter_scratch.bytes + q.filter_plan.bytes;
  return b;
}

// Admission against the budget: engine bytes not owned by queries + the
// footprints of the admitted queries + this one.  *fits_later: it would fit
// once every other query retired.
int Engine::admit(QueryPlan &plan, uint32_t *qid, bool *fits_later, int64_t want_id) {
  const size_t foot = query_footprint(plan);
  const size_t base = bytes_in_use - std::min(bytes_in_use, query_bytes_allocated());
  size_t charged = 0;
  for (const Slot &q : slots)
    if (q.live) charged += q.foot;
  if (fits_later) *fits_later = base + foot <= budget;
  if (base + charged + foot > budget)
    return fail(DSM_ERR_OOM, "query admission: footprint " + std::to_string(foot) + " bytes exceeds the budget");
  uint32_t id = (uint32_t)slots.size();
  if (want_id >= 0) {  // a resumed query keeps its id
    id = (uint32_t)want_id;
    if (id < slots.size() && slots[id].live) return fail(DSM_ERR_STATE, "query id already in use");
  } else {
    for (uint32_t i = 0; i < slots.size(); ++i)
      if (!slots[i].live) {
        id = i;
        break;
      }
  }
  if (id >= (1u << 23)) return fail(DSM_ERR_LIMIT, "too many queries");
  if (id >= slots.size()) slots.resize(id + 1);
  Slot &s = slots[id];
  s.live = true;
  s.plan = std::move(plan);
  s.filter_dirty = true;
  s.foot = foot;
  queries_dirty = true;
  *qid = id;
  return DSM_OK;
}

int Engine::register_query(const uint32_t *qoff, const uint32_t *qnbr, const uint32_t *qlab, uint32_t nq,
                           uint32_t *qid) {
  bool serving;
  {
    std::lock_guard<std::mutex> q(srv.qmu);
    serving = srv.running;
  }
  if (serving) {  // through the queue, in order with the batches
    uint64_t ticket = 0;
    if (int rc = register_async(qoff, qnbr, qlab, nq, &ticket)) return rc;
    return admission(ticket, -1, qid);
  }
  std::lock_guard<std::mutex> lk(mu);
  QueryPlan plan;
  std::string err;
  if (int rc = plan_query(nq, qoff, qnbr, qlab, plan, err)) return fail(rc, err);
  return admit(plan, qid, nullptr);
}

int Engine::retire_query(uint32_t qid) {
  bool serving;
  {
    std::lock_guard<std::mutex> q(srv.qmu);
    serving = srv.running;
  }
  if (serving) {
    uint64_t ticket = 0;
    if (int rc = retire_async(qid, &ticket)) return rc;
    uint32_t dummy = 0;
    return admission(ticket, -1, &dummy);
  }
  std::lock_guard<std::mutex> lk(mu);
  return retire_locked(qid);
}

int Engine::retire_locked(uint32_t qid) {
  if (qid >= slots.size() || !slots[qid].live) return fail(DSM_ERR_NOT_FOUND, "no such query");
  Slot &s = slots[qid];
  s.live = false;
  dfree(s.bitmap);
  dfree(s.filter_scratch);
  dfree(s.filter_plan);
  s.plan = QueryPlan();
  s.foot = 0;
  queries_dirty = true;
  return DSM_OK;
}

int Engine::sync_queries() {
  if (!queries_dirty) return DSM_OK;
  std::vector<QDev> qd(std::max<size_t>(slots.size(), 1));
  std::vector<OrderRec> orders;
  std::vector<std::vector<uint32_t>> buckets(32 * 32);
  live_ids.clear();
  max_width = 0;
  for (uint32_t id = 0; id < slots.size(); ++id) {
    Slot &s = slots[id];
    if (!s.live) continue;
    QDev &d = qd[id];
    std::memset(&d, 0, sizeof(d));
    d.nq = s.plan.nq;
    d.order_base = (uint32_t)orders.size();
    d.n_orders = (uint32_t)s.plan.orders.size();
    d.local = (uint32_t)live_ids.size();
    for (uint32_t u = 0; u < s.plan.nq; ++u) d.label[u] = s.plan.labels[u];
    d.bitmap = nullptr;
    d.col_len = (nv + 31) / 32;
    for (size_t o = 0; o < s.plan.orders.size(); ++o) {
      OrderRec r;
      std::memcpy(&r, &s.plan.orders[o], sizeof(r));
      orders.push_back(r);
      uint32_t u = s.plan.oedges[o].first, v = s.plan.oedges[o].second;
      buckets[s.plan.labels[u] * 32 + s.plan.labels[v]].push_back((id << 8) | (uint32_t)o);
    }
    live_ids.push_back(id);
    max_width = std::max(max_width, s.plan.nq);
  }
  std::vector<uint32_t> pair_off(32 * 32 + 1, 0), pair_ent;
  max_bucket = 0;
  for (size_t b = 0; b < buckets.size(); ++b) {
    pair_off[b + 1] = pair_off[b] + (uint32_t)buckets[b].size();
    pair_ent.insert(pair_ent.end(), buckets[b].begin(), buckets[b].end());
    max_bucket = std::max<uint32_t>(max_bucket, (uint32_t)buckets[b].size());
  }
  if (pair_ent.empty()) pair_ent.push_back(0);
  if (orders.empty()) orders.emplace_back();
  int rc;
  if ((rc = dalloc(d_qd, qd.size() * sizeof(QDev))) || (rc = dalloc(d_orders, orders.size() * sizeof(OrderRec))) ||
      (rc = dalloc(d_pair_off, pair_off.size() * 4)) || (rc = dalloc(d_pair_ent, pair_ent.size() * 4)))
    return rc;
  qd_host = qd;
  CK(cudaMemcpyAsync(d_orders.ptr, orders.data(), orders.size() * sizeof(OrderRec), cudaMemcpyHostToDevice, stream));
  CK(cudaMemcpyAsync(d_pair_off.ptr, pair_off.data(), pair_off.size() * 4, cudaMemcpyHostToDevice, stream));
  CK(cudaMemcpyAsync(d_pair_ent.ptr, pair_ent.data(), pair_ent.size() * 4, cudaMemcpyHostToDevice, stream));
  CK(cudaStreamSynchronize(stream));
  queries_dirty = false;
  qd_dirty = true;
  ++query_gen;
  return DSM_OK;
}

int Engine::upload_qd() {
  CK(cudaMemcpyAsync(d_qd.ptr, qd_host.data(), qd_host.size() * sizeof(QDev), cudaMemcpyHostToDevice, stream));
  qd_dirty = false;
  return DSM_OK;
}

// ---------------------------------------------------------------------------
// Batches
// ---------------------------------------------------------------------------

// Canonical order of the listed tuples: each (query, update) segment sorted
// lexicographically, segments shared among host threads (largest first) when
// the batch listed enough tuples to pay for the threads.
void Engine::sort_segments(BatchResult &R, const std::vector<uint64_t> &counts, uint32_t nq_live, uint32_t n,
                           size_t total) {
  std::vector<uint32_t> segs;
  for (size_t s = 0; s < (size_t)nq_live * n; ++s)
    if (counts[s] >= 2) segs.push_back((uint32_t)s);
  std::sort(segs.begin(), segs.end(), [&](uint32_t a, uint32_t b) { return counts[a] > counts[b]; });
  std::atomic<size_t> next{0};
  auto work = [&]() {
    std::vector<uint32_t> idx, tmp;
    for (size_t k; (k = next.fetch_add(1)) < segs.size();) {
      const size_t s = segs[k], c = counts[s];
      const uint32_t w = R.widths[s / n];
      uint32_t *base = &R.tuples[R.offsets[s]];
      idx.resize(c);
      for (size_t i = 0; i < c; ++i) idx[i] = (uint32_t)i;
      std::sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) {
        return std::lexicographical_compare(base + (size_t)x * w, base + (size_t)x * w + w, base + (size_t)y * w,
                                            base + (size_t)y * w + w);
      });
      tmp.resize(c * w);
      for (size_t i = 0; i < c; ++i) std::memcpy(&tmp[i * w], base + (size_t)idx[i] * w, w * 4);
      std::memcpy(base, tmp.data(), tmp.size() * 4);
    }
  };
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned nt = total < (1u << 16) ? 1u : std::min<unsigned>(std::min(hw, 32u), (unsigned)segs.size());
  std::vector<std::thread> th;
  for (unsigned t = 1; t < nt; ++t) th.emplace_back(work);
  work();
  for (auto &t : th) t.join();
}
int Engine::check_updates(const dsm_update *ups, uint32_t n) {
  if (!graph_loaded) return fail(DSM_ERR_STATE, "no graph loaded");
  if (n >= (1u << 30)) return fail(DSM_ERR_LIMIT, "batch larger than 2^30 updates");
  for (uint32_t i = 0; i < n; ++i)
    if (ups[i].src >= nv || ups[i].dst >= nv) return fail(DSM_ERR_ARG, "update names a vertex >= num_v");
  return DSM_OK;
}

int Engine::submit(const dsm_update *ups, uint32_t n, uint64_t *batch_id) {
  {
    std::unique_lock<std::mutex> q(srv.qmu);
    if (srv.running) {
      if (srv.stopping) return fail(DSM_ERR_STATE, "the serving loop is stopping");
      q.unlock();
      {
        std::lock_guard<std::mutex> lk(mu);
        if (int rc = check_updates(ups, n)) return rc;
      }
      Request r;
      r.kind = kReqBatch;
      r.ups.assign(ups, ups + n);
      r.t_submit = std::chrono::steady_clock::now();
      q.lock();
      r.id = next_batch_id++;
      *batch_id = r.id;
      srv.inflight.insert(r.id);
      srv.queue.push_back(std::move(r));
      srv.work_cv.notify_one();
      return DSM_OK;
    }
  }
  std::lock_guard<std::mutex> lk(mu);
  if (int rc = check_updates(ups, n)) return rc;
  CK(cudaSetDevice(device));
  const auto t0 = std::chrono::steady_clock::now();
  auto res = std::make_unique<BatchResult>();
  int rc = run_batch(ups, n, *res);
  if (rc) return rc;
  const uint64_t id = next_batch_id++;
  res->id = id;
  res->service_ms = res->total_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  res->merged_updates = n;
  {
    std::lock_guard<std::mutex> r(rmu);
    results[id] = std::move(res);
  }
  *batch_id = id;
  return DSM_OK;
}

int Engine::graph_apply(const dsm_update *ups, uint32_t n) {
  {
    std::lock_guard<std::mutex> q(srv.qmu);
    if (srv.running) return fail(DSM_ERR_STATE, "graph apply while the serving loop runs");
  }
  std::lock_guard<std::mutex> lk(mu);
  if (int rc = check_updates(ups, n)) return rc;
  CK(cudaSetDevice(device));
  BatchResult R;
  return run_batch(ups, n, R, false);
}

// Blocks until batch `id` is done; its status.  A failure is reported once,
// then forgotten (a later call finds no such batch).
int Engine::wait_batch(uint64_t id) {
  std::unique_lock<std::mutex> q(srv.qmu);
  if (id == 0 || id >= next_batch_id) return fail(DSM_ERR_NOT_FOUND, "no such batch");
  srv.done_cv.wait(q, [&] { return srv.inflight.count(id) == 0; });
  auto f = srv.failed.find(id);
  if (f != srv.failed.end()) {
    const Outcome o = f->second;
    srv.failed.erase(f);
    set_error(o.msg);
    return o.rc;
  }
  q.unlock();
  std::lock_guard<std::mutex> r(rmu);  // done: its results, unless released (or it failed and was reported)
  if (results.find(id) == results.end()) return fail(DSM_ERR_NOT_FOUND, "no such batch");
  return DSM_OK;
}

int Engine::timing(uint64_t id, dsm_batch_timing *t) {
  if (int rc = wait_batch(id)) return rc;
  std::lock_guard<std::mutex> lk(rmu);
  auto it = results.find(id);
  if (it == results.end()) return fail(DSM_ERR_NOT_FOUND, "no such batch (released?)");
  const BatchResult &R = *it->second;
  t->queue_ms = R.queue_ms;
  t->service_ms = R.service_ms;
  t->total_ms = R.total_ms;
  t->device_ms = R.device_ms;
  t->merged_requests = R.merged_requests;
  t->merged_updates = R.merged_updates;
  return DSM_OK;
}

// Uploads the filter's descriptor and op list of query `id` and sizes its
// per-vertex buffers (once per registration / graph load).
int Engine::prepare_filter(uint32_t id) {
  Slot &s = slots[id];
  if (!s.filter_dirty && s.filter_scratch.ptr && s.bitmap.ptr) return DSM_OK;
  const QueryPlan &p = s.plan;
  QFilterDesc desc;
  std::memset(&desc, 0, sizeof(desc));
  desc.nq = p.nq;
  desc.nlabels = p.nlabels;
  for (uint32_t u = 0; u < p.nq; ++u) {
    desc.label_us[p.labels[u]] |= 1u << u;
    desc.qdeg[u] = p.degree[u];
    desc.pos_of_u[u] = p.enc_pos_of_u[u];
    for (uint32_t l = 0; l < 32; ++l) desc.nlc[u][l] = (uint8_t)std::min<uint32_t>(p.nlc[(size_t)u * 32 + l], 255);
  }
  // incremental region: LDF+NLF alone reads one hop (the vertex's own
  // adjacency), each op one more
  uint32_t hops = filter_mode >= 2 ? (uint32_t)p.ops.size() : 0u;
  desc.fepoch = 0xFFFFFFFFu;  // never computed: the first run is full
  desc.full_now = 1;
  std::vector<DevFilterOp> ops(p.ops.size());
  for (size_t k = 0; k < p.ops.size(); ++k) {
    const FilterOp &o = p.ops[k];
    DevFilterOp &d = ops[k];
    std::memset(&d, 0, sizeof(d));
    d.kind = o.kind;
    d.core_u = o.core_u;
    d.pos = o.pos;
    d.nleaf = o.nleaf;
    for (int i = 0; i < 16; ++i) d.leaf_u[i] = o.leaf_u[i];
    d.lp = o.left_pos;
    d.rp = o.right_pos;
    d.lcp = o.left_core_pos;
    d.rcp = o.right_core_pos;
    d.comb_type = o.comb_type;
    d.nsmall = o.nsmall;
    for (int i = 0; i < 32; ++i) d.small_core_pos[i] = o.small_core_pos[i];
    for (int i = 0; i < 16; ++i) {
      d.leaf_src_count[i] = o.leaf_src_count[i];
      for (int j = 0; j < 32; ++j) d.leaf_src[i][j] = (uint16_t)o.leaf_src[i][j];
    }
    // the merges and combines before it with the same core (validity replay)
    for (size_t j = 0; j < k; ++j)
      if (p.ops[j].core_u == o.core_u && p.ops[j].kind != FilterOp::kEncode) {
        if (d.nprior == 15) {
          hops = kRegionMaxHops + 1;  // too long a history: always full
          break;
        }
        d.prior[d.nprior++] = (uint32_t)j;
      }
  }
  desc.hops = std::min<uint32_t>(hops, kRegionMaxHops + 1);
  s.filter_hops = desc.hops;
  const size_t plan_bytes = sizeof(QFilterDesc) + ops.size() * sizeof(DevFilterOp);
  const uint32_t col_len = (nv + 31) / 32;
  const size_t words = std::max<uint32_t>(p.enc_words, 1);
  int rc;
  if ((rc = dalloc(s.filter_plan, plan_bytes)) || (rc = dalloc(s.filter_scratch, (size_t)nv * (8 + 4 * words))) ||
      (rc = dalloc(s.bitmap, (size_t)p.nq * col_len * 4)))
    return rc;
  CK(cudaMemcpyAsync(s.filter_plan.ptr, &desc, sizeof(desc), cudaMemcpyHostToDevice, stream));
  if (!ops.empty())
    CK(cudaMemcpyAsync((char *)s.filter_plan.ptr + sizeof(QFilterDesc), ops.data(), ops.size() * sizeof(DevFilterOp),
                       cudaMemcpyHostToDevice, stream));
  CK(cudaStreamSynchronize(stream));  // `desc` and `ops` are stack / vector memory
  s.filter_nops = (uint32_t)ops.size();
  s.filter_dirty = false;
  ++query_gen;
  return DSM_OK;
}

int Engine::launch_filter(uint32_t id, int mode, int force_full) {
  Slot &s = slots[id];
  FilterDevice f;
  f.desc = (const QFilterDesc *)s.filter_plan.ptr;
  f.ops = (const DevFilterOp *)((const char *)s.filter_plan.ptr + sizeof(QFilterDesc));
  f.nops = s.filter_nops;
  f.vcand = (uint32_t *)s.filter_scratch.ptr;
  f.valid = f.vcand + nv;
  f.enc = f.valid + nv;
  f.words = std::max<uint32_t>(s.plan.enc_words, 1);
  f.col_len = (nv + 31) / 32;
  f.bitmap = (uint32_t *)s.bitmap.ptr;
  launch_query_filter(dev_graph(), f, mode, num_sms, stream, region_dev(), force_full || !filter_incremental);
  stats.kernel_launches += 2 + (mode >= 2 ? 3 * f.nops : 0);
  return DSM_OK;
}

// Candidate filters of every live query on the batch's union graph (sound
// for every state the batch passes through); the matcher and the seeds then
// test each candidate against its query vertex's bitmap.  prepare_filters
// (host: buffers, plans, descriptors) runs before the batch's device work;
// launch_filters only enqueues kernels and events.
int Engine::prepare_filters() {
  // the region's vertex marks carry a 26-bit epoch, one per filtered batch:
  // start afresh before it wraps (every query's next run is then full)
  if (filter_mode > 0 && ++region_batches >= (1u << 26) - 4) {
    if (int rc = region_init()) return rc;
    region_batches = 0;
  }
  bool changed = false;
  for (uint32_t id : live_ids) {
    QDev &q = qd_host[id];
    const uint32_t *want = nullptr;
    if (filter_mode > 0) {
      if (int rc = prepare_filter(id)) return rc;
      want = (const uint32_t *)slots[id].bitmap.ptr;
    }
    if (q.bitmap != want) {
      q.bitmap = want;
      changed = true;
    }
  }
  if (changed)
    if (int rc = upload_qd()) return rc;
  if (changed) CK(cudaStreamSynchronize(stream));  // qd_host is pageable
  return DSM_OK;
}

int Engine::launch_filters() {
  if (filter_mode == 0) return DSM_OK;
  cudaEvent_t f0 = ev_pool[5], f1 = ev_pool[6];
  if (int r = rec(f0)) return r;
  // the batch's region: as many hops as the farthest-reaching live query
  uint32_t hops = 0;
  for (uint32_t id : live_ids) hops = std::max(hops, std::min<uint32_t>(slots[id].filter_hops, kRegionMaxHops));
  const uint32_t *hdr_n = (const uint32_t *)d_hdr.ptr;  // BatchHdr::n
  const bool region = d_rinfo.ptr != nullptr;  // without its buffers every run is full
  if (region) {
    launch_region_build(dev_graph(), region_dev(), hdr_n, (const uint4 *)d_upd.ptr, hops, num_sms, stream);
    stats.kernel_launches += 3 + 2 * hops;
  }
  for (uint32_t id : live_ids)
    if (int rc = launch_filter(id, filter_mode, 0)) return rc;
  if (region) {
    launch_region_save(region_dev(), hdr_n, (const uint4 *)d_upd.ptr, stream);
    ++stats.kernel_launches;
  }
  if (int r = rec(f1)) return r;
  filter_timed = true;
  return DSM_OK;
}

// Records an event on the engine stream; while a segment is being captured
// the record becomes a node of the graph (a plain record would only mark a
// capture dependency and never time anything).
int Engine::rec(cudaEvent_t ev) {
  CK(cudaEventRecordWithFlags(ev, stream, capturing ? cudaEventRecordExternal : cudaEventRecordDefault));
  return DSM_OK;
}

void Engine::elapsed(cudaEvent_t a, cudaEvent_t b, float *ms) {
  if (cudaEventElapsedTime(ms, a, b) != cudaSuccess) {
    cudaGetLastError();  // not recorded (e.g. no matcher launch): no time
    *ms = 0;
  }
}

int Engine::query_filter(uint32_t qid, uint32_t *bitmaps, uint32_t *v_cand_us) {
  std::lock_guard<std::mutex> lk(mu);
  if (!graph_loaded) return fail(DSM_ERR_STATE, "no graph loaded");
  if (qid >= slots.size() || !slots[qid].live) return fail(DSM_ERR_NOT_FOUND, "no such query");
  CK(cudaSetDevice(device));
  if (int rc = prepare_filter(qid)) return rc;
  if (int rc = launch_filter(qid, 2, 1)) return rc;
  CK(cudaGetLastError());
  const Slot &s = slots[qid];
  if (bitmaps)
    CK(cudaMemcpyAsync(bitmaps, s.bitmap.ptr, (size_t)s.plan.nq * ((nv + 31) / 32) * 4, cudaMemcpyDeviceToHost,
                       stream));
  if (v_cand_us) CK(cudaMemcpyAsync(v_cand_us, s.filter_scratch.ptr, (size_t)nv * 4, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  return DSM_OK;
}

// The query's resident filter state, as its last run left it: bitmaps,
// LDF+NLF masks, and info[0] = 1 if that run recomputed every vertex,
// info[1] = vertices it recomputed.
int Engine::filter_state(uint32_t qid, uint32_t *bitmaps, uint32_t *v_cand_us, uint32_t *info) {
  std::lock_guard<std::mutex> lk(mu);
  if (!graph_loaded) return fail(DSM_ERR_STATE, "no graph loaded");
  if (qid >= slots.size() || !slots[qid].live) return fail(DSM_ERR_NOT_FOUND, "no such query");
  const Slot &s = slots[qid];
  if (!s.bitmap.ptr || !s.filter_plan.ptr) return fail(DSM_ERR_STATE, "the query's filter has not run");
  CK(cudaSetDevice(device));
  if (bitmaps)
    CK(cudaMemcpyAsync(bitmaps, s.bitmap.ptr, (size_t)s.plan.nq * ((nv + 31) / 32) * 4, cudaMemcpyDeviceToHost,
                       stream));
  if (v_cand_us) CK(cudaMemcpyAsync(v_cand_us, s.filter_scratch.ptr, (size_t)nv * 4, cudaMemcpyDeviceToHost, stream));
  QFilterDesc desc;
  RegionInfo I;
  std::memset(&I, 0, sizeof(I));
  CK(cudaMemcpyAsync(&desc, s.filter_plan.ptr, sizeof(desc), cudaMemcpyDeviceToHost, stream));
  if (d_rinfo.ptr) CK(cudaMemcpyAsync(&I, d_rinfo.ptr, sizeof(I), cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  if (info) {
    info[0] = desc.full_now;
    info[1] = desc.full_now ? nv : I.bound[std::min<uint32_t>(desc.hops, 63)];
  }
  return DSM_OK;
}

int Engine::view(uint64_t id, dsm_result_view *v) {
  if (int rc = wait_batch(id)) return rc;
  std::lock_guard<std::mutex> lk(rmu);
  auto it = results.find(id);
  if (it == results.end()) return fail(DSM_ERR_NOT_FOUND, "no such batch (released?)");
  BatchResult &R = *it->second;
  v->batch_id = id;
  v->num_updates = R.n;
  v->num_queries = (uint32_t)R.qids.size();
  v->qids = R.qids.data();
  v->widths = R.widths.data();
  v->signs = R.signs.data();
  v->counts = R.counts.data();
  v->offsets = R.offsets.data();
  v->tuples = R.tuples.data();
  v->listed = R.listed;
  v->query_listed = R.qlisted.data();
  return DSM_OK;
}

int Engine::release(uint64_t id) {
  std::lock_guard<std::mutex> lk(rmu);
  auto it = results.find(id);
  if (it == results.end()) return fail(DSM_ERR_NOT_FOUND, "no such batch");
  results.erase(it);
  return DSM_OK;
}

}  // namespace dsm
