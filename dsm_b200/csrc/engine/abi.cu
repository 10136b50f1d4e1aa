// extern "C" entry points of include/dsm.h.
#include <cstring>
#include <string>

#include "../../../include/dsm.h"
#include "../host/dsm_host.h"
#include "engine_internal.h"

using dsm::Engine;

struct dsm_engine {
  Engine e;
};
struct dsm_text {
  dsm::TextGraph g;       // parsed text
  dsm::MappedGraph m;     // or a mapped binary file
  dsm::GraphArrays a;     // views of whichever holds the arrays
};
struct dsm_workload {
  dsm::Workload w;
};

#define ENGINE_OR_ARG(e) \
  if (!(e)) return DSM_ERR_ARG

extern "C" {

const char *dsm_status_string(int status) { return dsm::status_string(status); }

int dsm_engine_create(int device, size_t mem_budget, dsm_engine **out) {
  if (!out) return DSM_ERR_ARG;
  *out = nullptr;
  auto *h = new dsm_engine();
  int rc = h->e.init(device, mem_budget);
  if (rc) {
    delete h;
    return rc;
  }
  *out = h;
  return DSM_OK;
}

int dsm_engine_destroy(dsm_engine *e) {
  ENGINE_OR_ARG(e);
  delete e;
  return DSM_OK;
}

const char *dsm_last_error(dsm_engine *e) {
  static thread_local std::string text;  // valid until this thread's next call
  text = e ? e->e.error_text() : "null engine";
  return text.c_str();
}

int dsm_engine_set_option(dsm_engine *e, int option, int64_t value) {
  ENGINE_OR_ARG(e);
  Engine &E = e->e;
  std::lock_guard<std::mutex> lk(E.mu);
  switch (option) {
    case DSM_OPT_LIST: E.list_mode = value ? 1 : 0; return DSM_OK;
    case DSM_OPT_FILTER:
      if (value < 0 || value > 2) return E.fail(DSM_ERR_ARG, "filter mode is 0, 1 or 2");
      E.filter_mode = (int)value;
      for (auto &s : E.slots) s.filter_dirty = true;
      E.qd_dirty = true;
      return DSM_OK;
    case DSM_OPT_RESULT_CAP:
      if (value <= 0) return E.fail(DSM_ERR_ARG, "result capacity must be positive");
      E.result_cap = (uint64_t)value;
      return DSM_OK;
    case DSM_OPT_WARPS_PER_SM:
      if (value < 0 || value > 64) return E.fail(DSM_ERR_ARG, "warps per SM in [0, 64]");
      E.warps_per_sm = (int)value;
      return DSM_OK;
    case DSM_OPT_DONATE: E.donate = value ? 1 : 0; return DSM_OK;
    case DSM_OPT_TIMEOUT_MS:
      if (value <= 0) return E.fail(DSM_ERR_ARG, "timeout must be positive");
      E.timeout_ms = value;
      return DSM_OK;
    case DSM_OPT_LABEL_QUIRK:
      if (value) return E.fail(DSM_ERR_LIMIT, "label overwrite on insert is not supported by the device store");
      E.label_quirk = 0;
      return DSM_OK;
    case DSM_OPT_SORT: E.sort_results = value ? 1 : 0; return DSM_OK;
    case DSM_OPT_LIST_LIMIT:
      if (value <= 0) return E.fail(DSM_ERR_ARG, "listing limit must be positive");
      E.list_limit_bytes = (uint64_t)value;
      return DSM_OK;
    case DSM_OPT_SPLIT_MIN:
      if (value != 0 && (value < 64 || value > (1 << 24))) return E.fail(DSM_ERR_ARG, "split threshold 0 or 64..2^24");
      E.split_min = (uint32_t)value;
      return DSM_OK;
    case DSM_OPT_DONATE_DEPTH:
      if (value < 0 || value > 4) return E.fail(DSM_ERR_ARG, "donation depth 0..4");
      E.donate_depth = (uint32_t)value;
      return DSM_OK;
    case DSM_OPT_FILTER_INCREMENTAL: E.filter_incremental = value ? 1 : 0; return DSM_OK;
    case DSM_OPT_BFS_LEVELS:
      if (value < 0 || value > 8) return E.fail(DSM_ERR_ARG, "breadth-first levels 0..8");
      E.bfs_levels = (uint32_t)value;
      return DSM_OK;
    case DSM_OPT_BFS_ROWS:
      if (value < 32 || value > (1ll << 28)) return E.fail(DSM_ERR_ARG, "row table 32..2^28 rows");
      E.bfs_rows = (uint64_t)value;
      return DSM_OK;
    case DSM_OPT_MERGE_MAX:
      if (value < 0 || value > 4096) return E.fail(DSM_ERR_ARG, "merge threshold 0..4096 entries");
      E.merge_max = (uint32_t)value;
      return DSM_OK;
    case DSM_OPT_PACK_MAX:
      if (value < 0 || value > (1 << 20)) return E.fail(DSM_ERR_ARG, "intersection tile 0..2^20 entries");
      E.pack_max = (uint32_t)value;
      return DSM_OK;
    case DSM_OPT_AUTOTUNE: E.tune_next = value != 0; return DSM_OK;
    case DSM_OPT_GRAPH: E.use_graph = value ? 1 : 0; return DSM_OK;
    case DSM_OPT_STALL_TEST: E.stall_test = value ? 1 : 0; return DSM_OK;
    case DSM_OPT_PLAIN: E.plain = value ? 1 : 0; return DSM_OK;
    case DSM_OPT_WORK_LIMIT:
      if (value < 0) return E.fail(DSM_ERR_ARG, "work limit must be >= 0");
      E.work_limit = (unsigned long long)value;
      return DSM_OK;
    case DSM_OPT_QUERY_LIST_LIMIT:
      if (value < 0) return E.fail(DSM_ERR_ARG, "per-query listing limit must be >= 0");
      E.query_list_limit = (unsigned long long)value;
      return DSM_OK;
    case DSM_OPT_MEM_BUDGET:
      if (value <= 0 || (uint64_t)value < E.bytes_in_use)
        return E.fail(DSM_ERR_ARG, "budget must cover the bytes in use");
      E.budget = (size_t)value;
      E.admit_pending();
      return DSM_OK;
  }
  return E.fail(DSM_ERR_ARG, "unknown option");
}

int dsm_engine_get_option(dsm_engine *e, int option, int64_t *value) {
  ENGINE_OR_ARG(e);
  if (!value) return DSM_ERR_ARG;
  Engine &E = e->e;
  switch (option) {
    case DSM_OPT_LIST: *value = E.list_mode; return DSM_OK;
    case DSM_OPT_FILTER: *value = E.filter_mode; return DSM_OK;
    case DSM_OPT_RESULT_CAP: *value = (int64_t)E.result_cap; return DSM_OK;
    case DSM_OPT_WARPS_PER_SM: *value = E.warps_per_sm; return DSM_OK;
    case DSM_OPT_DONATE: *value = E.donate; return DSM_OK;
    case DSM_OPT_TIMEOUT_MS: *value = E.timeout_ms; return DSM_OK;
    case DSM_OPT_LABEL_QUIRK: *value = E.label_quirk; return DSM_OK;
    case DSM_OPT_SORT: *value = E.sort_results; return DSM_OK;
    case DSM_OPT_LIST_LIMIT: *value = (int64_t)E.list_limit_bytes; return DSM_OK;
    case DSM_OPT_MEM_BUDGET: *value = (int64_t)E.budget; return DSM_OK;
    case DSM_OPT_SPLIT_MIN: *value = E.split_min; return DSM_OK;
    case DSM_OPT_DONATE_DEPTH: *value = E.donate_depth; return DSM_OK;
    case DSM_OPT_PACK_MAX: *value = E.pack_max; return DSM_OK;
    case DSM_OPT_FILTER_INCREMENTAL: *value = E.filter_incremental; return DSM_OK;
    case DSM_OPT_MERGE_MAX: *value = E.merge_max; return DSM_OK;
    case DSM_OPT_BFS_LEVELS: *value = E.bfs_levels; return DSM_OK;
    case DSM_OPT_BFS_ROWS: *value = (int64_t)E.bfs_rows; return DSM_OK;
    case DSM_OPT_AUTOTUNE: *value = E.tune_next ? 1 : 0; return DSM_OK;
    case DSM_OPT_GRAPH: *value = E.use_graph; return DSM_OK;
    case DSM_OPT_STALL_TEST: *value = E.stall_test; return DSM_OK;
    case DSM_OPT_PLAIN: *value = E.plain; return DSM_OK;
    case DSM_OPT_WORK_LIMIT: *value = (int64_t)E.work_limit; return DSM_OK;
    case DSM_OPT_QUERY_LIST_LIMIT: *value = (int64_t)E.query_list_limit; return DSM_OK;
  }
  return E.fail(DSM_ERR_ARG, "unknown option");
}

int dsm_graph_load(dsm_engine *e, const uint32_t *offsets, const uint32_t *nbrs, const uint32_t *labels,
                   uint32_t nv) {
  ENGINE_OR_ARG(e);
  if (!offsets || !labels || (!nbrs && offsets[nv] != 0)) return DSM_ERR_ARG;
  std::vector<uint64_t> keys;
  keys.reserve(offsets[nv]);
  for (uint32_t v = 0; v < nv; ++v) {
    if (offsets[v + 1] < offsets[v]) return e->e.fail(DSM_ERR_ARG, "offsets not monotone");
    for (uint32_t k = offsets[v]; k < offsets[v + 1]; ++k) {
      uint32_t w = nbrs[k];
      if (w >= nv) return e->e.fail(DSM_ERR_ARG, "neighbour id >= num_v");
      if (w == v) continue;
      keys.push_back(v < w ? ((uint64_t)v << 32) | w : ((uint64_t)w << 32) | v);
    }
  }
  return e->e.load_graph(nv, labels, keys);
}

int dsm_graph_load_edges(dsm_engine *e, uint32_t nv, const uint32_t *labels, uint64_t ne, const uint32_t *edges) {
  ENGINE_OR_ARG(e);
  if (!labels || (!edges && ne)) return DSM_ERR_ARG;
  std::vector<uint64_t> keys;
  keys.reserve(ne);
  for (uint64_t k = 0; k < ne; ++k) {
    uint32_t a = edges[2 * k], b = edges[2 * k + 1];
    if (a >= nv || b >= nv) return e->e.fail(DSM_ERR_ARG, "edge endpoint >= num_v");
    if (a == b) continue;
    keys.push_back(a < b ? ((uint64_t)a << 32) | b : ((uint64_t)b << 32) | a);
  }
  return e->e.load_graph(nv, labels, keys);
}

int dsm_graph_export(dsm_engine *e, uint32_t *offsets, uint32_t *nbrs, uint64_t *num_entries) {
  ENGINE_OR_ARG(e);
  return e->e.export_graph(offsets, nbrs, num_entries);
}

int dsm_query_live(dsm_engine *e, uint32_t *qids, uint32_t cap, uint32_t *num) {
  ENGINE_OR_ARG(e);
  if (!num) return DSM_ERR_ARG;
  Engine &E = e->e;
  std::lock_guard<std::mutex> lk(E.mu);
  uint32_t n = 0;
  for (uint32_t id = 0; id < E.slots.size(); ++id)
    if (E.slots[id].live) {
      if (qids && n < cap) qids[n] = id;
      ++n;
    }
  *num = n;
  return DSM_OK;
}

int dsm_graph_apply(dsm_engine *e, const dsm_update *ups, uint32_t n) {
  ENGINE_OR_ARG(e);
  if (!ups && n) return DSM_ERR_ARG;
  return e->e.graph_apply(ups, n);
}

int dsm_graph_info(dsm_engine *e, uint32_t *nv, uint64_t *num_entries, uint64_t *arena_words) {
  ENGINE_OR_ARG(e);
  Engine &E = e->e;
  if (!E.graph_loaded) return E.fail(DSM_ERR_STATE, "no graph loaded");
  if (nv) *nv = E.nv;
  if (num_entries) {
    uint64_t n = 0;
    int rc = E.export_graph(nullptr, nullptr, &n);
    if (rc) return rc;
    *num_entries = n;
  }
  if (arena_words) *arena_words = E.arena_words;
  return DSM_OK;
}

int dsm_query_register(dsm_engine *e, const uint32_t *q_offsets, const uint32_t *q_nbrs, const uint32_t *q_labels,
                       uint32_t nq, uint32_t *qid) {
  ENGINE_OR_ARG(e);
  if (!q_offsets || !q_nbrs || !q_labels || !qid) return DSM_ERR_ARG;
  return e->e.register_query(q_offsets, q_nbrs, q_labels, nq, qid);
}

int dsm_query_retire(dsm_engine *e, uint32_t qid) {
  ENGINE_OR_ARG(e);
  return e->e.retire_query(qid);
}

int dsm_query_order(dsm_engine *e, uint32_t qid, uint32_t u, uint32_t v, uint32_t *order, uint32_t *bn_mask) {
  ENGINE_OR_ARG(e);
  Engine &E = e->e;
  std::lock_guard<std::mutex> lk(E.mu);
  if (qid >= E.slots.size() || !E.slots[qid].live) return E.fail(DSM_ERR_NOT_FOUND, "no such query");
  const dsm::QueryPlan &p = E.slots[qid].plan;
  for (size_t o = 0; o < p.oedges.size(); ++o)
    if (p.oedges[o].first == u && p.oedges[o].second == v) {
      for (uint32_t k = 0; k < p.nq; ++k) {
        if (order) order[k] = p.orders[o].vert[k];
        if (bn_mask) bn_mask[k] = p.orders[o].bn[k];
      }
      return DSM_OK;
    }
  return E.fail(DSM_ERR_NOT_FOUND, "(u, v) is not a query edge");
}

int dsm_query_filter(dsm_engine *e, uint32_t qid, uint32_t *bitmaps, uint32_t *v_cand_us) {
  ENGINE_OR_ARG(e);
  return e->e.query_filter(qid, bitmaps, v_cand_us);
}

int dsm_query_filter_state(dsm_engine *e, uint32_t qid, uint32_t *bitmaps, uint32_t *v_cand_us, uint32_t *info) {
  ENGINE_OR_ARG(e);
  return e->e.filter_state(qid, bitmaps, v_cand_us, info);
}

int dsm_query_plan(const uint32_t *q_offsets, const uint32_t *q_nbrs, const uint32_t *q_labels, uint32_t nq,
                   uint32_t *orders, uint32_t *bn_masks, uint32_t *oedges, uint32_t *num_oedges,
                   uint32_t *enc_pos_of_u) {
  if (!q_offsets || !q_nbrs || !q_labels) return DSM_ERR_ARG;
  dsm::QueryPlan p;
  std::string err;
  int rc = dsm::plan_query(nq, q_offsets, q_nbrs, q_labels, p, err);
  if (rc) return rc;
  for (size_t o = 0; o < p.orders.size(); ++o) {
    for (uint32_t k = 0; k < nq; ++k) {
      if (orders) orders[o * nq + k] = p.orders[o].vert[k];
      if (bn_masks) bn_masks[o * nq + k] = p.orders[o].bn[k];
    }
    if (oedges) {
      oedges[2 * o] = p.oedges[o].first;
      oedges[2 * o + 1] = p.oedges[o].second;
    }
  }
  if (num_oedges) *num_oedges = (uint32_t)p.orders.size();
  if (enc_pos_of_u)
    for (uint32_t u = 0; u < nq; ++u) enc_pos_of_u[u] = p.enc_pos_of_u[u];
  return DSM_OK;
}

int dsm_batch_submit(dsm_engine *e, const dsm_update *ups, uint32_t n, uint64_t *batch_id) {
  ENGINE_OR_ARG(e);
  if ((!ups && n) || !batch_id) return DSM_ERR_ARG;
  return e->e.submit(ups, n, batch_id);
}

int dsm_batch_wait(dsm_engine *e, uint64_t batch_id) {
  ENGINE_OR_ARG(e);
  return e->e.wait_batch(batch_id);
}

int dsm_batch_timing_get(dsm_engine *e, uint64_t batch_id, dsm_batch_timing *t) {
  ENGINE_OR_ARG(e);
  if (!t) return DSM_ERR_ARG;
  return e->e.timing(batch_id, t);
}

int dsm_serve_start(dsm_engine *e, uint32_t max_merge_updates) {
  ENGINE_OR_ARG(e);
  return e->e.serve_start(max_merge_updates);
}

int dsm_serve_stop(dsm_engine *e) {
  ENGINE_OR_ARG(e);
  return e->e.serve_stop();
}

int dsm_query_register_async(dsm_engine *e, const uint32_t *q_offsets, const uint32_t *q_nbrs,
                             const uint32_t *q_labels, uint32_t nq, uint64_t *ticket) {
  ENGINE_OR_ARG(e);
  if (!q_offsets || !q_nbrs || !q_labels || !ticket) return DSM_ERR_ARG;
  return e->e.register_async(q_offsets, q_nbrs, q_labels, nq, ticket);
}

int dsm_query_retire_async(dsm_engine *e, uint32_t qid, uint64_t *ticket) {
  ENGINE_OR_ARG(e);
  if (!ticket) return DSM_ERR_ARG;
  return e->e.retire_async(qid, ticket);
}

int dsm_query_admission(dsm_engine *e, uint64_t ticket, int64_t timeout_ms, uint32_t *qid) {
  ENGINE_OR_ARG(e);
  if (!qid) return DSM_ERR_ARG;
  return e->e.admission(ticket, timeout_ms, qid);
}

int dsm_batch_results(dsm_engine *e, uint64_t batch_id, dsm_result_view *view) {
  ENGINE_OR_ARG(e);
  if (!view) return DSM_ERR_ARG;
  return e->e.view(batch_id, view);
}

int dsm_batch_release(dsm_engine *e, uint64_t batch_id) {
  ENGINE_OR_ARG(e);
  return e->e.release(batch_id);
}

int dsm_engine_snapshot(dsm_engine *e, const char *path) {
  ENGINE_OR_ARG(e);
  if (!path) return DSM_ERR_ARG;
  return e->e.snapshot(path);
}

int dsm_engine_resume(dsm_engine *e, const char *path) {
  ENGINE_OR_ARG(e);
  if (!path) return DSM_ERR_ARG;
  return e->e.resume(path);
}

int dsm_engine_stats(dsm_engine *e, dsm_stats *s) {
  ENGINE_OR_ARG(e);
  if (!s) return DSM_ERR_ARG;
  std::lock_guard<std::mutex> lk(e->e.mu);
  std::lock_guard<std::mutex> ls(e->e.smu);
  *s = e->e.stats;
  s->device_bytes_in_use = e->e.bytes_in_use;
  s->query_bytes = s->live_queries = 0;
  for (const auto &q : e->e.slots)
    if (q.live) {
      s->query_bytes += q.foot;
      s->live_queries++;
    }
  return DSM_OK;
}

// ---- text ------------------------------------------------------------------
int dsm_text_read(const char *path, int is_query, dsm_text **out, char *err, size_t err_len) {
  if (!path || !out) return DSM_ERR_ARG;
  auto *t = new dsm_text();
  std::string msg;
  int bad;
  if (dsm::is_binary_graph(path)) {
    bad = dsm::map_binary_graph(path, is_query != 0, t->m, msg);
    t->a = t->m.a;
  } else {
    bad = dsm::read_text_graph(path, is_query != 0, t->g, msg);
    dsm::GraphArrays &a = t->a;
    a.is_query = is_query != 0;
    a.nv = t->g.nv;
    a.ne = t->g.ne;
    a.labels = t->g.labels.data();
    a.offsets = t->g.offsets.data();
    a.nbrs = t->g.nbrs.data();
    a.edges = t->g.edges.data();
    a.num_batches = (uint32_t)t->g.batch_sizes.size();
    a.batch_sizes = t->g.batch_sizes.data();
    a.num_updates = (uint32_t)(t->g.updates.size() / 4);
    a.updates = t->g.updates.data();
  }
  if (bad) {
    if (err && err_len) {
      std::strncpy(err, msg.c_str(), err_len - 1);
      err[err_len - 1] = 0;
    }
    delete t;
    return DSM_ERR_PARSE;
  }
  *out = t;
  return DSM_OK;
}

int dsm_text_write_binary(const dsm_text *t, const char *path) {
  if (!t || !path) return DSM_ERR_ARG;
  std::string msg;
  return dsm::write_binary_graph(path, t->a, msg) ? DSM_ERR_ARG : DSM_OK;
}

void dsm_text_free(dsm_text *t) { delete t; }
uint32_t dsm_text_nv(const dsm_text *t) { return t->a.nv; }
uint32_t dsm_text_ne(const dsm_text *t) { return t->a.ne; }
const uint32_t *dsm_text_labels(const dsm_text *t) { return t->a.labels; }
const uint32_t *dsm_text_offsets(const dsm_text *t) { return t->a.offsets; }
const uint32_t *dsm_text_nbrs(const dsm_text *t) { return t->a.nbrs; }
const uint32_t *dsm_text_edges(const dsm_text *t) { return t->a.edges; }
uint32_t dsm_text_num_batches(const dsm_text *t) { return t->a.num_batches; }
const uint32_t *dsm_text_batch_sizes(const dsm_text *t) { return t->a.batch_sizes; }
uint32_t dsm_text_num_updates(const dsm_text *t) { return t->a.num_updates; }
const dsm_update *dsm_text_updates(const dsm_text *t) { return reinterpret_cast<const dsm_update *>(t->a.updates); }

// ---- workloads ---------------------------------------------------------------
int dsm_workload_generate(int config, uint64_t seed, int scale_log2, uint32_t num_batches, dsm_workload **out) {
  if (!out) return DSM_ERR_ARG;
  dsm::GenParams p;
  if (dsm::preset_params(config, p)) return DSM_ERR_ARG;
  if (seed) p.seed = seed;
  if (scale_log2 < 0) {
    int s = -scale_log2;
    if ((int)p.log2_nv - s < 4) return DSM_ERR_ARG;
    p.log2_nv -= s;
    p.num_edges >>= s;
    if (p.stream == dsm::GenParams::kStreamWithheld) p.num_deletes >>= s;
  }
  if (num_batches) p.num_batches = num_batches;
  auto *w = new dsm_workload();
  if (dsm::generate_workload(p, w->w)) {
    delete w;
    return DSM_ERR_LIMIT;
  }
  *out = w;
  return DSM_OK;
}
void dsm_workload_free(dsm_workload *w) { delete w; }
uint32_t dsm_workload_nv(const dsm_workload *w) { return w->w.nv; }
const uint32_t *dsm_workload_labels(const dsm_workload *w) { return w->w.labels.data(); }
uint64_t dsm_workload_num_edges(const dsm_workload *w) { return w->w.edges.size() / 2; }
const uint32_t *dsm_workload_edges(const dsm_workload *w) { return w->w.edges.data(); }
uint32_t dsm_workload_num_queries(const dsm_workload *w) { return (uint32_t)w->w.queries.size(); }
uint32_t dsm_workload_query_nv(const dsm_workload *w, uint32_t q) { return w->w.queries[q].nv; }
const uint32_t *dsm_workload_query_labels(const dsm_workload *w, uint32_t q) { return w->w.queries[q].labels.data(); }
const uint32_t *dsm_workload_query_offsets(const dsm_workload *w, uint32_t q) {
  return w->w.queries[q].offsets.data();
}
const uint32_t *dsm_workload_query_nbrs(const dsm_workload *w, uint32_t q) { return w->w.queries[q].nbrs.data(); }
uint32_t dsm_workload_num_batches(const dsm_workload *w) { return (uint32_t)w->w.batch_sizes.size(); }
const uint32_t *dsm_workload_batch_sizes(const dsm_workload *w) { return w->w.batch_sizes.data(); }
uint32_t dsm_workload_num_updates(const dsm_workload *w) { return (uint32_t)(w->w.updates.size() / 4); }
const dsm_update *dsm_workload_updates(const dsm_workload *w) {
  return reinterpret_cast<const dsm_update *>(w->w.updates.data());
}
int dsm_workload_write(const dsm_workload *w, const char *query_prefix, const char *data_path) {
  if (!w || !query_prefix || !data_path) return DSM_ERR_ARG;
  for (size_t q = 0; q < w->w.queries.size(); ++q)
    if (dsm::write_query_file(std::string(query_prefix) + std::to_string(q) + ".in", w->w.queries[q]))
      return DSM_ERR_ARG;
  return dsm::write_data_file(data_path, w->w) ? DSM_ERR_ARG : DSM_OK;
}

}  // extern "C"
