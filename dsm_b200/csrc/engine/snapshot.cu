// Snapshot and resume of an engine (no counterpart in the reference, which
// keeps its graph only for the life of one process): the current data graph
// as a sorted CSR with its labels, every registered query with its id, and
// the batch counter, in one file.  A snapshot is taken between device
// batches (it holds the engine lock, which a running batch holds too), so it
// covers exactly the batches that finished before it.
//
// Layout (little-endian): header (64 bytes): magic "DSMSNAP1", version,
// nv, entries (u64), number of queries, next batch id (u64); labels[nv],
// offsets[nv + 1], nbrs[entries]; per query: id, nq, query entries,
// labels[nq], offsets[nq + 1], nbrs[query entries].
#include <cstdio>
#include <cstring>
#include <vector>

#include "engine_internal.h"

namespace dsm {

namespace {

constexpr char kSnapMagic[8] = {'D', 'S', 'M', 'S', 'N', 'A', 'P', '1'};

struct SnapHeader {
  char magic[8];
  uint32_t version, nv;
  uint64_t entries;
  uint32_t num_queries, pad0;
  uint64_t next_batch;
  uint32_t pad[6];
};
static_assert(sizeof(SnapHeader) == 64, "snapshot header is 64 bytes");

struct File {
  FILE *f = nullptr;
  explicit File(FILE *x) : f(x) {}
  ~File() {
    if (f) std::fclose(f);
  }
  bool put(const void *p, size_t words) { return words == 0 || std::fwrite(p, 4, words, f) == words; }
  bool get(void *p, size_t words) { return words == 0 || std::fread(p, 4, words, f) == words; }
};

}  // namespace

int Engine::snapshot(const char *path) {
  std::lock_guard<std::mutex> lk(mu);
  if (!graph_loaded) return fail(DSM_ERR_STATE, "no graph loaded");
  if (cudaError_t e = cudaSetDevice(device)) return cuda_fail(e, "cudaSetDevice");
  uint64_t entries = 0;
  if (int rc = export_graph_locked(nullptr, nullptr, &entries)) return rc;
  std::vector<uint32_t> off(nv + 1), nbr(std::max<uint64_t>(entries, 1));
  if (int rc = export_graph_locked(off.data(), nbr.data(), &entries)) return rc;
  SnapHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kSnapMagic, 8);
  h.version = 1;
  h.nv = nv;
  h.entries = entries;
  for (const Slot &s : slots) h.num_queries += s.live ? 1 : 0;
  h.next_batch = next_batch_id;
  File f(std::fopen(path, "wb"));
  if (!f.f) return fail(DSM_ERR_ARG, std::string("cannot open ") + path);
  bool ok = std::fwrite(&h, sizeof(h), 1, f.f) == 1 && f.put(label_host.data(), nv) && f.put(off.data(), nv + 1) &&
            f.put(nbr.data(), entries);
  for (uint32_t id = 0; id < slots.size() && ok; ++id) {
    const Slot &s = slots[id];
    if (!s.live) continue;
    const QueryPlan &p = s.plan;
    const uint32_t rec[3] = {id, p.nq, (uint32_t)p.nbrs.size()};
    ok = f.put(rec, 3) && f.put(p.labels.data(), p.nq) && f.put(p.offsets.data(), p.nq + 1) &&
         f.put(p.nbrs.data(), p.nbrs.size());
  }
  if (!ok) return fail(DSM_ERR_ARG, std::string("write failed: ") + path);
  return DSM_OK;
}

int Engine::resume(const char *path) {
  {
    std::lock_guard<std::mutex> q(srv.qmu);
    if (srv.running) return fail(DSM_ERR_STATE, "resume with the serving loop stopped");
  }
  {
    std::lock_guard<std::mutex> lk(mu);
    for (const Slot &s : slots)
      if (s.live) return fail(DSM_ERR_STATE, "resume needs an engine without registered queries");
  }
  File f(std::fopen(path, "rb"));
  if (!f.f) return fail(DSM_ERR_ARG, std::string("cannot open ") + path);
  SnapHeader h;
  if (std::fread(&h, sizeof(h), 1, f.f) != 1 || std::memcmp(h.magic, kSnapMagic, 8) != 0 || h.version != 1)
    return fail(DSM_ERR_PARSE, "not a snapshot file");
  std::vector<uint32_t> labels(h.nv), off(h.nv + 1), nbr(h.entries);
  if (!f.get(labels.data(), h.nv) || !f.get(off.data(), h.nv + 1) || !f.get(nbr.data(), h.entries) ||
      off[h.nv] != h.entries)
    return fail(DSM_ERR_PARSE, "snapshot truncated");
  std::vector<uint64_t> keys;
  keys.reserve(h.entries / 2);
  for (uint32_t v = 0; v < h.nv; ++v)
    for (uint32_t k = off[v]; k < off[v + 1]; ++k) {
      if (nbr[k] >= h.nv) return fail(DSM_ERR_PARSE, "snapshot: neighbour id >= num_v");
      if (v < nbr[k]) keys.push_back(((uint64_t)v << 32) | nbr[k]);
    }
  if (int rc = load_graph(h.nv, labels.data(), keys)) return rc;
  std::lock_guard<std::mutex> lk(mu);
  for (uint32_t k = 0; k < h.num_queries; ++k) {
    uint32_t rec[3];
    if (!f.get(rec, 3) || rec[1] == 0 || rec[1] > 16) return fail(DSM_ERR_PARSE, "snapshot: bad query record");
    std::vector<uint32_t> ql(rec[1]), qo(rec[1] + 1), qn(rec[2]);
    if (!f.get(ql.data(), rec[1]) || !f.get(qo.data(), rec[1] + 1) || !f.get(qn.data(), rec[2]) ||
        qo[rec[1]] != rec[2])
      return fail(DSM_ERR_PARSE, "snapshot: query truncated");
    QueryPlan plan;
    std::string err;
    if (int rc = plan_query(rec[1], qo.data(), qn.data(), ql.data(), plan, err)) return fail(rc, err);
    uint32_t qid = 0;
    if (int rc = admit(plan, &qid, nullptr, rec[0])) return rc;
  }
  if (h.next_batch > next_batch_id) next_batch_id = h.next_batch;
  return DSM_OK;
}

}  // namespace dsm
