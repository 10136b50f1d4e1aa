// TEST INFRASTRUCTURE ONLY.  The seeded workload generator of the engine's
// host code (dsm_b200/csrc/host/gen.cpp, compiled into this library as well)
// behind a C ABI of the oracle, so that the CPU baseline and the reference
// arm of the benchmark generate exactly the engine's inputs without loading
// the engine library.
#include <cstdint>

#include "../dsm_b200/csrc/host/dsm_host.h"

struct orc_workload {
  dsm::Workload w;
};

extern "C" {

int orc_workload_generate(int config, uint64_t seed, int scale_log2, uint32_t num_batches, orc_workload **out) {
  dsm::GenParams p;
  if (!out || dsm::preset_params(config, p)) return -1;
  if (seed) p.seed = seed;
  if (scale_log2 < 0) {
    const int s = -scale_log2;
    if ((int)p.log2_nv - s < 4) return -1;
    p.log2_nv -= s;
    p.num_edges >>= s;
    if (p.stream == dsm::GenParams::kStreamWithheld) p.num_deletes >>= s;
  }
  if (num_batches) p.num_batches = num_batches;
  auto *h = new orc_workload();
  if (dsm::generate_workload(p, h->w)) {
    delete h;
    return -2;
  }
  *out = h;
  return 0;
}
void orc_workload_free(orc_workload *h) { delete h; }
uint32_t orc_workload_nv(const orc_workload *h) { return h->w.nv; }
const uint32_t *orc_workload_labels(const orc_workload *h) { return h->w.labels.data(); }
uint64_t orc_workload_num_edges(const orc_workload *h) { return h->w.edges.size() / 2; }
const uint32_t *orc_workload_edges(const orc_workload *h) { return h->w.edges.data(); }
uint32_t orc_workload_num_queries(const orc_workload *h) { return (uint32_t)h->w.queries.size(); }
uint32_t orc_workload_query_nv(const orc_workload *h, uint32_t q) { return h->w.queries[q].nv; }
const uint32_t *orc_workload_query_labels(const orc_workload *h, uint32_t q) { return h->w.queries[q].labels.data(); }
const uint32_t *orc_workload_query_offsets(const orc_workload *h, uint32_t q) {
  return h->w.queries[q].offsets.data();
}
const uint32_t *orc_workload_query_nbrs(const orc_workload *h, uint32_t q) { return h->w.queries[q].nbrs.data(); }
uint32_t orc_workload_num_batches(const orc_workload *h) { return (uint32_t)h->w.batch_sizes.size(); }
const uint32_t *orc_workload_batch_sizes(const orc_workload *h) { return h->w.batch_sizes.data(); }
uint32_t orc_workload_num_updates(const orc_workload *h) { return (uint32_t)(h->w.updates.size() / 4); }
const uint32_t *orc_workload_updates(const orc_workload *h) { return h->w.updates.data(); }

}  // extern "C"
