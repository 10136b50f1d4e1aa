// Device side of the cluster-encoding candidate filter.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace dsm {

// Per-query constants of the filter (full query: labels, degrees, neighbour
// label counts; plan: candidacy positions).
struct QFilterDesc {
  uint32_t nq;
  uint32_t nlabels;          // largest query label + 1 (copyMeta, io.cu:334)
  uint32_t label_us[32];     // per label: mask of query vertices carrying it
  uint32_t qdeg[16];
  uint32_t pos_of_u[16];
  uint8_t nlc[16][32];       // neighbour label counts of the full query
  // incremental filter: hops of the query's region (its op count), the
  // region epoch its state was last computed in (0xFFFFFFFF: never), and
  // whether the run in progress recomputes every vertex (decided by the
  // run's first kernel, read by the others)
  uint32_t hops;
  uint32_t fepoch;
  uint32_t full_now;
  uint32_t pad;
};

// One op of the plan (see host/query_plan.h FilterOp), compact form.
struct DevFilterOp {
  uint32_t kind, core_u, pos, nleaf;
  uint32_t leaf_u[16];
  uint32_t lp, rp, lcp, rcp;
  uint32_t comb_type, nsmall;
  uint32_t small_core_pos[32];
  uint32_t leaf_src_count[16];
  uint16_t leaf_src[16][32];
  // earlier ops with the same core vertex that can withdraw its candidates
  // (merges and combines), for the incremental filter's validity replay
  uint32_t nprior;
  uint32_t prior[15];
};

// Incremental region (one per engine, shared by the queries of a batch).
// The region of a batch is every vertex within r hops of the endpoints of
// this batch's and the previous batch's updates, on the batch's union graph:
// list[bound[r-1] .. bound[r]) holds the vertices first reached at hop r
// (bound[-1] = 0); mark[v] = epoch << 6 | hop for vertices reached in this
// epoch.  A query whose plan has D ops needs hops 0..D; if the list overflowed
// at or before hop D (ov_round <= D), that query is filtered in full.
constexpr uint32_t kRegionMaxHops = 62;
struct RegionInfo {
  uint32_t stale;      // set by the host when the graph changed outside a filtered batch
  uint32_t stale_now;  // this batch: the previous union graph is unknown
  uint32_t epoch;
  uint32_t total;      // entries appended (may exceed the capacity)
  uint32_t cap;        // list capacity
  uint32_t ov_round;   // first hop whose vertices did not all fit (64: none)
  uint32_t prev_cnt;   // endpoints kept from the previous batch
  uint32_t prev_cap;
  uint32_t prev_ov;    // 1: the previous batch had more endpoints than prev_cap
  uint32_t hops;       // hops built this batch
  uint32_t pad[7];
  uint32_t bound[64];  // list length after each hop
};

struct RegionDevice {
  RegionInfo *info;
  uint32_t *mark;      // [nv]
  uint32_t *list;      // [cap]
  uint32_t *prev;      // [prev_cap] endpoints of the previous batch's updates
};

struct FilterDevice {
  const QFilterDesc *desc;
  const DevFilterOp *ops;
  uint32_t nops;
  uint32_t *vcand, *valid, *enc, *bitmap;
  uint32_t words, col_len;
};

// mode 1: LDF+NLF only; mode 2: cluster encoding.  Writes f.bitmap.  With a
// region (rg.info != nullptr) and force_full == 0, only the vertices of the
// query's region are recomputed, unless the region overflowed.
void launch_query_filter(const DevGraph &g, const FilterDevice &f, int mode, int num_sms, cudaStream_t s,
                         const RegionDevice &rg, int force_full);

// Region of a batch: hops 0..hops from the endpoints of the batch's updates
// (upd, hdr->n) and of the previous batch's (rg.prev); then the batch's own
// endpoints are kept for the next batch.  Launches 1 + 2 * hops + 1 kernels
// around the filters: begin/expand before them, save after.
void launch_region_build(const DevGraph &g, const RegionDevice &rg, const uint32_t *hdr_n, const uint4 *upd,
                         uint32_t hops, int num_sms, cudaStream_t s);
void launch_region_save(const RegionDevice &rg, const uint32_t *hdr_n, const uint4 *upd, cudaStream_t s);

}  // namespace dsm
