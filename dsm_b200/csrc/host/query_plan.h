// Host-side preprocessing of one query: validation, spanning tree, matching
// orders per ordered query edge, and the op list of the cluster-encoding
// candidate filter.  The result is uploaded as a fixed-size descriptor.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "order_rec.h"

namespace dsm {


// One op of the cluster-encoding filter, executed in list order.
struct FilterOp {
  enum Kind : uint32_t { kEncode = 0, kMerge = 1, kCombine = 2 };
  uint32_t kind;
  uint32_t core_u;    // query vertex whose candidate list drives the op
  uint32_t pos;       // first encoding position of the cluster written
  uint32_t nleaf;     // leaves of that cluster (size - 1)
  uint32_t leaf_u[16];  // encode: leaf query vertices
  // merge: the bits read
  uint32_t left_pos, right_pos, left_core_pos, right_core_pos;
  // combine
  uint32_t comb_type;          // 0: new cluster (OR leaves), 1: existing cluster (AND)
  uint32_t nsmall;
  uint32_t small_core_pos[32];
  // for leaf i of the combined cluster: positions in the small clusters that
  // hold the same query vertex (first match per small cluster)
  uint32_t leaf_src_count[16];
  uint32_t leaf_src[16][32];
};

struct QueryPlan {
  uint32_t nq = 0, ne = 0;
  std::vector<uint32_t> labels, degree;  // full query
  std::vector<uint32_t> adj_mask;        // full query adjacency as bit masks
  std::vector<uint32_t> offsets, nbrs;   // full query CSR (file order)
  // spanning tree (decycle.cpp:6-135)
  std::vector<uint32_t> tree_offsets, tree_nbrs, tree_degree;
  // ordered query edges in CSR order: (u, nbrs[k]); orders[k] seeds with it
  std::vector<std::pair<uint32_t, uint32_t>> oedges;
  std::vector<OrderRec> orders;
  // filter
  uint32_t nlabels = 0;                  // largest query label + 1 (copyMeta, io.cu:334)
  std::vector<uint32_t> nlc;             // nq x 32: neighbour label counts (full query)
  std::vector<FilterOp> ops;
  uint32_t enc_positions = 0;            // total cluster members
  uint32_t enc_words = 0;                // words per data vertex
  std::vector<uint32_t> enc_pos_of_u;    // encoding position whose bit is u's candidacy
  std::vector<std::vector<uint32_t>> clusters;  // for inspection
  std::vector<uint8_t> cluster_valid;
};

// Returns 0, or a DSM_ERR_* code with a message.
int plan_query(uint32_t nq, const uint32_t *offsets, const uint32_t *nbrs, const uint32_t *labels,
               QueryPlan &qp, std::string &err);

}  // namespace dsm
