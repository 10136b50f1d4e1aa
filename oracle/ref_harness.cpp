// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's own host code, compiled from its sources by
// oracle/ref.mk into oracle/_ref/libref.so, so that the oracle's restatements
// of decycle (decycle.cpp:6-135) and of the BFS matching order with backward
// neighbours (order.cpp:367-402, 647-676) are checked against the original.
// The query cpuGraph is filled the way readGraphToCPUDynamic fills it
// (io.cu:122-252: CSR in file order of the edges, vve / evv edge ids 2e and
// 2e + 1) and `keep` is allocated as main.cu:76-77 does.
#include <cstdint>
#include <cstring>
#include <vector>

#include "cpuGraph.h"
#include "decycle.h"
#include "filter.cuh"
#include "globals.cuh"
#include "io.cuh"
#include "order.h"
#include "structure.cuh"

// The host globals these sources read (NUM_VQ, NUM_EQ, ...) come from the
// reference's own globals.cu, linked into the same library.

namespace {

// nq vertices, ne undirected edges (pairs, file order).
void fill_query(cpuGraph &g, uint32_t nq, uint32_t ne, const uint32_t *edges) {
  g.isQuery = true;
  g.num_v = nq;
  g.num_e = ne;
  g.vertexIDs_ = new vtype[nq];
  g.offsets_ = new offtype[nq + 1];
  g.neighbors_ = new vtype[2 * ne];
  g.edgeIDs_ = new etype[2 * ne];
  g.outdeg_ = new degtype[nq];
  g.vLabels_ = new vltype[nq];
  std::memset(g.outdeg_, 0, sizeof(degtype) * nq);
  for (uint32_t e = 0; e < ne; ++e) {
    g.outdeg_[edges[2 * e]]++;
    g.outdeg_[edges[2 * e + 1]]++;
  }
  g.offsets_[0] = 0;
  for (uint32_t v = 0; v < nq; ++v) {
    g.vertexIDs_[v] = v;
    g.vLabels_[v] = 0;
    g.offsets_[v + 1] = g.offsets_[v] + g.outdeg_[v];
  }
  uint32_t *fill = new uint32_t[nq]();
  for (uint32_t e = 0; e < ne; ++e) {
    const uint32_t a = edges[2 * e], b = edges[2 * e + 1];
    g.vve.insert({std::pair<vtype, vtype>(a, b), 2 * e});
    g.evv.insert({2 * e, std::make_pair(a, b)});
    g.vve.insert({std::pair<vtype, vtype>(b, a), 2 * e + 1});
    g.evv.insert({2 * e + 1, std::make_pair(b, a)});
    g.neighbors_[g.offsets_[a] + fill[a]] = b;
    g.edgeIDs_[g.offsets_[a] + fill[a]++] = 2 * e;
    g.neighbors_[g.offsets_[b] + fill[b]] = a;
    g.edgeIDs_[g.offsets_[b] + fill[b]++] = 2 * e + 1;
  }
  delete[] fill;
  g.keep = new bool[2 * ne];
  std::memset(g.keep, false, sizeof(bool) * 2 * ne);
}

}  // namespace

extern "C" {

// keep_out[e] = 1 when the reference's decycle keeps edge e; deg_out[v] = its
// degree in the spanning tree.
int ref_decycle(uint32_t nq, uint32_t ne, const uint32_t *edges, uint8_t *keep_out, uint32_t *deg_out) {
  if (nq == 0 || nq > 16) return -1;
  cpuGraph g;
  fill_query(g, nq, ne, edges);
  NUM_VQ = nq;
  NUM_EQ = ne;
  decycle(&g);
  for (uint32_t e = 0; e < ne; ++e) keep_out[e] = g.keep[2 * e] ? 1 : 0;
  for (uint32_t v = 0; v < nq; ++v) deg_out[v] = g.outdeg_[v];
  return 0;
}

// The matching order rooted at the ordered query edge (u, v): order_out[p] =
// query vertex at position p, bn_out[p] = mask of positions < p adjacent to
// it (the reference's backward_neighbors lists turned into position masks).
int ref_order(uint32_t nq, uint32_t ne, const uint32_t *edges, uint32_t u, uint32_t v, uint32_t *order_out,
              uint32_t *bn_out) {
  if (nq == 0 || nq > 16) return -1;
  cpuGraph g;
  fill_query(g, nq, ne, edges);
  NUM_VQ = nq;
  NUM_EQ = ne;
  OrderCPU o(1);
  o.roots.push_back(u);
  o.sub_roots.push_back(v);
  o.getVertexOrderBFS(&g);
  o.constructBackwardNeighbors(&g);
  if (o.v_orders[0].size() != nq) return -2;  // disconnected
  uint32_t pos[16];
  for (uint32_t p = 0; p < nq; ++p) {
    order_out[p] = o.v_orders[0][p];
    pos[o.v_orders[0][p]] = p;
  }
  for (uint32_t p = 0; p < nq; ++p) {
    uint32_t m = 0;
    for (vtype w : o.backward_neighbors[0][order_out[p]]) m |= 1u << pos[w];
    bn_out[p] = m;
  }
  return 0;
}

// ---- cluster-filter plan (filter.cu:23-392, structure.cu:113-135) -------
// The reference's decycle, then its clustering of the spanning tree
// (vertex cover, merges, combines, encodingMeta::init), then the position
// pick of clusterFilter (filter.cu:1582-1609, which sits inside a function
// that launches kernels, so it is restated here: newest valid cluster first,
// each query vertex at its first position there).  Serialised into out:
//   num_clusters, final_cluster_id, merge_count, combine_cnt, num_layers,
//   per cluster c: valid, size, its query vertices (core first),
//   per merge: left, right,
//   per combine: out cluster, type, number of others, the others (ascending),
//   layer offsets (num_layers + 1),
//   enc_pos_of_u (nq).
// Returns the number of words written, or a negative code.
int ref_cluster_plan(uint32_t nq, uint32_t ne, const uint32_t *edges, uint32_t *out, uint32_t cap) {
  if (nq == 0 || nq > 16) return -1;
  cpuGraph g;
  fill_query(g, nq, ne, edges);
  NUM_VQ = nq;
  NUM_EQ = ne;
  decycle(&g);
  std::vector<cpuCluster> cl;
  encodingMeta meta;
  clustering(&g, cl, &meta);
  std::vector<uint32_t> w;
  const uint32_t nc = meta.num_clusters;
  w.push_back(nc);
  w.push_back(meta.final_cluster_id);
  w.push_back(meta.merge_count);
  w.push_back(meta.combine_cnt);
  w.push_back(meta.num_layers);
  for (uint32_t c = 0; c < nc; ++c) {
    w.push_back(meta.is_a_valid_cluster_[c] ? 1 : 0);
    w.push_back(cl[c].num_query_us);
    for (uint32_t k = 0; k < cl[c].num_query_us; ++k) w.push_back(cl[c].query_us_[k]);
  }
  for (uint32_t k = 0; k < meta.merge_count; ++k) {
    w.push_back(meta.merged_cluster_left_[k]);
    w.push_back(meta.merged_cluster_right_[k]);
  }
  for (uint32_t k = 0; k < meta.combine_cnt; ++k) {
    w.push_back(meta.combine_cluster_out_[k]);
    w.push_back((uint32_t)meta.combine_type_[k]);
    w.push_back((uint32_t)meta.combine_clusters_other_[k].size());
    for (int o : meta.combine_clusters_other_[k]) w.push_back((uint32_t)o);
  }
  for (uint32_t l = 0; l <= meta.num_layers; ++l) w.push_back(meta.layer_offsets_[l]);
  std::vector<uint32_t> pos(nq, 0xFFFFFFFFu);
  std::vector<char> vis(nq, 0);
  uint32_t cnt = 0;
  for (int c = (int)meta.final_cluster_id; c >= 0; --c) {
    if (!meta.is_a_valid_cluster_[c]) continue;
    if (cnt == nq) break;
    for (uint32_t p = meta.cluster_offsets_[c]; p < meta.cluster_offsets_[c + 1]; ++p) {
      const uint32_t u = meta.query_us_compact_[p];
      if (!vis[u]) {
        vis[u] = 1;
        pos[u] = p;
        ++cnt;
      }
    }
  }
  for (uint32_t u = 0; u < nq; ++u) w.push_back(pos[u]);
  if (w.size() > cap) return -3;
  std::copy(w.begin(), w.end(), out);
  return (int)w.size();
}

// ---- text files (readGraphToCPUDynamic, io.cu:122-252) --------------------
void *ref_file_read(const char *path, int is_query) {
  auto *g = new cpuGraph();
  g->isQuery = is_query != 0;
  readGraphToCPUDynamic(g, path);
  return g;
}

// nv, ne; then the CSR as parsed (off: nv + 1, nbr: 2 ne, labels: nv) and
// the batches (sizes: one per batch; ups: 4 words per update, op 1 = add).
void ref_file_sizes(void *h, uint32_t *nv, uint32_t *ne, uint32_t *nbatches, uint32_t *nupdates) {
  const cpuGraph &g = *static_cast<cpuGraph *>(h);
  *nv = g.num_v;
  *ne = g.num_e;
  *nbatches = (uint32_t)g.batches.size();
  size_t n = 0;
  for (const auto &b : g.batches) n += b.size();
  *nupdates = (uint32_t)n;
}

void ref_file_export(void *h, uint32_t *off, uint32_t *nbr, uint32_t *labels, uint32_t *sizes, uint32_t *ups) {
  const cpuGraph &g = *static_cast<cpuGraph *>(h);
  for (uint32_t v = 0; v <= g.num_v; ++v) off[v] = g.offsets_[v];
  for (uint64_t k = 0; k < 2ull * g.num_e; ++k) nbr[k] = g.neighbors_[k];
  for (uint32_t v = 0; v < g.num_v; ++v) labels[v] = g.vLabels_[v];
  size_t i = 0;
  for (size_t b = 0; b < g.batches.size(); ++b) {
    sizes[b] = (uint32_t)g.batches[b].size();
    for (const change &c : g.batches[b]) {
      ups[4 * i] = c.add ? 1 : 0;
      ups[4 * i + 1] = c.src;
      ups[4 * i + 2] = c.dst;
      ups[4 * i + 3] = c.labelChange;
      ++i;
    }
  }
}

void ref_file_free(void *h) { delete static_cast<cpuGraph *>(h); }

// ---- data graph and updateHostGraph (cpuGraph.cpp:521-607) ---------------
// A data cpuGraph filled as readGraphToCPUDynamic fills it (io.cu:122-252):
// CSR over both directions, each list in file order of the edges.
void *ref_graph_new(uint32_t nv, const uint32_t *labels, uint64_t ne, const uint32_t *edges) {
  auto *g = new cpuGraph();
  g->isQuery = false;
  g->num_v = nv;
  g->num_e = (numtype)ne;
  g->vertexIDs_ = new vtype[nv];
  g->offsets_ = new offtype[nv + 1];
  g->outdeg_ = new degtype[nv];
  g->vLabels_ = new vltype[nv];
  g->neighbors_ = new vtype[2 * ne + 1];
  std::memset(g->outdeg_, 0, sizeof(degtype) * nv);
  for (uint64_t e = 0; e < ne; ++e) {
    g->outdeg_[edges[2 * e]]++;
    g->outdeg_[edges[2 * e + 1]]++;
  }
  g->offsets_[0] = 0;
  for (uint32_t v = 0; v < nv; ++v) {
    g->vertexIDs_[v] = v;
    g->vLabels_[v] = labels[v];
    g->offsets_[v + 1] = g->offsets_[v] + g->outdeg_[v];
  }
  uint32_t *fill = new uint32_t[nv]();
  for (uint64_t e = 0; e < ne; ++e) {
    const uint32_t a = edges[2 * e], b = edges[2 * e + 1];
    g->neighbors_[g->offsets_[a] + fill[a]++] = b;
    g->neighbors_[g->offsets_[b] + fill[b]++] = a;
  }
  delete[] fill;
  return g;
}

// One batch through the reference's updateHostGraph; updates are 4 words
// each (op 1 = add, src, dst, label).  The reference replaces neighbors_
// without freeing the old array; the harness frees it afterwards.
int ref_graph_update(void *h, uint32_t n, const uint32_t *ups) {
  cpuGraph &g = *static_cast<cpuGraph *>(h);
  std::vector<change> batch(n);
  for (uint32_t i = 0; i < n; ++i) {
    batch[i].add = ups[4 * i] == 1;
    batch[i].src = ups[4 * i + 1];
    batch[i].dst = ups[4 * i + 2];
    batch[i].labelChange = ups[4 * i + 3];
  }
  vtype *old = g.neighbors_;
  updateHostGraph(g, batch);
  if (old != g.neighbors_) delete[] old;
  return 0;
}

// The graph as a CSR (off: nv + 1 words; nbr may be null to size it) and
// the labels.  Returns the number of neighbour entries.
uint64_t ref_graph_export(void *h, uint32_t *off, uint32_t *nbr, uint32_t *labels) {
  const cpuGraph &g = *static_cast<cpuGraph *>(h);
  const uint64_t total = g.offsets_[g.num_v];
  if (off)
    for (uint32_t v = 0; v <= g.num_v; ++v) off[v] = g.offsets_[v];
  if (nbr)
    for (uint64_t k = 0; k < total; ++k) nbr[k] = g.neighbors_[k];
  if (labels)
    for (uint32_t v = 0; v < g.num_v; ++v) labels[v] = g.vLabels_[v];
  return total;
}

void ref_graph_free(void *h) { delete static_cast<cpuGraph *>(h); }

}  // extern "C"
