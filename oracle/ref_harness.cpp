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
#include "order.h"

// The two host globals these sources read (declared in globals.cuh; the
// reference's globals.cu does not compile on its own).
uint32_t NUM_VQ = 0;
uint32_t NUM_EQ = 0;

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
