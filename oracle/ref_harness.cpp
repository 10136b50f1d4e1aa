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

}  // extern "C"
