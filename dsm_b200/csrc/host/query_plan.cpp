// Query preprocessing on the host.  Mirrors the reference's decycle.cpp,
// order.cpp and the host half of filter.cu, with the query kept as 32-bit
// adjacency masks (a query has at most 16 vertices here).
#include "query_plan.h"

#include <algorithm>
#include <cstring>
#include <set>

#include "../../../include/dsm.h"
#include "dsm_host.h"

namespace dsm {

namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr size_t kClusterCap = 150;  // MAX_CLUSTERS (defs.h:22)
constexpr size_t kLayerCap = 100;    // MAX_LAYERS (defs.h:23)

// BFS spanning tree from the first vertex of maximum degree; an edge is a
// tree edge when the BFS first reaches a vertex through it (decycle.cpp:6-135).
void spanning_tree(QueryPlan &qp) {
  const uint32_t nq = qp.nq;
  uint32_t root = 0;
  for (uint32_t u = 1; u < nq; ++u)
    if (qp.degree[u] > qp.degree[root]) root = u;
  std::vector<uint32_t> tree_mask(nq, 0);
  uint32_t seen = 1u << root;
  std::vector<uint32_t> fifo{root};
  for (size_t h = 0; h < fifo.size(); ++h) {
    uint32_t top = fifo[h];
    for (uint32_t k = qp.offsets[top]; k < qp.offsets[top + 1]; ++k) {
      uint32_t w = qp.nbrs[k];
      if (seen & (1u << w)) continue;
      seen |= 1u << w;
      fifo.push_back(w);
      tree_mask[top] |= 1u << w;
      tree_mask[w] |= 1u << top;
    }
  }
  qp.tree_offsets.assign(nq + 1, 0);
  qp.tree_nbrs.clear();
  qp.tree_degree.assign(nq, 0);
  for (uint32_t u = 0; u < nq; ++u) {
    for (uint32_t k = qp.offsets[u]; k < qp.offsets[u + 1]; ++k)
      if (tree_mask[u] & (1u << qp.nbrs[k])) qp.tree_nbrs.push_back(qp.nbrs[k]);
    qp.tree_offsets[u + 1] = (uint32_t)qp.tree_nbrs.size();
    qp.tree_degree[u] = qp.tree_offsets[u + 1] - qp.tree_offsets[u];
  }
}

// BFS from the ordered edge (u, v) on the full query (order.cpp:367-402);
// backward neighbours are the earlier positions adjacent to each vertex
// (order.cpp:647-676).
OrderRec make_order(const QueryPlan &qp, uint32_t u, uint32_t v) {
  OrderRec r;
  std::memset(&r, 0, sizeof(r));
  uint32_t seen = (1u << u) | (1u << v);
  std::vector<uint32_t> fifo{u, v};
  for (size_t h = 0; h < fifo.size(); ++h) {
    uint32_t top = fifo[h];
    for (uint32_t k = qp.offsets[top]; k < qp.offsets[top + 1]; ++k) {
      uint32_t w = qp.nbrs[k];
      if (!(seen & (1u << w))) {
        seen |= 1u << w;
        fifo.push_back(w);
      }
    }
  }
  for (uint32_t p = 0; p < qp.nq; ++p) {
    r.vert[p] = (uint8_t)fifo[p];
    r.pos_of[fifo[p]] = (uint8_t)p;
  }
  for (uint32_t p = 1; p < qp.nq; ++p)
    for (uint32_t j = 0; j < p; ++j)
      if (qp.adj_mask[fifo[p]] & (1u << fifo[j])) r.bn[p] |= (uint16_t)(1u << j);
  return r;
}

// Tree vertex cover: DP bottom-up, then a LIFO walk that takes a vertex when
// its "taken" cost is no worse, or when its parent was not taken
// (filter.cu:23-116).
std::vector<uint32_t> tree_cover(const QueryPlan &qp) {
  const uint32_t nq = qp.nq;
  uint32_t root = 0;
  for (uint32_t u = 1; u < nq; ++u)
    if (qp.tree_degree[u] > qp.tree_degree[root]) root = u;
  // post-order via an explicit DFS that visits children in CSR order
  std::vector<int> skip(nq, 0), take(nq, 1);
  struct Frame {
    uint32_t v, parent, next;
  };
  std::vector<Frame> st{{root, kNone, qp.tree_offsets[root]}};
  while (!st.empty()) {
    Frame &f = st.back();
    if (f.next < qp.tree_offsets[f.v + 1]) {
      uint32_t c = qp.tree_nbrs[f.next++];
      if (c == f.parent) continue;
      st.push_back({c, f.v, qp.tree_offsets[c]});
      continue;
    }
    uint32_t v = f.v, parent = f.parent;
    st.pop_back();
    skip[v] = 0;
    take[v] = 1;
    for (uint32_t k = qp.tree_offsets[v]; k < qp.tree_offsets[v + 1]; ++k) {
      uint32_t c = qp.tree_nbrs[k];
      if (c == parent) continue;
      skip[v] += take[c];
      take[v] += std::min(skip[c], take[c]);
    }
  }
  std::vector<uint32_t> cover;
  struct Item {
    uint32_t v, parent;
    bool parent_taken;
  };
  std::vector<Item> lifo{{root, kNone, false}};
  while (!lifo.empty()) {
    Item it = lifo.back();
    lifo.pop_back();
    bool taken = (take[it.v] <= skip[it.v]) || !(it.parent_taken || it.parent == kNone);
    if (taken) cover.push_back(it.v);
    for (uint32_t k = qp.tree_offsets[it.v]; k < qp.tree_offsets[it.v + 1]; ++k)
      if (qp.tree_nbrs[k] != it.parent) lifo.push_back({qp.tree_nbrs[k], it.v, taken});
  }
  return cover;
}

// Clustering (filter.cu:131-392) and the encode driver's op order
// (filter.cu:936-1177).
int plan_filter(QueryPlan &qp, std::string &err) {
  std::vector<uint32_t> cover = tree_cover(qp);
  std::vector<std::vector<uint32_t>> cl;
  std::vector<uint8_t> valid(kClusterCap, 1);
  for (uint32_t core : cover) {
    std::vector<uint32_t> c{core};
    for (uint32_t k = qp.tree_offsets[core]; k < qp.tree_offsets[core + 1]; ++k) c.push_back(qp.tree_nbrs[k]);
    cl.push_back(c);
  }
  std::vector<uint32_t> per_layer(kLayerCap, 0), layer_start(kLayerCap, 0);
  std::vector<int> checkpoint(kLayerCap, -1);
  struct Merge {
    uint32_t left, right;
  };
  struct Combine {
    uint32_t out;
    std::vector<uint32_t> smalls;  // ascending
    uint32_t type;
  };
  std::vector<Merge> merges;
  std::vector<Combine> combines;
  uint32_t final_cluster = 0;
  per_layer[0] = (uint32_t)cl.size();
  uint32_t layer = 0, scan_from = 0;
  auto overflow = [&]() {
    err = "query needs more than 150 filter clusters (MAX_CLUSTERS)";
    return DSM_ERR_LIMIT;
  };
  while (true) {
    const uint32_t base = (uint32_t)cl.size();
    // merge every pair of valid clusters of the previous layer that share a
    // leaf of the left one with any member of the right one
    for (uint32_t i = scan_from; i < base; ++i) {
      if (!valid[i]) continue;
      for (uint32_t j = i + 1; j < base; ++j) {
        if (!valid[j]) continue;
        for (size_t ip = 1; ip < cl[i].size(); ++ip)
          for (size_t jp = 0; jp < cl[j].size(); ++jp) {
            if (cl[i][ip] != cl[j][jp]) continue;
            std::vector<uint32_t> m{cl[i][ip], cl[i][0]};
            if (jp != 0 && cl[j][0] != cl[i][0]) m.push_back(cl[j][0]);
            if (cl.size() >= kClusterCap) return overflow();
            final_cluster = (uint32_t)cl.size();
            cl.push_back(m);
            merges.push_back({i, j});
          }
      }
    }
    scan_from = base;
    ++layer;
    if (layer + 1 >= kLayerCap) {
      err = "filter clustering exceeded 100 layers";
      return DSM_ERR_LIMIT;
    }
    long long distinct = (long long)(cl.size() - base);
    checkpoint[layer] = (int)cl.size();
    // combine clusters of this layer that share a core
    for (uint32_t o = base; o < cl.size(); ++o) {
      if (!valid[o]) continue;
      std::vector<uint32_t> group{o};
      std::set<uint32_t> leaves(cl[o].begin() + 1, cl[o].end());
      for (uint32_t in = o + 1; in < cl.size(); ++in)
        if (valid[in] && cl[in][0] == cl[o][0]) {
          group.push_back(in);
          leaves.insert(cl[in].begin() + 1, cl[in].end());
        }
      if (group.size() == 1) continue;
      // the first cluster of the group that already holds every leaf is kept
      auto full = std::find_if(group.begin(), group.end(),
                               [&](uint32_t c) { return cl[c].size() == leaves.size() + 1; });
      Combine cb;
      if (full != group.end()) {
        cb.out = *full;
        cb.type = 1;
        group.erase(full);
      } else {
        if (cl.size() >= kClusterCap) return overflow();
        std::vector<uint32_t> c{cl[o][0]};
        c.insert(c.end(), leaves.begin(), leaves.end());
        cb.out = (uint32_t)cl.size();
        cb.type = 0;
        cl.push_back(c);
        ++distinct;
      }
      cb.smalls = group;
      final_cluster = cb.out;
      distinct -= (long long)group.size();
      for (uint32_t s : group) valid[s] = 0;
      combines.push_back(cb);
    }
    per_layer[layer] = (uint32_t)cl.size() - base;
    if (distinct <= 1) break;
  }
  const uint32_t num_layers = layer + 1;
  for (uint32_t l = 1; l <= layer; ++l) layer_start[l] = layer_start[l - 1] + per_layer[l - 1];
  layer_start[layer + 1] = (uint32_t)cl.size();

  // encoding positions
  std::vector<uint32_t> cpos(cl.size() + 1, 0), members;
  for (size_t c = 0; c < cl.size(); ++c) {
    cpos[c + 1] = cpos[c] + (uint32_t)cl[c].size();
    members.insert(members.end(), cl[c].begin(), cl[c].end());
  }
  qp.enc_positions = cpos.back();
  qp.enc_words = (qp.enc_positions + 31) / 32;

  auto emit_encode = [&](uint32_t c) {
    FilterOp op;
    std::memset(&op, 0, sizeof(op));
    op.kind = FilterOp::kEncode;
    op.core_u = cl[c][0];
    op.pos = cpos[c];
    op.nleaf = (uint32_t)cl[c].size() - 1;
    for (uint32_t i = 0; i < op.nleaf; ++i) op.leaf_u[i] = cl[c][i + 1];
    qp.ops.push_back(op);
  };
  auto find_member = [&](uint32_t from, uint32_t u) {
    while (from < members.size() && members[from] != u) ++from;
    return from;
  };
  auto emit_merge = [&](uint32_t c, const Merge &m) -> int {
    FilterOp op;
    std::memset(&op, 0, sizeof(op));
    op.kind = FilterOp::kMerge;
    op.core_u = cl[c][0];
    op.pos = cpos[c];
    op.nleaf = (uint32_t)cl[c].size() - 1;
    op.left_pos = find_member(cpos[m.left], op.core_u);
    op.right_pos = find_member(cpos[m.right], op.core_u);
    op.left_core_pos = cpos[m.left];
    op.right_core_pos = cpos[m.right];
    if (op.left_pos >= members.size() || op.right_pos >= members.size()) {
      err = "filter merge lost its connection vertex";
      return DSM_ERR_LIMIT;
    }
    qp.ops.push_back(op);
    return 0;
  };
  auto emit_combine = [&](const Combine &cb) -> int {
    if (cb.smalls.size() > 32) {
      err = "filter combine over more than 32 clusters";
      return DSM_ERR_LIMIT;
    }
    FilterOp op;
    std::memset(&op, 0, sizeof(op));
    op.kind = FilterOp::kCombine;
    op.core_u = cl[cb.out][0];
    op.pos = cpos[cb.out];
    op.nleaf = (uint32_t)cl[cb.out].size() - 1;
    op.comb_type = cb.type;
    op.nsmall = (uint32_t)cb.smalls.size();
    std::vector<uint32_t> smalls = cb.smalls;
    std::sort(smalls.begin(), smalls.end());
    for (uint32_t s = 0; s < op.nsmall; ++s) op.small_core_pos[s] = cpos[smalls[s]];
    for (uint32_t i = 0; i < op.nleaf; ++i) {
      uint32_t tu = cl[cb.out][i + 1];
      for (uint32_t s : smalls)
        for (uint32_t p = cpos[s] + 1; p < cpos[s + 1]; ++p)
          if (members[p] == tu) {
            op.leaf_src[i][op.leaf_src_count[i]++] = p;
            break;
          }
    }
    qp.ops.push_back(op);
    return 0;
  };

  // op order of the encode driver
  for (uint32_t c = 0; c < per_layer[0]; ++c) emit_encode(c);
  uint32_t l = 1, layer_sum = per_layer[0];
  size_t ci_merge = 0, ci_comb = 0;
  for (uint32_t c = per_layer[0]; c < cl.size(); ++c) {
    if (c == layer_sum + per_layer[l]) {
      layer_sum += per_layer[l];
      ++l;
      if (l + 1 >= kLayerCap) break;
    }
    if ((int)c == checkpoint[l]) {
      while (ci_comb < combines.size() && combines[ci_comb].out < layer_start[l + 1])
        if (int rc = emit_combine(combines[ci_comb++])) return rc;
      if (c != layer_start[l + 1]) {
        c = layer_start[l + 1] - 1;
        continue;
      }
    }
    if (ci_merge >= merges.size()) {
      err = "filter plan ran out of merges";
      return DSM_ERR_LIMIT;
    }
    if (int rc = emit_merge(c, merges[ci_merge++])) return rc;
  }
  if (checkpoint[num_layers - 1] == (int)cl.size())
    while (ci_comb < combines.size())
      if (int rc = emit_combine(combines[ci_comb++])) return rc;

  // candidacy position of each u: its first occurrence scanning valid
  // clusters from the last one down (filter.cu:1582-1609)
  qp.enc_pos_of_u.assign(qp.nq, kNone);
  uint32_t found = 0;
  for (int c = (int)final_cluster; c >= 0 && found < qp.nq; --c) {
    if (!valid[c]) continue;
    for (uint32_t p = cpos[c]; p < cpos[c + 1]; ++p)
      if (qp.enc_pos_of_u[members[p]] == kNone) {
        qp.enc_pos_of_u[members[p]] = p;
        ++found;
      }
  }
  qp.clusters = cl;
  qp.cluster_valid.assign(valid.begin(), valid.begin() + cl.size());
  return 0;
}

}  // namespace

int plan_query(uint32_t nq, const uint32_t *offsets, const uint32_t *nbrs, const uint32_t *labels,
               QueryPlan &qp, std::string &err) {
  qp = QueryPlan();
  if (nq < 2) {
    err = "a query needs at least one edge";
    return DSM_ERR_LIMIT;
  }
  if (nq > kMaxQueryVertices) {
    err = "query has more than 16 vertices";
    return DSM_ERR_LIMIT;
  }
  if (offsets[0] != 0) {
    err = "query offsets must start at 0";
    return DSM_ERR_ARG;
  }
  qp.nq = nq;
  qp.labels.assign(labels, labels + nq);
  qp.offsets.assign(offsets, offsets + nq + 1);
  qp.nbrs.assign(nbrs, nbrs + offsets[nq]);
  qp.degree.resize(nq);
  qp.adj_mask.assign(nq, 0);
  for (uint32_t u = 0; u < nq; ++u) {
    if (labels[u] >= kMaxLabels) {
      err = "query label >= 32";
      return DSM_ERR_LIMIT;
    }
    if (offsets[u + 1] < offsets[u]) {
      err = "query offsets not monotone";
      return DSM_ERR_ARG;
    }
    qp.degree[u] = offsets[u + 1] - offsets[u];
    for (uint32_t k = offsets[u]; k < offsets[u + 1]; ++k) {
      uint32_t w = nbrs[k];
      if (w >= nq || w == u || (qp.adj_mask[u] & (1u << w))) {
        err = "query has a self loop, a duplicate edge or a bad vertex id";
        return DSM_ERR_ARG;
      }
      qp.adj_mask[u] |= 1u << w;
    }
  }
  for (uint32_t u = 0; u < nq; ++u)
    for (uint32_t w = 0; w < nq; ++w)
      if (((qp.adj_mask[u] >> w) & 1u) != ((qp.adj_mask[w] >> u) & 1u)) {
        err = "query CSR is not symmetric";
        return DSM_ERR_ARG;
      }
  qp.ne = offsets[nq] / 2;
  // connected?
  uint32_t reach = 1, frontier = 1;
  while (frontier) {
    uint32_t next = 0;
    for (uint32_t u = 0; u < nq; ++u)
      if (frontier & (1u << u)) next |= qp.adj_mask[u];
    frontier = next & ~reach;
    reach |= next;
  }
  if (reach != (nq == 32 ? 0xFFFFFFFFu : ((1u << nq) - 1))) {
    err = "query graph is not connected";
    return DSM_ERR_LIMIT;
  }
  spanning_tree(qp);
  for (uint32_t u = 0; u < nq; ++u)
    for (uint32_t k = offsets[u]; k < offsets[u + 1]; ++k) {
      qp.oedges.push_back({u, nbrs[k]});
      qp.orders.push_back(make_order(qp, u, nbrs[k]));
    }
  qp.nlabels = 0;
  for (uint32_t u = 0; u < nq; ++u) qp.nlabels = std::max(qp.nlabels, labels[u] + 1);
  qp.nlc.assign((size_t)nq * 32, 0);
  for (uint32_t u = 0; u < nq; ++u)
    for (uint32_t k = offsets[u]; k < offsets[u + 1]; ++k) qp.nlc[(size_t)u * 32 + labels[nbrs[k]]]++;
  return plan_filter(qp, err);
}

}  // namespace dsm
