// oracle.cpp -- TEST INFRASTRUCTURE ONLY (see oracle.h).
//
// CPU restatement of qxk152/DSM's continuous subgraph matching path, used as
// the checker for the CUDA engine.  Each function cites the reference code it
// restates.  Where the reference has a data race (plain read-modify-write of
// encoding words next to atomicOr from other warps, filter.cu:688, 763, 868,
// 874) or an out-of-bounds shared write (filter.cu:453, s_bitmap[lid][wid]
// with lid up to 31 against a first dimension of MAX_VQ=16), this file
// restates the race-free, in-bounds intent: every bit update is applied as if
// atomic, and only s_bitmap's own 16 rows are cleared.
#include "oracle.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <fstream>
#include <map>
#include <queue>
#include <set>
#include <stack>
#include <string>
#include <vector>

namespace {

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr int kMaxClusters = 150;  // defs.h:22
constexpr int kMaxLayers = 100;    // defs.h:23

// ------------------------------------------------------------------------
// Parsed text file (io.cu:122-252)
// ------------------------------------------------------------------------
struct File {
  uint32_t nv = 0, ne = 0;
  std::vector<uint32_t> labels, offsets, nbrs, edges;
  std::vector<uint32_t> batch_sizes;
  std::vector<uint32_t> updates;  // 4 words each
};

bool parse_file(const char *path, bool is_query, File &g) {
  std::ifstream ifs(path);
  if (!ifs.is_open()) return false;
  char type;
  long long nv, ne;
  if (!(ifs >> type >> nv >> ne) || type != 't' || nv < 0 || ne < 0) return false;
  g.nv = (uint32_t)nv;
  g.ne = (uint32_t)ne;
  g.labels.assign(g.nv, 0);
  g.offsets.assign(g.nv + 1, 0);
  g.nbrs.assign(2 * (size_t)g.ne, 0);
  std::vector<uint32_t> fill(g.nv, 0);
  uint32_t next_v = 0;
  uint64_t edges_seen = 0;
  while (ifs >> type) {
    if (type == 'v') {
      long long vid, lab, deg;
      if (!(ifs >> vid >> lab >> deg)) return false;
      // offsets_[vid+1] = offsets_[vid] + deg needs v-lines in id order.
      if (vid != next_v || lab < 0 || deg < 0) return false;
      g.labels[vid] = (uint32_t)lab;
      g.offsets[vid + 1] = g.offsets[vid] + (uint32_t)deg;
      ++next_v;
    } else if (type == 'e') {
      long long s, d;
      if (!(ifs >> s >> d)) return false;
      if (s < 0 || d < 0 || s >= g.nv || d >= g.nv || edges_seen >= g.ne) return false;
      if (next_v != g.nv) return false;
      uint32_t src = (uint32_t)s, dst = (uint32_t)d;
      if (g.offsets[src] + fill[src] >= g.offsets[src + 1]) return false;
      g.nbrs[g.offsets[src] + fill[src]++] = dst;
      if (g.offsets[dst] + fill[dst] >= g.offsets[dst + 1]) return false;
      g.nbrs[g.offsets[dst] + fill[dst]++] = src;
      g.edges.push_back(src);
      g.edges.push_back(dst);
      ++edges_seen;
    } else if (type == '-') {
      break;
    } else {
      return false;
    }
  }
  if (next_v != g.nv || edges_seen != g.ne || g.offsets[g.nv] != 2 * (uint64_t)g.ne) return false;
  for (uint32_t v = 0; v < g.nv; ++v)
    if (fill[v] != g.offsets[v + 1] - g.offsets[v]) return false;
  if (!is_query) {
    // 'b' bid size, then size x ('a'|'d' src dst label)  (io.cu:216-246)
    std::vector<std::vector<uint32_t>> batches;
    while (ifs >> type) {
      if (type != 'b') continue;  // the reference skips any other token here
      long long bid, bsize;
      if (!(ifs >> bid >> bsize) || bsize < 0) return false;
      batches.emplace_back();
      if (bid < 0 || bid >= (long long)batches.size()) return false;
      g.batch_sizes.push_back((uint32_t)bsize);
      for (long long i = 0; i < bsize; ++i) {
        char op;
        long long s, d, l;
        if (!(ifs >> op >> s >> d >> l)) return false;
        if (op != 'a' && op != 'd') return false;
        if (s < 0 || d < 0 || s >= g.nv || d >= g.nv || l < 0) return false;
        auto &b = batches[bid];
        b.push_back(op == 'a' ? 1u : 0u);
        b.push_back((uint32_t)s);
        b.push_back((uint32_t)d);
        b.push_back((uint32_t)l);
      }
    }
    for (auto &b : batches) g.updates.insert(g.updates.end(), b.begin(), b.end());
  }
  return true;
}

// ------------------------------------------------------------------------
// Query helpers
// ------------------------------------------------------------------------
// True adjacency test on the query.  The reference's is_neighbor
// (order.h:9-27) is a lower_bound that assumes sorted neighbour lists; for
// sorted lists the two agree.
bool q_adjacent(const uint32_t *qoff, const uint32_t *qnbr, uint32_t a, uint32_t b) {
  for (uint32_t k = qoff[a]; k < qoff[a + 1]; ++k)
    if (qnbr[k] == b) return true;
  return false;
}

// decycle.cpp:6-135: BFS spanning tree from the first vertex of maximum
// degree; non-tree edges are dropped (both directions) and degrees fixed.
int decycle_impl(uint32_t nq, const uint32_t *qoff, const uint32_t *qnbr,
                 std::vector<uint32_t> &toff, std::vector<uint32_t> &tnbr,
                 std::vector<uint32_t> &tdeg) {
  // Edge ids: file edge k carries ids 2k (src->dst) and 2k+1 (dst->src).
  // Recover them from the CSR: the j-th occurrence of the unordered pair.
  std::map<std::pair<uint32_t, uint32_t>, uint32_t> vve;
  std::vector<uint32_t> eid(qoff[nq]);
  {
    // Rebuild file order of edges: an edge (s,d) first appears in s's list
    // when the file lists it.  The reference's vve map keys (src,dst) with
    // the first id; ids only matter as undirected pair identities here.
    uint32_t next = 0;
    for (uint32_t a = 0; a < nq; ++a)
      for (uint32_t k = qoff[a]; k < qoff[a + 1]; ++k) {
        uint32_t b = qnbr[k];
        auto key = std::make_pair(std::min(a, b), std::max(a, b));
        auto it = vve.find(key);
        uint32_t base;
        if (it == vve.end()) {
          base = next;
          vve[key] = next;
          next += 2;
        } else {
          base = it->second;
        }
        eid[k] = base + (a < b ? 0 : 1);
      }
  }
  std::vector<uint32_t> deg(nq);
  for (uint32_t u = 0; u < nq; ++u) deg[u] = qoff[u + 1] - qoff[u];
  uint32_t root = 0;
  for (uint32_t u = 1; u < nq; ++u)
    if (deg[u] > deg[root]) root = u;
  std::vector<char> vis(nq, 0), keep(qoff[nq] + 2, 0);
  std::queue<uint32_t> q;
  q.push(root);
  vis[root] = 1;
  while (!q.empty()) {
    uint32_t top = q.front();
    q.pop();
    for (uint32_t k = qoff[top]; k < qoff[top + 1]; ++k) {
      uint32_t nb = qnbr[k];
      if (!vis[nb]) {
        vis[nb] = 1;
        q.push(nb);
        keep[eid[k]] = 1;
      }
    }
  }
  tdeg = deg;
  for (auto &kv : vve) {
    uint32_t e = kv.second;
    if (keep[e] || keep[e + 1]) {
      keep[e] = keep[e + 1] = 1;
    } else {
      tdeg[kv.first.first]--;
      tdeg[kv.first.second]--;
    }
  }
  toff.assign(nq + 1, 0);
  tnbr.clear();
  for (uint32_t u = 0; u < nq; ++u) {
    for (uint32_t k = qoff[u]; k < qoff[u + 1]; ++k)
      if (keep[eid[k]]) tnbr.push_back(qnbr[k]);
    toff[u + 1] = (uint32_t)tnbr.size();
  }
  return (int)(tnbr.size() / 2);
}

// order.cpp:367-402 (getVertexOrderBFS) and 647-676
// (constructBackwardNeighbors), both on the full query.
void order_impl(uint32_t nq, const uint32_t *qoff, const uint32_t *qnbr, uint32_t u,
                uint32_t v, std::vector<uint32_t> &order, std::vector<uint32_t> &bn) {
  order.clear();
  std::vector<char> vis(nq, 0);
  std::queue<uint32_t> q;
  q.push(u);
  vis[u] = 1;
  q.push(v);
  vis[v] = 1;
  while (!q.empty()) {
    uint32_t top = q.front();
    q.pop();
    order.push_back(top);
    for (uint32_t k = qoff[top]; k < qoff[top + 1]; ++k) {
      uint32_t nb = qnbr[k];
      if (!vis[nb]) {
        vis[nb] = 1;
        q.push(nb);
      }
    }
  }
  bn.assign(order.size(), 0);
  for (size_t p = 1; p < order.size(); ++p)
    for (size_t j = 0; j < p; ++j)
      if (q_adjacent(qoff, qnbr, order[p], order[j])) bn[p] |= 1u << j;
}

// ------------------------------------------------------------------------
// Cluster-encoding filter (filter.cu)
// ------------------------------------------------------------------------
struct Csr {
  uint32_t nv;
  const uint32_t *labels, *off, *nbr;
  uint32_t deg(uint32_t v) const { return off[v + 1] - off[v]; }
};

// filter.cu:23-116: minimum vertex cover of the tree by DP, then a top-down
// pick with an explicit stack.
void dfs_cover(uint32_t cur, uint32_t father, std::vector<std::array<int, 2>> &f,
               const std::vector<uint32_t> &toff, const std::vector<uint32_t> &tnbr) {
  f[cur][0] = 0;
  f[cur][1] = 1;
  for (uint32_t k = toff[cur]; k < toff[cur + 1]; ++k) {
    uint32_t nb = tnbr[k];
    if (nb == father) continue;
    dfs_cover(nb, cur, f, toff, tnbr);
    f[cur][0] += f[nb][1];
    f[cur][1] += std::min(f[nb][0], f[nb][1]);
  }
}

std::vector<uint32_t> vertex_cover(uint32_t nq, const std::vector<uint32_t> &toff,
                                   const std::vector<uint32_t> &tnbr,
                                   const std::vector<uint32_t> &tdeg) {
  std::vector<std::array<int, 2>> f(nq, {0, 0});
  uint32_t root = 0;
  for (uint32_t u = 1; u < nq; ++u)
    if (tdeg[u] > tdeg[root]) root = u;
  dfs_cover(root, kInvalid, f, toff, tnbr);
  std::vector<uint32_t> cover;
  struct Item {
    uint32_t v, father;
    bool father_sel;
  };
  std::stack<Item> st;
  st.push({root, kInvalid, false});
  while (!st.empty()) {
    Item it = st.top();
    st.pop();
    bool sel;
    if (f[it.v][1] <= f[it.v][0]) {
      cover.push_back(it.v);
      sel = true;
    } else if (it.father_sel || it.father == kInvalid) {
      sel = false;
    } else {
      cover.push_back(it.v);
      sel = true;
    }
    for (uint32_t k = toff[it.v]; k < toff[it.v + 1]; ++k) {
      uint32_t nb = tnbr[k];
      if (nb == it.father) continue;
      st.push({nb, it.v, sel});
    }
  }
  return cover;
}

struct Plan {
  std::vector<std::vector<uint32_t>> cl;  // clusters; cl[i][0] is the core
  std::vector<char> valid;
  std::vector<uint32_t> per_layer, layer_off;
  std::vector<int> checkpoint;
  std::vector<uint32_t> merge_left, merge_right;
  std::vector<uint32_t> comb_out;
  std::vector<std::set<int>> comb_small;
  std::vector<int> comb_type;
  uint32_t final_cluster = 0, num_layers = 0, num_clusters = 0;
  std::vector<uint32_t> cl_off, compact;
  uint32_t num_blocks = 0;
};

// filter.cu:131-392 (clustering) + structure.cu:113-135 (encodingMeta::init)
int clustering(uint32_t nq, const std::vector<uint32_t> &toff,
               const std::vector<uint32_t> &tnbr, const std::vector<uint32_t> &tdeg, Plan &P) {
  std::vector<uint32_t> cover = vertex_cover(nq, toff, tnbr, tdeg);
  P.cl.assign(kMaxClusters, {});
  P.valid.assign(kMaxClusters, 1);
  P.per_layer.assign(kMaxLayers, 0);
  P.layer_off.assign(kMaxLayers, 0);
  P.checkpoint.assign(kMaxLayers, -1);
  uint32_t nc = (uint32_t)cover.size();
  if (nc > (uint32_t)kMaxClusters) return -2;
  for (uint32_t i = 0; i < nc; ++i) {
    uint32_t core = cover[i];
    P.cl[i].push_back(core);
    for (uint32_t k = toff[core]; k < toff[core + 1]; ++k) P.cl[i].push_back(tnbr[k]);
  }
  uint32_t num_clusters = nc;
  P.per_layer[0] = nc;
  int layer = 0;
  uint32_t i = 0;
  long long actual_new;
  do {
    uint32_t num_new = 0;
    for (; i < num_clusters; ++i) {
      if (!P.valid[i]) continue;
      uint32_t core_i = P.cl[i][0];
      for (uint32_t j = i + 1; j < num_clusters; ++j) {
        if (!P.valid[j]) continue;
        uint32_t core_j = P.cl[j][0];
        for (size_t ip = 1; ip < P.cl[i].size(); ++ip) {
          uint32_t ui = P.cl[i][ip];
          for (size_t jp = 0; jp < P.cl[j].size(); ++jp) {
            if (ui != P.cl[j][jp]) continue;
            ++num_new;
            uint32_t idx = num_clusters + num_new - 1;
            if (idx >= (uint32_t)kMaxClusters) return -2;
            P.final_cluster = idx;
            P.valid[idx] = 1;
            std::vector<uint32_t> nc_us;
            if (jp) {
              nc_us = {ui, core_i};
              if (core_i != core_j) nc_us.push_back(core_j);
            } else {
              nc_us = {ui, core_i};
            }
            P.cl[idx] = nc_us;
            P.merge_left.push_back(i);
            P.merge_right.push_back(j);
          }
        }
      }
    }
    ++layer;
    if (layer + 1 >= kMaxLayers) return -2;
    actual_new = num_new;
    P.checkpoint[layer] = (int)(num_clusters + num_new);
    for (uint32_t out = num_clusters; out < num_clusters + num_new; ++out) {
      if (!P.valid[out]) continue;
      uint32_t core_out = P.cl[out][0];
      bool dup = false;
      std::set<int> S;
      S.insert((int)out);
      std::set<uint32_t> nbrs(P.cl[out].begin() + 1, P.cl[out].end());
      for (uint32_t in = out + 1; in < num_clusters + num_new; ++in) {
        if (!P.valid[in]) continue;
        if (P.cl[in][0] == core_out) {
          dup = true;
          S.insert((int)in);
          nbrs.insert(P.cl[in].begin() + 1, P.cl[in].end());
        }
      }
      if (!dup) continue;
      bool create_new = true;
      auto it = S.begin();
      while (create_new && it != S.end()) {
        if (P.cl[*it].size() == nbrs.size() + 1) create_new = false;
        ++it;
      }
      int largest;
      if (!create_new) {
        --it;
        largest = *it;
        S.erase(largest);
        P.comb_type.push_back(1);
      } else {
        ++num_new;
        ++actual_new;
        P.comb_type.push_back(0);
        uint32_t idx = num_clusters + num_new - 1;
        if (idx >= (uint32_t)kMaxClusters) return -2;
        P.valid[idx] = 1;
        std::vector<uint32_t> us{core_out};
        us.insert(us.end(), nbrs.begin(), nbrs.end());
        P.cl[idx] = us;
        largest = (int)idx;
      }
      P.final_cluster = (uint32_t)largest;
      P.comb_out.push_back((uint32_t)largest);
      P.comb_small.push_back(S);
      actual_new -= (long long)S.size();
      for (int s : S) P.valid[s] = 0;
    }
    num_clusters += num_new;
    P.per_layer[layer] = num_new;
  } while (actual_new > 1);
  if (P.checkpoint[layer] == -1) P.checkpoint[layer] = (int)num_clusters;
  for (int l = 1; l <= layer; ++l) P.layer_off[l] = P.layer_off[l - 1] + P.per_layer[l - 1];
  P.layer_off[layer + 1] = num_clusters;
  P.num_layers = (uint32_t)layer + 1;
  P.num_clusters = num_clusters;
  P.cl.resize(num_clusters);
  P.cl_off.assign(num_clusters + 1, 0);
  for (uint32_t c = 0; c < num_clusters; ++c) {
    P.cl_off[c + 1] = P.cl_off[c] + (uint32_t)P.cl[c].size();
    P.compact.insert(P.compact.end(), P.cl[c].begin(), P.cl[c].end());
  }
  P.num_blocks = (P.cl_off[num_clusters] + 31) / 32;
  return 0;
}

// final position of each u (filter.cu:1582-1609): newest valid cluster
// first, each query vertex at its first position there
std::vector<uint32_t> pick_positions(const Plan &P, uint32_t nq) {
  std::vector<uint32_t> pos_of_u(nq, kInvalid);
  std::vector<char> vis(nq, 0);
  uint32_t cnt = 0;
  for (int cid = (int)P.final_cluster; cid >= 0; --cid) {
    if (!P.valid[cid]) continue;
    if (cnt == nq) break;
    for (uint32_t p = P.cl_off[cid]; p < P.cl_off[cid + 1]; ++p) {
      uint32_t u = P.compact[p];
      if (!vis[u]) {
        vis[u] = 1;
        pos_of_u[u] = p;
        ++cnt;
      }
    }
  }
  return pos_of_u;
}

struct Enc {
  uint32_t nb;
  std::vector<uint32_t> w;
  bool get(uint32_t v, uint32_t pos) const { return (w[(size_t)v * nb + pos / 32] >> (pos % 32)) & 1u; }
  void set(uint32_t v, uint32_t pos) { w[(size_t)v * nb + pos / 32] |= 1u << (pos % 32); }
  void clr(uint32_t v, uint32_t pos) { w[(size_t)v * nb + pos / 32] &= ~(1u << (pos % 32)); }
};

int cluster_filter_impl(uint32_t nq, const uint32_t *qlabels, const uint32_t *qoff,
                        const uint32_t *qnbr, const Csr &G, std::vector<uint32_t> &bitmaps,
                        std::vector<uint32_t> &vcand, std::vector<uint32_t> &pos_of_u,
                        std::vector<uint32_t> &plan_log) {
  if (nq == 0 || nq > 32) return -2;
  // --- LDF + NLF (filter.cu:394-613), full query degrees and NLC.
  uint32_t vlq = 0;
  for (uint32_t u = 0; u < nq; ++u) vlq = std::max(vlq, qlabels[u] + 1);
  if (vlq > 32) return -2;
  std::vector<uint32_t> qnlc((size_t)nq * vlq, 0);
  for (uint32_t u = 0; u < nq; ++u)
    for (uint32_t k = qoff[u]; k < qoff[u + 1]; ++k) qnlc[(size_t)u * vlq + qlabels[qnbr[k]]]++;
  vcand.assign(G.nv, 0);
  std::vector<std::vector<uint32_t>> cand(nq);
  std::vector<uint32_t> dnlc(vlq);
  for (uint32_t v = 0; v < G.nv; ++v) {
    uint32_t lv = G.labels[v];
    if (lv >= vlq) continue;
    std::fill(dnlc.begin(), dnlc.end(), 0);
    for (uint32_t k = G.off[v]; k < G.off[v + 1]; ++k) {
      uint32_t l = G.labels[G.nbr[k]];
      if (l < vlq) dnlc[l]++;
    }
    for (uint32_t u = 0; u < nq; ++u) {
      if (!(qoff[u + 1] - qoff[u] <= G.deg(v) && qlabels[u] == lv)) continue;
      bool ok = true;
      for (uint32_t l = 0; l < vlq; ++l)
        if (dnlc[l] < qnlc[(size_t)u * vlq + l]) ok = false;
      if (ok) {
        vcand[v] |= 1u << u;
        cand[u].push_back(v);
      }
    }
  }
  // --- clustering on the decycled query (filter.cu:131-392)
  std::vector<uint32_t> toff, tnbr, tdeg;
  decycle_impl(nq, qoff, qnbr, toff, tnbr, tdeg);
  Plan P;
  int rc = clustering(nq, toff, tnbr, tdeg, P);
  if (rc) return rc;
  Enc E{P.num_blocks, std::vector<uint32_t>((size_t)G.nv * P.num_blocks, 0)};
  auto log_op = [&](uint32_t kind, uint32_t c, uint32_t a, uint32_t b, uint32_t x, uint32_t y,
                    uint32_t z, uint32_t t) {
    uint32_t rec[8] = {kind, c, a, b, x, y, z, t};
    plan_log.insert(plan_log.end(), rec, rec + 8);
  };
  // encodeKernel (filter.cu:615-717)
  auto op_encode = [&](uint32_t c) {
    uint32_t core = P.cl[c][0], pos = P.cl_off[c];
    log_op(0, c, core, pos, (uint32_t)P.cl[c].size(), 0, 0, 0);
    for (uint32_t v : cand[core]) {
      if (v >= G.nv) continue;
      E.set(v, pos);
      for (uint32_t k = G.off[v]; k < G.off[v + 1]; ++k) {
        uint32_t n = G.nbr[k];
        uint32_t code = vcand[n];
        for (size_t i = 1; i < P.cl[c].size(); ++i)
          if (code & (1u << P.cl[c][i])) E.set(n, pos + (uint32_t)i);
      }
    }
  };
  // mergeKernel (filter.cu:719-803)
  auto op_merge = [&](uint32_t c, uint32_t lp, uint32_t rp, uint32_t lcp, uint32_t rcp) {
    uint32_t core = P.cl[c][0], pos = P.cl_off[c];
    log_op(1, c, core, pos, lp, rp, lcp, rcp);
    for (auto &slot : cand[core]) {
      uint32_t v = slot;
      if (v == kInvalid) continue;
      if (E.get(v, lp) && E.get(v, rp))
        E.set(v, pos);
      else
        slot = kInvalid;
      for (uint32_t k = G.off[v]; k < G.off[v + 1]; ++k) {
        uint32_t n = G.nbr[k];
        if (E.get(n, lcp)) E.set(n, pos + 1);
        if (rcp != rp && E.get(n, rcp)) E.set(n, pos + 2);
      }
    }
  };
  // combineMultipleClustersKernel (filter.cu:805-934)
  auto op_combine = [&](uint32_t k) -> int {
    uint32_t big = P.comb_out[k];
    std::vector<int> smalls(P.comb_small[k].begin(), P.comb_small[k].end());
    if (smalls.size() > 32 || smalls.empty()) return -2;
    int type = P.comb_type[k];
    uint32_t core = P.cl[big][0], bpos = P.cl_off[big];
    log_op(2, big, core, bpos, (uint32_t)type, (uint32_t)smalls.size(), k, 0);
    for (auto &slot : cand[core]) {
      uint32_t v = slot;
      if (v == kInvalid) continue;
      bool all = true;
      for (int s : smalls) all = all && E.get(v, P.cl_off[s]);
      if (all) {
        if (type == 0) E.set(v, bpos);
      } else {
        E.clr(v, bpos);
        slot = kInvalid;
      }
      for (uint32_t e = G.off[v]; e < G.off[v + 1]; ++e) {
        uint32_t n = G.nbr[e];
        for (size_t i = 1; i < P.cl[big].size(); ++i) {
          uint32_t tpos = bpos + (uint32_t)i, tu = P.compact[tpos];
          bool fv = true;
          for (int s : smalls) {
            for (uint32_t p = P.cl_off[s] + 1; p < P.cl_off[s] + P.cl[s].size(); ++p)
              if (P.compact[p] == tu) {
                fv = fv && E.get(n, p);
                break;
              }
          }
          if (type == 1) {
            if (!fv) E.clr(n, tpos);
          } else if (fv) {
            E.set(n, tpos);
          }
        }
      }
    }
    return 0;
  };
  // encode() driver (filter.cu:936-1177)
  for (uint32_t c = 0; c < P.per_layer[0]; ++c) op_encode(c);
  uint32_t layer = 1, sum = P.per_layer[0], cptr = 0, mptr = 0;
  const uint32_t comb_cnt = (uint32_t)P.comb_out.size();
  for (uint32_t ci = P.per_layer[0]; ci < P.num_clusters; ++ci) {
    if (ci == sum + P.per_layer[layer]) {
      sum += P.per_layer[layer];
      ++layer;
      if (layer + 1 >= (uint32_t)kMaxLayers) return -2;
    }
    if ((int)ci == P.checkpoint[layer]) {
      if (comb_cnt != 0) {
        uint32_t next_start = P.layer_off[layer + 1];
        while (cptr < comb_cnt && P.comb_out[cptr] < next_start) {
          if (op_combine(cptr)) return -2;
          ++cptr;
        }
      }
      if (ci != P.layer_off[layer + 1]) {
        ci = P.layer_off[layer + 1] - 1;
        continue;
      }
    }
    if (mptr >= P.merge_left.size()) return -2;
    uint32_t core = P.cl[ci][0];
    uint32_t left = P.merge_left[mptr], right = P.merge_right[mptr];
    uint32_t lp = P.cl_off[left], rp = P.cl_off[right];
    while (lp < P.compact.size() && P.compact[lp] != core) ++lp;
    while (rp < P.compact.size() && P.compact[rp] != core) ++rp;
    if (lp >= P.compact.size() || rp >= P.compact.size()) return -2;
    op_merge(ci, lp, rp, P.cl_off[left], P.cl_off[right]);
    ++mptr;
  }
  if (P.checkpoint[P.num_layers - 1] == (int)P.num_clusters)
    while (cptr < comb_cnt) {
      if (op_combine(cptr)) return -2;
      ++cptr;
    }
  pos_of_u = pick_positions(P, nq);
  // compact (filter.cu:1692-1749): per-u bitmaps over data vertices.
  uint32_t col = (G.nv + 31) / 32;
  bitmaps.assign((size_t)nq * col, 0);
  for (uint32_t u = 0; u < nq; ++u) {
    if (pos_of_u[u] == kInvalid) continue;
    for (uint32_t v = 0; v < G.nv; ++v)
      if (E.get(v, pos_of_u[u])) bitmaps[(size_t)u * col + v / 32] |= 1u << (v % 32);
  }
  return 0;
}

// ------------------------------------------------------------------------
// Continuous matching (main.cu:268-329 seeding, gpu_match.cu:947-1118
// expansion) with per-update sequential semantics.
// ------------------------------------------------------------------------
constexpr uint64_t kIncomplete = 1ull << 63;  // count bit: the search reached the work limit

struct Stream {
  uint32_t nv = 0, nq = 0;
  std::vector<uint32_t> labels;
  std::vector<std::vector<uint32_t>> adj;
  std::vector<uint32_t> qlabels, qoff, qnbr;
  struct Seed {
    uint32_t u, v;
    std::vector<uint32_t> order, bn;
  };
  std::vector<Seed> seeds;  // one per ordered query edge
  std::vector<int8_t> sign;
  std::vector<uint64_t> count;
  std::vector<uint32_t> tuples;
  uint64_t bytes = 0;
  uint64_t work_budget = ~0ull;  // apply() stops enumerating once `bytes` passes this
  uint64_t work_limit = 0;       // per-update search bound (struct Work), 0: none
  uint32_t complete = 0;         // updates of the last apply with full results

  bool has_edge(uint32_t a, uint32_t b) const {
    const auto &l = adj[a];
    return std::binary_search(l.begin(), l.end(), b);
  }
};

// Search bound per update (the engine's DSM_OPT_WORK_LIMIT): the valid
// partial embeddings of 3 or more positions the update's search generates,
// embeddings included, summed over every thread working on the update.  The
// total depends only on graph, query and order, so "total >= limit" is
// exact; counts are flushed to the shared total every 256, and a search that
// sees the total at the limit stops early.
struct Work {
  uint64_t limit = 0;  // 0: no bound
  std::atomic<uint64_t> *total = nullptr;
  uint64_t local = 0;
  bool stop = false;
  bool bump() {  // one more prefix; true: stop searching
    if (!limit) return false;
    if (++local < 256) return false;
    return flush();
  }
  bool flush() {
    if (limit && local) {
      stop = total->fetch_add(local) + local >= limit;
      local = 0;
    } else if (limit) {
      stop = total->load() >= limit;
    }
    return stop;
  }
};

void enumerate(const Stream &S, const Stream::Seed &sd, std::vector<uint32_t> &f, size_t p,
               bool list, uint64_t &cnt, std::vector<uint32_t> &out, uint64_t &bytes, Work &W) {
  const uint32_t nq = S.nq;
  if (bytes > S.work_budget || W.stop) return;
  if (p == nq) {
    ++cnt;
    if (list) {
      size_t base = out.size();
      out.resize(base + nq);
      for (uint32_t k = 0; k < nq; ++k) out[base + sd.order[k]] = f[k];
    }
    bytes += 4ull * (nq + 1);
    return;
  }
  uint32_t u = sd.order[p];
  uint32_t mask = sd.bn[p];
  // pivot: the backward neighbour whose image has the fewest neighbours
  int pivot = -1;
  for (uint32_t j = 0; j < p; ++j)
    if (mask & (1u << j))
      if (pivot < 0 || S.adj[f[j]].size() < S.adj[f[pivot]].size()) pivot = (int)j;
  const auto &plist = S.adj[f[pivot]];
  bytes += 4ull * plist.size();
  for (uint32_t w : plist) {
    bytes += 4;  // label
    if (S.labels[w] != S.qlabels[u]) continue;
    bool ok = true;
    for (uint32_t j = 0; j < p && ok; ++j)
      if (f[j] == w) ok = false;
    for (uint32_t j = 0; j < p && ok; ++j)
      if ((mask & (1u << j)) && (int)j != pivot) {
        bytes += 4;
        if (!S.has_edge(f[j], w)) ok = false;
      }
    if (!ok) continue;
    f[p] = w;
    if (W.bump()) return;
    enumerate(S, sd, f, p + 1, list, cnt, out, bytes, W);
    if (W.stop) return;
  }
}

// Embeddings through edge {a, b} of the current graph.  With S.work_limit,
// a search that reaches the limit returns a partial count with bit 63 set and
// lists nothing.
uint64_t match_edge(const Stream &S, uint32_t a, uint32_t b, bool list, std::vector<uint32_t> &out,
                    uint64_t &bytes) {
  uint64_t cnt = 0;
  std::vector<uint32_t> f(S.nq);
  size_t first = out.size();
  std::atomic<uint64_t> total{0};
  Work W;
  W.limit = S.work_limit;
  W.total = &total;
  for (const auto &sd : S.seeds) {
    if (S.labels[a] != S.qlabels[sd.u] || S.labels[b] != S.qlabels[sd.v]) continue;
    f[0] = a;
    f[1] = b;
    enumerate(S, sd, f, 2, list, cnt, out, bytes, W);
    if (W.stop) break;
  }
  if (W.limit && W.flush()) {
    out.resize(first);
    return cnt | kIncomplete;
  }
  if (list) {
    // canonical order: lexicographic over (f(0), ..., f(nq-1))
    size_t n = (out.size() - first) / S.nq;
    std::vector<uint32_t> idx(n);
    for (size_t i = 0; i < n; ++i) idx[i] = (uint32_t)i;
    const uint32_t *base = out.data() + first;
    const uint32_t w = S.nq;
    std::sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) {
      return std::lexicographical_compare(base + (size_t)x * w, base + (size_t)x * w + w,
                                          base + (size_t)y * w, base + (size_t)y * w + w);
    });
    std::vector<uint32_t> sorted(n * w);
    for (size_t i = 0; i < n; ++i)
      std::copy(base + (size_t)idx[i] * w, base + (size_t)idx[i] * w + w, sorted.begin() + i * w);
    std::copy(sorted.begin(), sorted.end(), out.begin() + first);
  }
  return cnt;
}

// ------------------------------------------------------------------------
// The same per-update matcher on many host threads: updates still apply one
// at a time in stream order; inside one update, the seeds' search trees are
// expanded breadth-first into a frontier of partial embeddings (at least
// 16 per thread), which the threads then expand depth-first.
// ------------------------------------------------------------------------
struct Pool {
  std::vector<std::thread> th;
  std::mutex m;
  std::condition_variable cv, done_cv;
  std::function<void(int)> job;
  uint64_t gen = 0;
  int pending = 0;
  bool stop = false;
  explicit Pool(int n) {
    for (int t = 0; t < n; ++t)
      th.emplace_back([this, t] {
        uint64_t seen = 0;
        for (;;) {
          std::unique_lock<std::mutex> lk(m);
          cv.wait(lk, [&] { return stop || gen != seen; });
          if (stop) return;
          seen = gen;
          lk.unlock();
          job(t);
          lk.lock();
          if (--pending == 0) done_cv.notify_all();
        }
      });
  }
  void run(std::function<void(int)> f) {
    std::unique_lock<std::mutex> lk(m);
    job = std::move(f);
    pending = (int)th.size();
    ++gen;
    cv.notify_all();
    done_cv.wait(lk, [&] { return pending == 0; });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> lk(m);
      stop = true;
    }
    cv.notify_all();
    for (auto &t : th) t.join();
  }
};

struct Partial {
  uint32_t seed;
  uint32_t depth;
  std::array<uint32_t, 16> f;
};

// Children of a partial embedding (one level of enumerate()).
void expand_one(const Stream &S, const Partial &x, std::vector<Partial> &out, Work &W) {
  const Stream::Seed &sd = S.seeds[x.seed];
  const uint32_t p = x.depth, u = sd.order[p], mask = sd.bn[p];
  int pivot = -1;
  for (uint32_t j = 0; j < p; ++j)
    if (mask & (1u << j))
      if (pivot < 0 || S.adj[x.f[j]].size() < S.adj[x.f[pivot]].size()) pivot = (int)j;
  for (uint32_t w : S.adj[x.f[pivot]]) {
    if (S.labels[w] != S.qlabels[u]) continue;
    bool ok = true;
    for (uint32_t j = 0; j < p && ok; ++j)
      if (x.f[j] == w) ok = false;
    for (uint32_t j = 0; j < p && ok; ++j)
      if ((mask & (1u << j)) && (int)j != pivot && !S.has_edge(x.f[j], w)) ok = false;
    if (!ok) continue;
    Partial y = x;
    y.f[p] = w;
    y.depth = p + 1;
    out.push_back(y);
    if (W.bump()) return;
  }
}

uint64_t match_edge_mt(const Stream &S, uint32_t a, uint32_t b, bool list, std::vector<uint32_t> &out,
                       Pool &pool, int nt) {
  std::vector<Partial> front;
  for (uint32_t k = 0; k < S.seeds.size(); ++k) {
    const auto &sd = S.seeds[k];
    if (S.labels[a] != S.qlabels[sd.u] || S.labels[b] != S.qlabels[sd.v]) continue;
    Partial x;
    x.seed = k;
    x.depth = 2;
    x.f[0] = a;
    x.f[1] = b;
    front.push_back(x);
  }
  // breadth-first until there is enough work to share (or leaves are reached)
  uint64_t done_cnt = 0;
  std::vector<uint32_t> done_tuples;
  std::atomic<uint64_t> total{0};
  Work W0;
  W0.limit = S.work_limit;
  W0.total = &total;
  while (!front.empty() && front.size() < (size_t)16 * nt && !W0.stop) {
    std::vector<Partial> next;
    for (const Partial &x : front) {
      if (x.depth == S.nq) {
        ++done_cnt;
        if (list) {
          const auto &sd = S.seeds[x.seed];
          size_t base = done_tuples.size();
          done_tuples.resize(base + S.nq);
          for (uint32_t k = 0; k < S.nq; ++k) done_tuples[base + sd.order[k]] = x.f[k];
        }
        continue;
      }
      expand_one(S, x, next, W0);
      if (W0.stop) break;
    }
    front.swap(next);
  }
  W0.flush();
  std::atomic<size_t> next_task{0};
  std::vector<uint64_t> cnt(nt, 0);
  std::vector<std::vector<uint32_t>> tup(nt);
  if (!W0.stop)
    pool.run([&](int t) {
      std::vector<uint32_t> f(S.nq);
      uint64_t bytes = 0;
      Work W;
      W.limit = S.work_limit;
      W.total = &total;
      for (size_t i; (i = next_task.fetch_add(1)) < front.size() && !W.stop;) {
        const Partial &x = front[i];
        std::copy(x.f.begin(), x.f.begin() + x.depth, f.begin());
        enumerate(S, S.seeds[x.seed], f, x.depth, list, cnt[t], tup[t], bytes, W);
      }
      W.flush();
    });
  uint64_t sum = done_cnt;
  for (int t = 0; t < nt; ++t) sum += cnt[t];
  if (S.work_limit && total.load() >= S.work_limit) return sum | kIncomplete;
  if (list) {
    const size_t first = out.size(), w = S.nq;
    out.insert(out.end(), done_tuples.begin(), done_tuples.end());
    for (int t = 0; t < nt; ++t) out.insert(out.end(), tup[t].begin(), tup[t].end());
    const size_t n = (out.size() - first) / w;
    std::vector<uint32_t> idx(n);
    for (size_t i = 0; i < n; ++i) idx[i] = (uint32_t)i;
    const uint32_t *base = out.data() + first;
    std::sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) {
      return std::lexicographical_compare(base + (size_t)x * w, base + (size_t)x * w + w, base + (size_t)y * w,
                                          base + (size_t)y * w + w);
    });
    std::vector<uint32_t> sorted(n * w);
    for (size_t i = 0; i < n; ++i)
      std::copy(base + (size_t)idx[i] * w, base + (size_t)idx[i] * w + w, sorted.begin() + i * w);
    std::copy(sorted.begin(), sorted.end(), out.begin() + first);
  }
  return sum;
}

void count_all_rec(const Stream &S, const std::vector<uint32_t> &order,
                   const std::vector<uint32_t> &bn, std::vector<uint32_t> &f, size_t p,
                   uint64_t &cnt) {
  if (p == S.nq) {
    ++cnt;
    return;
  }
  uint32_t u = order[p];
  int pivot = -1;
  for (uint32_t j = 0; j < p; ++j)
    if (bn[p] & (1u << j))
      if (pivot < 0 || S.adj[f[j]].size() < S.adj[f[pivot]].size()) pivot = (int)j;
  auto try_w = [&](uint32_t w) {
    if (S.labels[w] != S.qlabels[u]) return;
    for (uint32_t j = 0; j < p; ++j)
      if (f[j] == w) return;
    for (uint32_t j = 0; j < p; ++j)
      if ((bn[p] & (1u << j)) && (int)j != pivot && !S.has_edge(f[j], w)) return;
    f[p] = w;
    count_all_rec(S, order, bn, f, p + 1, cnt);
  };
  if (pivot < 0) {
    for (uint32_t w = 0; w < S.nv; ++w) try_w(w);
  } else {
    for (uint32_t w : S.adj[f[pivot]]) try_w(w);
  }
}

}  // namespace

struct orc_file {
  File f;
};
struct orc_stream {
  Stream s;
  std::unique_ptr<Pool> pool;  // kept between calls (probe is called per update)
  Pool &threads(int n) {
    if (!pool || (int)pool->th.size() != n) pool.reset(new Pool(n));
    return *pool;
  }
};

extern "C" {

int orc_file_parse(const char *path, int is_query, orc_file **out) {
  auto *h = new orc_file();
  if (!parse_file(path, is_query != 0, h->f)) {
    delete h;
    return -1;
  }
  *out = h;
  return 0;
}
void orc_file_free(orc_file *f) { delete f; }
uint32_t orc_file_nv(const orc_file *f) { return f->f.nv; }
uint32_t orc_file_ne(const orc_file *f) { return f->f.ne; }
const uint32_t *orc_file_labels(const orc_file *f) { return f->f.labels.data(); }
const uint32_t *orc_file_offsets(const orc_file *f) { return f->f.offsets.data(); }
const uint32_t *orc_file_nbrs(const orc_file *f) { return f->f.nbrs.data(); }
const uint32_t *orc_file_edges(const orc_file *f) { return f->f.edges.data(); }
uint32_t orc_file_num_batches(const orc_file *f) { return (uint32_t)f->f.batch_sizes.size(); }
const uint32_t *orc_file_batch_sizes(const orc_file *f) { return f->f.batch_sizes.data(); }
uint32_t orc_file_num_updates(const orc_file *f) { return (uint32_t)(f->f.updates.size() / 4); }
const uint32_t *orc_file_updates(const orc_file *f) { return f->f.updates.data(); }

int orc_decycle(uint32_t nq, const uint32_t *qoff, const uint32_t *qnbr, uint32_t *tree_off,
                uint32_t *tree_nbr, uint32_t *tree_deg) {
  std::vector<uint32_t> toff, tnbr, tdeg;
  int n = decycle_impl(nq, qoff, qnbr, toff, tnbr, tdeg);
  std::copy(toff.begin(), toff.end(), tree_off);
  std::copy(tnbr.begin(), tnbr.end(), tree_nbr);
  std::copy(tdeg.begin(), tdeg.end(), tree_deg);
  return n;
}

int orc_order(uint32_t nq, const uint32_t *qoff, const uint32_t *qnbr, uint32_t u, uint32_t v,
              uint32_t *order, uint32_t *bn_mask) {
  std::vector<uint32_t> o, bn;
  order_impl(nq, qoff, qnbr, u, v, o, bn);
  if (o.size() != nq) return -1;  // disconnected query
  std::copy(o.begin(), o.end(), order);
  std::copy(bn.begin(), bn.end(), bn_mask);
  return 0;
}

int orc_cluster_filter(uint32_t nq, const uint32_t *qlabels, const uint32_t *qoff,
                       const uint32_t *qnbr, uint32_t nv, const uint32_t *labels,
                       const uint32_t *off, const uint32_t *nbr, uint32_t *bitmaps,
                       uint32_t *v_cand_us, uint32_t *enc_pos_of_u, uint32_t *plan_out,
                       uint32_t *plan_len_out) {
  Csr G{nv, labels, off, nbr};
  std::vector<uint32_t> bm, vc, pos, plan;
  int rc = cluster_filter_impl(nq, qlabels, qoff, qnbr, G, bm, vc, pos, plan);
  if (rc) return rc;
  if (bitmaps) std::copy(bm.begin(), bm.end(), bitmaps);
  if (v_cand_us) std::copy(vc.begin(), vc.end(), v_cand_us);
  if (enc_pos_of_u) std::copy(pos.begin(), pos.end(), enc_pos_of_u);
  if (plan_out) std::copy(plan.begin(), plan.begin() + std::min<size_t>(plan.size(), 4096), plan_out);
  if (plan_len_out) *plan_len_out = (uint32_t)(plan.size() / 8);
  return 0;
}

int orc_cluster_plan(uint32_t nq, const uint32_t *qoff, const uint32_t *qnbr, uint32_t *out, uint32_t cap) {
  if (nq == 0 || nq > 32) return -2;
  std::vector<uint32_t> toff, tnbr, tdeg;
  decycle_impl(nq, qoff, qnbr, toff, tnbr, tdeg);
  Plan P;
  if (int rc = clustering(nq, toff, tnbr, tdeg, P)) return rc;
  std::vector<uint32_t> w{P.num_clusters, P.final_cluster, (uint32_t)P.merge_left.size(),
                          (uint32_t)P.comb_out.size(), P.num_layers};
  for (uint32_t c = 0; c < P.num_clusters; ++c) {
    w.push_back(P.valid[c] ? 1 : 0);
    w.push_back((uint32_t)P.cl[c].size());
    w.insert(w.end(), P.cl[c].begin(), P.cl[c].end());
  }
  for (size_t k = 0; k < P.merge_left.size(); ++k) {
    w.push_back(P.merge_left[k]);
    w.push_back(P.merge_right[k]);
  }
  for (size_t k = 0; k < P.comb_out.size(); ++k) {
    w.push_back(P.comb_out[k]);
    w.push_back((uint32_t)P.comb_type[k]);
    w.push_back((uint32_t)P.comb_small[k].size());
    for (int o : P.comb_small[k]) w.push_back((uint32_t)o);
  }
  for (uint32_t l = 0; l <= P.num_layers; ++l) w.push_back(P.layer_off[l]);
  std::vector<uint32_t> pos = pick_positions(P, nq);
  w.insert(w.end(), pos.begin(), pos.end());
  if (w.size() > cap) return -3;
  std::copy(w.begin(), w.end(), out);
  return (int)w.size();
}

int orc_stream_new(uint32_t nv, const uint32_t *labels, uint64_t ne, const uint32_t *edges,
                   uint32_t nq, const uint32_t *qlabels, const uint32_t *qoff,
                   const uint32_t *qnbr, orc_stream **out) {
  if (nq < 2 || nq > 32) return -2;
  auto *h = new orc_stream();
  Stream &S = h->s;
  S.nv = nv;
  S.nq = nq;
  S.labels.assign(labels, labels + nv);
  S.adj.assign(nv, {});
  for (uint64_t k = 0; k < ne; ++k) {
    uint32_t a = edges[2 * k], b = edges[2 * k + 1];
    if (a == b || a >= nv || b >= nv) continue;
    S.adj[a].push_back(b);
    S.adj[b].push_back(a);
  }
  for (auto &l : S.adj) {
    std::sort(l.begin(), l.end());
    l.erase(std::unique(l.begin(), l.end()), l.end());
  }
  S.qlabels.assign(qlabels, qlabels + nq);
  S.qoff.assign(qoff, qoff + nq + 1);
  S.qnbr.assign(qnbr, qnbr + qoff[nq]);
  for (uint32_t u = 0; u < nq; ++u)
    for (uint32_t k = qoff[u]; k < qoff[u + 1]; ++k) {
      Stream::Seed sd;
      sd.u = u;
      sd.v = qnbr[k];
      order_impl(nq, qoff, qnbr, sd.u, sd.v, sd.order, sd.bn);
      if (sd.order.size() != nq) {
        delete h;
        return -1;
      }
      S.seeds.push_back(sd);
    }
  *out = h;
  return 0;
}

void orc_stream_free(orc_stream *s) { delete s; }

int orc_stream_apply(orc_stream *h, uint32_t n, const uint32_t *ups, int list) {
  Stream &S = h->s;
  S.sign.assign(n, 0);
  S.count.assign(n, 0);
  S.tuples.clear();
  S.bytes = 0;
  S.complete = n;
  bool skipping = false;
  for (uint32_t i = 0; i < n; ++i) {
    if (!skipping && S.bytes > S.work_budget) {
      // out of budget: update i onward change the graph without enumeration
      skipping = true;
      S.complete = i;
    }
    if (skipping) {
      uint32_t op = ups[4 * i], a = ups[4 * i + 1], b = ups[4 * i + 2];
      if (a >= S.nv || b >= S.nv) return -1;
      if (a == b) continue;
      bool present = S.has_edge(a, b);
      auto &la = S.adj[a], &lb = S.adj[b];
      if (op == 1 && !present) {
        la.insert(std::lower_bound(la.begin(), la.end(), b), b);
        lb.insert(std::lower_bound(lb.begin(), lb.end(), a), a);
        S.sign[i] = 1;
      } else if (op == 0 && present) {
        la.erase(std::lower_bound(la.begin(), la.end(), b));
        lb.erase(std::lower_bound(lb.begin(), lb.end(), a));
        S.sign[i] = -1;
      }
      continue;
    }
    uint32_t op = ups[4 * i], a = ups[4 * i + 1], b = ups[4 * i + 2];
    if (a >= S.nv || b >= S.nv) return -1;
    if (a == b) continue;  // a self loop never lies on an embedding
    bool present = S.has_edge(a, b);
    S.bytes += 8ull * (S.adj[a].size() + S.adj[b].size());
    if (op == 1) {
      if (present) continue;
      auto &la = S.adj[a], &lb = S.adj[b];
      la.insert(std::lower_bound(la.begin(), la.end(), b), b);
      lb.insert(std::lower_bound(lb.begin(), lb.end(), a), a);
      S.sign[i] = 1;
      S.count[i] = match_edge(S, a, b, list != 0, S.tuples, S.bytes);
    } else {
      if (!present) continue;
      S.sign[i] = -1;
      S.count[i] = match_edge(S, a, b, list != 0, S.tuples, S.bytes);
      auto &la = S.adj[a], &lb = S.adj[b];
      la.erase(std::lower_bound(la.begin(), la.end(), b));
      lb.erase(std::lower_bound(lb.begin(), lb.end(), a));
    }
    if (S.bytes > S.work_budget && !skipping) {
      skipping = true;  // update i's own count may be partial
      S.complete = i;
    }
  }
  if (S.complete < n && list) {
    // drop tuples of updates past the complete prefix
    uint64_t keep = 0;
    for (uint32_t i = 0; i < S.complete; ++i)
      if (!(S.count[i] & kIncomplete)) keep += S.count[i];  // over the work limit: nothing listed
    S.tuples.resize(keep * S.nq);
  }
  for (uint32_t i = S.complete; i < n; ++i) S.count[i] = 0;
  return S.complete < n ? 1 : 0;
}

int orc_stream_apply_mt(orc_stream *h, uint32_t n, const uint32_t *ups, int list, int threads) {
  Stream &S = h->s;
  if (threads < 1) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  Pool &pool = h->threads(threads);
  S.sign.assign(n, 0);
  S.count.assign(n, 0);
  S.tuples.clear();
  S.complete = n;
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t op = ups[4 * i], a = ups[4 * i + 1], b = ups[4 * i + 2];
    if (a >= S.nv || b >= S.nv) return -1;
    if (a == b) continue;
    bool present = S.has_edge(a, b);
    auto &la = S.adj[a], &lb = S.adj[b];
    if (op == 1) {
      if (present) continue;
      la.insert(std::lower_bound(la.begin(), la.end(), b), b);
      lb.insert(std::lower_bound(lb.begin(), lb.end(), a), a);
      S.sign[i] = 1;
      S.count[i] = match_edge_mt(S, a, b, list != 0, S.tuples, pool, threads);
    } else {
      if (!present) continue;
      S.sign[i] = -1;
      S.count[i] = match_edge_mt(S, a, b, list != 0, S.tuples, pool, threads);
      la.erase(std::lower_bound(la.begin(), la.end(), b));
      lb.erase(std::lower_bound(lb.begin(), lb.end(), a));
    }
  }
  return 0;
}

int orc_stream_apply_graph(orc_stream *h, uint32_t n, const uint32_t *ups) {
  Stream &S = h->s;
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t op = ups[4 * i], a = ups[4 * i + 1], b = ups[4 * i + 2];
    if (a >= S.nv || b >= S.nv) return -1;
    if (a == b) continue;
    bool present = S.has_edge(a, b);
    auto &la = S.adj[a], &lb = S.adj[b];
    if (op == 1 && !present) {
      la.insert(std::lower_bound(la.begin(), la.end(), b), b);
      lb.insert(std::lower_bound(lb.begin(), lb.end(), a), a);
    } else if (op == 0 && present) {
      la.erase(std::lower_bound(la.begin(), la.end(), b));
      lb.erase(std::lower_bound(lb.begin(), lb.end(), a));
    }
  }
  return 0;
}

int orc_stream_set_query(orc_stream *h, uint32_t nq, const uint32_t *qlabels, const uint32_t *qoff,
                         const uint32_t *qnbr) {
  if (nq < 2 || nq > 16) return -2;
  Stream &S = h->s;
  std::vector<Stream::Seed> seeds;
  for (uint32_t u = 0; u < nq; ++u)
    for (uint32_t k = qoff[u]; k < qoff[u + 1]; ++k) {
      Stream::Seed sd;
      sd.u = u;
      sd.v = qnbr[k];
      order_impl(nq, qoff, qnbr, sd.u, sd.v, sd.order, sd.bn);
      if (sd.order.size() != nq) return -1;
      seeds.push_back(sd);
    }
  S.nq = nq;
  S.qlabels.assign(qlabels, qlabels + nq);
  S.qoff.assign(qoff, qoff + nq + 1);
  S.qnbr.assign(qnbr, qnbr + qoff[nq]);
  S.seeds.swap(seeds);
  return 0;
}

uint64_t orc_stream_probe(orc_stream *h, uint32_t op, uint32_t a, uint32_t b, int threads) {
  Stream &S = h->s;
  if (a >= S.nv || b >= S.nv || a == b) return 0;
  if (threads < 1) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  const bool present = S.has_edge(a, b);
  if (op == 1 && present) return 0;
  if (op != 1 && !present) return 0;
  auto &la = S.adj[a], &lb = S.adj[b];
  if (op == 1) {
    la.insert(std::lower_bound(la.begin(), la.end(), b), b);
    lb.insert(std::lower_bound(lb.begin(), lb.end(), a), a);
  }
  std::vector<uint32_t> none;
  const uint64_t c = match_edge_mt(S, a, b, false, none, h->threads(threads), threads);
  if (op == 1) {
    la.erase(std::lower_bound(la.begin(), la.end(), b));
    lb.erase(std::lower_bound(lb.begin(), lb.end(), a));
  }
  return c;
}

void orc_stream_set_budget(orc_stream *h, uint64_t bytes) { h->s.work_budget = bytes; }
void orc_stream_set_work_limit(orc_stream *h, uint64_t limit) { h->s.work_limit = limit; }
uint32_t orc_stream_complete(const orc_stream *h) { return h->s.complete; }

int8_t orc_stream_sign(const orc_stream *s, uint32_t i) { return s->s.sign[i]; }
uint64_t orc_stream_count(const orc_stream *s, uint32_t i) { return s->s.count[i]; }
const uint32_t *orc_stream_tuples(const orc_stream *s, uint64_t *num) {
  *num = s->s.tuples.size() / s->s.nq;
  return s->s.tuples.data();
}
uint64_t orc_stream_bytes(const orc_stream *s) { return s->s.bytes; }

uint64_t orc_stream_count_all(const orc_stream *h) {
  const Stream &S = h->s;
  // BFS order from query vertex 0; backward neighbours on the full query.
  std::vector<uint32_t> order;
  std::vector<char> vis(S.nq, 0);
  std::queue<uint32_t> q;
  q.push(0);
  vis[0] = 1;
  while (!q.empty()) {
    uint32_t t = q.front();
    q.pop();
    order.push_back(t);
    for (uint32_t k = S.qoff[t]; k < S.qoff[t + 1]; ++k)
      if (!vis[S.qnbr[k]]) {
        vis[S.qnbr[k]] = 1;
        q.push(S.qnbr[k]);
      }
  }
  if (order.size() != S.nq) return 0;
  std::vector<uint32_t> bn(S.nq, 0);
  for (size_t p = 1; p < S.nq; ++p)
    for (size_t j = 0; j < p; ++j)
      if (q_adjacent(S.qoff.data(), S.qnbr.data(), order[p], order[j])) bn[p] |= 1u << j;
  uint64_t cnt = 0;
  std::vector<uint32_t> f(S.nq);
  count_all_rec(S, order, bn, f, 0, cnt);
  return cnt;
}

uint64_t orc_stream_export(const orc_stream *h, uint32_t *off, uint32_t *nbr) {
  const Stream &S = h->s;
  uint64_t k = 0;
  for (uint32_t v = 0; v < S.nv; ++v) {
    if (off) off[v] = (uint32_t)k;
    for (uint32_t w : S.adj[v]) {
      if (nbr) nbr[k] = w;
      ++k;
    }
  }
  if (off) off[S.nv] = (uint32_t)k;
  return k;
}

uint64_t orc_bruteforce_count(uint32_t nq, const uint32_t *qlabels, const uint32_t *qoff,
                              const uint32_t *qnbr, uint32_t nv, const uint32_t *labels,
                              const uint32_t *off, const uint32_t *nbr) {
  // Every assignment in lexicographic order; injectivity and labels are
  // checked as it grows, every query edge at the end.
  std::vector<uint32_t> f(nq, 0);
  uint64_t cnt = 0;
  auto edge = [&](uint32_t a, uint32_t b) {
    for (uint32_t k = off[a]; k < off[a + 1]; ++k)
      if (nbr[k] == b) return true;
    return false;
  };
  std::vector<uint32_t> stackv(nq + 1, 0);
  size_t p = 0;
  stackv[0] = 0;
  while (true) {
    if (p == nq) {
      bool ok = true;
      for (uint32_t u = 0; u < nq && ok; ++u)
        for (uint32_t k = qoff[u]; k < qoff[u + 1] && ok; ++k)
          if (!edge(f[u], f[qnbr[k]])) ok = false;
      if (ok) ++cnt;
      if (p == 0) break;
      --p;
      stackv[p]++;
      continue;
    }
    uint32_t w = stackv[p];
    if (w >= nv) {
      if (p == 0) break;
      --p;
      stackv[p]++;
      continue;
    }
    bool ok = labels[w] == qlabels[p];
    for (size_t j = 0; j < p && ok; ++j)
      if (f[j] == w) ok = false;
    if (!ok) {
      stackv[p]++;
      continue;
    }
    f[p] = w;
    ++p;
    stackv[p] = 0;
  }
  return cnt;
}

}  // extern "C"
