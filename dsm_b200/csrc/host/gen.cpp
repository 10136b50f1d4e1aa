// Seeded synthetic workloads for continuous subgraph matching.
//
// The reference's dataset (an "amazon-dyna" stream, named in run.sh:3) is not
// available, so every workload is generated: a data graph (R-MAT or
// Chung-Lu), vertex labels (uniform or Zipf), random-walk queries whose labels
// are copied from the data graph, and an update stream whose insertions come
// from a withheld pool of edges and whose deletions pick live edges.
//
// Determinism: std::mt19937_64 streams with hand-written samplers (no
// std::*_distribution, whose output differs between standard libraries).
#include "dsm_host.h"
#include "par.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <random>
#include <thread>
#include <unordered_set>

namespace dsm {

namespace {

struct Rng {
  std::mt19937_64 g;
  explicit Rng(uint64_t seed) : g(seed) {}
  uint64_t u64() { return g(); }
  // uniform in [0, 1) with 53 random bits
  double unit() { return (double)(g() >> 11) * (1.0 / 9007199254740992.0); }
  // uniform integer in [0, n) by rejection (no modulo bias)
  uint64_t below(uint64_t n) {
    if (n <= 1) return 0;
    uint64_t lim = UINT64_MAX - UINT64_MAX % n;
    uint64_t x;
    do x = g(); while (x >= lim);
    return x % n;
  }
};

inline uint64_t edge_key(uint32_t a, uint32_t b) {
  if (a > b) std::swap(a, b);
  return ((uint64_t)a << 32) | b;
}

template <class T>
void shuffle(std::vector<T> &v, Rng &r) {
  for (size_t i = v.size(); i > 1; --i) std::swap(v[i - 1], v[r.below(i)]);
}

// Sample from a discrete CDF (cdf.back() == total) by binary search.
uint32_t sample_cdf(const std::vector<double> &cdf, Rng &r) {
  double x = r.unit() * cdf.back();
  size_t k = std::upper_bound(cdf.begin(), cdf.end(), x) - cdf.begin();
  return (uint32_t)std::min(k, cdf.size() - 1);
}

// Distinct undirected edges without self loops until `m` are found, then a
// seeded shuffle fixes their order.  Graphs of up to 2^25 edges draw from
// the one generator in sequence.  Larger ones draw each round in fixed chunks
// of 2^20 edges, chunk c with its own generator seeded from the round's seed
// and c, so the chunks run on all host threads and the result does not
// depend on the thread count.
template <class Draw>
std::vector<uint64_t> distinct_edges(uint64_t m, Rng &r, Draw draw) {
  std::vector<uint64_t> keys;
  keys.reserve(m + m / 4);
  constexpr size_t kGrain = 1u << 20;
  if (m <= (1ull << 25)) {
    while (keys.size() < m) {
      const uint64_t need = m - keys.size();
      const uint64_t batch = need + need / 8 + 1024;
      for (uint64_t k = 0; k < batch; ++k) {
        uint32_t a, b;
        draw(r, a, b);
        if (a != b) keys.push_back(edge_key(a, b));
      }
      parallel_sort(keys);
      keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    }
  }
  while (keys.size() < m) {
    const uint64_t need = m - keys.size();
    const uint64_t batch = need + need / 8 + 1024;
    const uint64_t round_seed = r.u64();
    const size_t nchunks = (batch + kGrain - 1) / kGrain;
    std::vector<std::vector<uint64_t>> part(nchunks);
    parallel_chunks(nchunks, [&](size_t c) {
      Rng rc(round_seed ^ (0x9E3779B97F4A7C15ull * (c + 1)));
      const uint64_t lo = c * kGrain, hi = std::min<uint64_t>(batch, lo + kGrain);
      part[c].reserve(hi - lo);
      for (uint64_t k = lo; k < hi; ++k) {
        uint32_t a, b;
        draw(rc, a, b);
        if (a != b) part[c].push_back(edge_key(a, b));
      }
    });
    for (auto &pc : part) keys.insert(keys.end(), pc.begin(), pc.end());
    parallel_sort(keys);
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  }
  shuffle(keys, r);
  keys.resize(m);
  return keys;
}

void relabel_ids(std::vector<uint64_t> &keys, uint32_t nv, Rng &r) {
  std::vector<uint32_t> perm(nv);
  for (uint32_t i = 0; i < nv; ++i) perm[i] = i;
  shuffle(perm, r);
  parallel_for(keys.size(), 1u << 20, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i) keys[i] = edge_key(perm[keys[i] >> 32], perm[(uint32_t)keys[i]]);
  });
}

std::vector<uint64_t> gen_rmat(uint32_t log2_nv, uint64_t m, double a, double b, double c,
                               Rng &r) {
  const double ab = a + b, abc = a + b + c;
  auto draw = [&](Rng &rr, uint32_t &s, uint32_t &d) {
    s = d = 0;
    for (uint32_t l = 0; l < log2_nv; ++l) {
      double x = rr.unit();
      uint32_t bs = 0, bd = 0;
      if (x < a) {
      } else if (x < ab) {
        bd = 1;
      } else if (x < abc) {
        bs = 1;
      } else {
        bs = bd = 1;
      }
      s = (s << 1) | bs;
      d = (d << 1) | bd;
    }
  };
  auto keys = distinct_edges(m, r, draw);
  relabel_ids(keys, 1u << log2_nv, r);
  return keys;
}

// Chung-Lu: expected degrees w_i ~ (i+1)^(-1/(gamma-1)), scaled to mean 2m/n
// and capped at sqrt(sum w) (the model's admissibility bound); endpoints are
// drawn in proportion to w.
std::vector<uint64_t> gen_chung_lu(uint32_t nv, uint64_t m, double gamma, Rng &r) {
  std::vector<double> w(nv);
  double sum = 0;
  for (uint32_t i = 0; i < nv; ++i) sum += w[i] = std::pow((double)i + 1.0, -1.0 / (gamma - 1.0));
  double scale = 2.0 * (double)m / sum;
  double cap = std::sqrt(2.0 * (double)m);
  std::vector<double> cdf(nv);
  double acc = 0;
  for (uint32_t i = 0; i < nv; ++i) {
    acc += std::min(w[i] * scale, cap);
    cdf[i] = acc;
  }
  auto draw = [&](Rng &rr, uint32_t &s, uint32_t &d) {
    s = sample_cdf(cdf, rr);
    d = sample_cdf(cdf, rr);
  };
  auto keys = distinct_edges(m, r, draw);
  relabel_ids(keys, nv, r);
  return keys;
}

std::vector<uint32_t> gen_labels(uint32_t nv, uint32_t nl, double zipf_s, Rng &r) {
  std::vector<uint32_t> lab(nv);
  if (zipf_s <= 0) {
    for (auto &l : lab) l = (uint32_t)r.below(nl);
    return lab;
  }
  std::vector<double> cdf(nl);
  double acc = 0;
  for (uint32_t k = 0; k < nl; ++k) cdf[k] = acc += std::pow((double)k + 1.0, -zipf_s);
  for (auto &l : lab) l = sample_cdf(cdf, r);
  return lab;
}

struct Adj {
  std::vector<uint64_t> off;
  std::vector<uint32_t> nbr;
  bool has(uint32_t a, uint32_t b) const {
    return std::binary_search(nbr.begin() + off[a], nbr.begin() + off[a + 1], b);
  }
  uint32_t deg(uint32_t v) const { return (uint32_t)(off[v + 1] - off[v]); }
};

Adj build_adj(uint32_t nv, const std::vector<uint64_t> &keys) {
  Adj g;
  g.off.assign(nv + 1, 0);
  for (uint64_t k : keys) {
    g.off[(k >> 32) + 1]++;
    g.off[(uint32_t)k + 1]++;
  }
  for (uint32_t v = 0; v < nv; ++v) g.off[v + 1] += g.off[v];
  g.nbr.resize(g.off[nv]);
  std::vector<uint64_t> pos(g.off.begin(), g.off.end() - 1);
  for (uint64_t k : keys) {
    uint32_t a = (uint32_t)(k >> 32), b = (uint32_t)k;
    g.nbr[pos[a]++] = b;
    g.nbr[pos[b]++] = a;
  }
  parallel_for(nv, 1u << 14, [&](size_t lo, size_t hi) {
    for (size_t v = lo; v < hi; ++v) std::sort(g.nbr.begin() + g.off[v], g.nbr.begin() + g.off[v + 1]);
  });
  return g;
}

// Embeddings of query q that map some query edge onto data edge (a, b),
// counted by backtracking and capped at `cap` (returns cap when reached).
uint64_t capped_edge_count(const Adj &g, const std::vector<uint32_t> &labels, const Query &q, uint32_t a,
                           uint32_t b, uint64_t cap) {
  const uint32_t nq = q.nv;
  uint64_t cnt = 0, steps = 0;
  std::vector<uint32_t> f(nq);
  for (uint32_t u = 0; u < nq && cnt < cap; ++u)
    for (uint32_t k = q.offsets[u]; k < q.offsets[u + 1] && cnt < cap; ++k) {
      uint32_t v = q.nbrs[k];
      if (labels[a] != q.labels[u] || labels[b] != q.labels[v]) continue;
      // BFS order from (u, v) and backward-neighbour masks
      std::vector<uint32_t> ord{u, v};
      uint32_t seen = (1u << u) | (1u << v);
      for (size_t h = 0; h < ord.size(); ++h)
        for (uint32_t j = q.offsets[ord[h]]; j < q.offsets[ord[h] + 1]; ++j)
          if (!(seen & (1u << q.nbrs[j]))) {
            seen |= 1u << q.nbrs[j];
            ord.push_back(q.nbrs[j]);
          }
      std::vector<uint32_t> pos(nq), bn(nq, 0);
      for (uint32_t p = 0; p < nq; ++p) pos[ord[p]] = p;
      for (uint32_t p = 2; p < nq; ++p)
        for (uint32_t j = q.offsets[ord[p]]; j < q.offsets[ord[p] + 1]; ++j)
          if (pos[q.nbrs[j]] < p) bn[p] |= 1u << pos[q.nbrs[j]];
      f[0] = a;
      f[1] = b;
      // iterative DFS over positions 2..nq-1
      std::vector<uint64_t> it(nq, 0);
      uint32_t p = 2;
      if (nq == 2) {
        ++cnt;
        continue;
      }
      auto pivot_of = [&](uint32_t pp) {
        uint32_t best = 0xFFFFFFFFu, bd = 0xFFFFFFFFu;
        for (uint32_t j = 0; j < pp; ++j)
          if ((bn[pp] >> j) & 1u)
            if (g.deg(f[j]) < bd) bd = g.deg(f[j]), best = j;
        return best;
      };
      it[2] = 0;
      while (p >= 2 && cnt < cap) {
        uint32_t pv = pivot_of(p);
        uint32_t x = f[pv];
        bool advanced = false;
        while (it[p] < g.deg(x)) {
          // dead-end search counts too: past 32 x cap candidates examined,
          // the edge is reported at the cap
          if (++steps > 32 * cap) {
            cnt = cap;
            break;
          }
          uint32_t w = g.nbr[g.off[x] + it[p]++];
          if (labels[w] != q.labels[ord[p]]) continue;
          bool ok = true;
          for (uint32_t j = 0; j < p && ok; ++j)
            if (f[j] == w || (((bn[p] >> j) & 1u) && j != pv && !g.has(f[j], w))) ok = false;
          if (!ok) continue;
          f[p] = w;
          if (p + 1 == nq) {
            if (++cnt >= cap) break;
            continue;
          }
          ++p;
          it[p] = 0;
          advanced = true;
          break;
        }
        if (!advanced && cnt < cap) --p;
      }
    }
  return std::min(cnt, cap);
}

// Random-walk query: a walk from a random vertex adds each newly reached
// vertex with the walk edge that reached it (a spanning tree), then `extra`
// further edges are drawn from the data edges induced on the sampled
// vertices.  Labels are copied.  Returns false when no sample was found.
//
// With max_mean > 0 a sample must also be selective enough to be listed:
// on a power-law graph a tree-like query through two hubs has ~deg^k
// embeddings per update, which no engine can list.  The test counts the
// embeddings through each probe edge (the workload's own update edges, in
// random order), each capped at 10 x max_mean; a candidate passes when no
// edge reaches the cap and the mean stays within max_mean.  Candidates are
// drawn in tiers: tier t walks only over vertices whose label is not among
// the t most frequent labels (the walk stays put when the step would leave
// the allowed vertices), so later tiers copy rarer labels.  Each tier tries
// kPerTier candidates; if no tier passes, the candidate with the smallest
// capped total is returned.
bool sample_query(const Adj &g, const std::vector<uint32_t> &labels, const std::vector<uint32_t> &label_rank,
                  const std::vector<uint64_t> &probe, uint32_t nq, uint32_t extra, double max_mean, Rng &r,
                  Query &q) {
  const uint32_t nv = (uint32_t)labels.size();
  const bool selective = max_mean > 0 && !probe.empty();
  constexpr int kPerTier = 64;
  const uint32_t nlabels = (uint32_t)label_rank.size();
  const uint32_t tiers = selective ? std::max<uint32_t>(1, nlabels > 3 ? nlabels - 3 : 1) : 1;
  double best_total = 1e300;
  Query best;
  for (uint32_t tier = 0; tier < tiers; ++tier) {
    auto allowed = [&](uint32_t v) { return label_rank[labels[v]] >= tier; };
    int scored = 0;
    for (int attempt = 0; attempt < 20000 && scored < kPerTier; ++attempt) {
      // dense shapes need the dense part of the graph: those walks start at
      // the end of a uniformly drawn edge (degree-biased), the others at a
      // uniformly drawn vertex
      uint32_t start = extra * 2 > nq ? g.nbr[r.below(g.nbr.size())] : (uint32_t)r.below(nv);
      if (g.deg(start) == 0 || !allowed(start)) continue;
      std::vector<uint32_t> vs{start};
      std::vector<std::pair<uint32_t, uint32_t>> tree;
      uint32_t cur = start;
      for (uint32_t step = 0; step < 64 * nq && vs.size() < nq; ++step) {
        uint32_t d = g.deg(cur);
        if (d == 0) break;
        uint32_t w = g.nbr[g.off[cur] + r.below(d)];
        if (!allowed(w)) continue;
        auto it = std::find(vs.begin(), vs.end(), w);
        if (it == vs.end()) {
          tree.push_back({(uint32_t)(std::find(vs.begin(), vs.end(), cur) - vs.begin()), (uint32_t)vs.size()});
          vs.push_back(w);
        }
        cur = w;
      }
      if (vs.size() < nq) continue;
      std::vector<std::pair<uint32_t, uint32_t>> cand;
      for (uint32_t i = 0; i < nq; ++i)
        for (uint32_t j = i + 1; j < nq; ++j) {
          bool in_tree = false;
          for (auto &t : tree)
            if ((t.first == i && t.second == j) || (t.first == j && t.second == i)) in_tree = true;
          if (!in_tree && g.has(vs[i], vs[j])) cand.push_back({i, j});
        }
      if (cand.size() < extra) continue;
      shuffle(cand, r);
      std::vector<std::pair<uint32_t, uint32_t>> edges = tree;
      edges.insert(edges.end(), cand.begin(), cand.begin() + extra);
      for (auto &e : edges)
        if (e.first > e.second) std::swap(e.first, e.second);
      std::sort(edges.begin(), edges.end());
      q.nv = nq;
      q.labels.resize(nq);
      for (uint32_t i = 0; i < nq; ++i) q.labels[i] = labels[vs[i]];
      q.edges.clear();
      for (auto &e : edges) {
        q.edges.push_back(e.first);
        q.edges.push_back(e.second);
      }
      q.build_csr();
      if (!selective) return true;
      ++scored;
      const uint64_t cap = (uint64_t)(10 * max_mean) + 1;
      const double budget = max_mean * (double)probe.size();
      double total = 0;
      bool pass = true;
      for (uint64_t k : probe) {
        uint32_t a = (uint32_t)(k >> 32), b = (uint32_t)k;
        uint64_t c = capped_edge_count(g, labels, q, a, b, cap);
        if (c < cap) c += capped_edge_count(g, labels, q, b, a, cap - c);
        total += (double)c;
        if (c >= cap || total > budget) {
          pass = false;
          if (total >= best_total) break;
        }
      }
      if (pass) return true;
      if (total < best_total) {
        best_total = total;
        best = q;
      }
    }
  }
  if (best_total < 1e300) {
    q = best;
    return true;
  }
  return false;
}

}  // namespace

void Query::build_csr() {
  offsets.assign(nv + 1, 0);
  uint32_t ne = (uint32_t)(edges.size() / 2);
  for (uint32_t k = 0; k < ne; ++k) {
    offsets[edges[2 * k] + 1]++;
    offsets[edges[2 * k + 1] + 1]++;
  }
  for (uint32_t u = 0; u < nv; ++u) offsets[u + 1] += offsets[u];
  nbrs.assign(2 * ne, 0);
  std::vector<uint32_t> fill(offsets.begin(), offsets.end() - 1);
  // file order: each edge appends to both endpoints' lists (io.cu:181-189)
  for (uint32_t k = 0; k < ne; ++k) {
    uint32_t s = edges[2 * k], d = edges[2 * k + 1];
    nbrs[fill[s]++] = d;
    nbrs[fill[d]++] = s;
  }
}

int generate_workload(const GenParams &p, Workload &w) {
  // independent streams: graph and labels, update stream, queries
  Rng r(p.seed * 0x9E3779B97F4A7C15ull + 0x5DEECE66Dull);
  Rng rs(p.seed * 0xD1B54A32D192ED03ull + 0x2545F4914F6CDD1Dull);
  Rng rq(p.seed * 0xA0761D6478BD642Full + 0xE7037ED1A0B428DBull);
  std::vector<uint64_t> keys;
  uint32_t nv = 1u << p.log2_nv;
  if (p.graph == GenParams::kRmat)
    keys = gen_rmat(p.log2_nv, p.num_edges, p.a, p.b, p.c, r);
  else
    keys = gen_chung_lu(nv, p.num_edges, p.gamma, r);
  w.nv = nv;
  w.labels = gen_labels(nv, p.num_labels, p.zipf_s, r);

  // withheld pool = the first fraction of the shuffled edge list
  uint64_t withheld = (uint64_t)std::floor((double)p.num_edges * p.withheld_frac);
  std::vector<uint64_t> pool(keys.begin(), keys.begin() + withheld);
  std::vector<uint64_t> live(keys.begin() + withheld, keys.end());
  w.edges.resize(2 * live.size());
  for (size_t i = 0; i < live.size(); ++i) {
    w.edges[2 * i] = (uint32_t)(live[i] >> 32);
    w.edges[2 * i + 1] = (uint32_t)live[i];
  }
  Adj g = build_adj(nv, live);  // the initial graph, for query sampling

  // update stream
  w.updates.clear();
  w.batch_sizes.clear();
  shuffle(pool, rs);
  size_t pool_head = 0;
  auto push = [&](uint32_t op, uint64_t k) {
    uint32_t s = (uint32_t)(k >> 32), d = (uint32_t)k;
    if (rs.below(2)) std::swap(s, d);
    w.updates.push_back(op);
    w.updates.push_back(s);
    w.updates.push_back(d);
    w.updates.push_back(w.labels[s]);  // 4th field = label(src)
  };
  if (p.stream == GenParams::kStreamWithheld) {
    // every withheld edge re-inserted once, plus `num_deletes` deletions of
    // live edges, interleaved in seeded order, one update per batch
    std::vector<uint8_t> ops(withheld, 1);
    ops.insert(ops.end(), p.num_deletes, 0);
    shuffle(ops, rs);
    for (uint8_t op : ops) {
      if (op) {
        uint64_t k = pool[pool_head++];
        live.push_back(k);
        push(1, k);
      } else {
        size_t i = rs.below(live.size());
        uint64_t k = live[i];
        live[i] = live.back();
        live.pop_back();
        push(0, k);
      }
      w.batch_sizes.push_back(1);
    }
  } else {
    for (uint32_t b = 0; b < p.num_batches; ++b) {
      uint32_t size = p.batch_size;
      if (p.lognormal_sigma > 0) {
        // lognormal(mu = ln median, sigma) by Box-Muller, capped
        double u1 = std::max(rs.unit(), 1e-300), u2 = rs.unit();
        double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
        double s = std::exp(std::log((double)p.batch_size) + p.lognormal_sigma * z);
        size = (uint32_t)std::max(1.0, std::min(s, (double)p.batch_cap));
      }
      uint32_t n_ins = (uint32_t)std::llround(size * p.insert_frac);
      std::vector<uint8_t> ops(size, 0);
      std::fill(ops.begin(), ops.begin() + n_ins, 1);
      shuffle(ops, rs);
      uint32_t pushed = 0;
      for (uint8_t op : ops) {
        ++pushed;
        if (op && pool_head < pool.size()) {
          uint64_t k = pool[pool_head++];
          live.push_back(k);
          push(1, k);
        } else if (!live.empty()) {
          size_t i = rs.below(live.size());
          uint64_t k = live[i];
          live[i] = live.back();
          live.pop_back();
          pool.push_back(k);  // a deleted edge may come back later
          push(0, k);
        } else {
          --pushed;
        }
      }
      w.batch_sizes.push_back(pushed);
    }
  }

  // queries: random walks on the initial graph; the selectivity test probes
  // the distinct edges of the first q_probe_updates updates
  std::vector<uint64_t> probe;
  if (p.q_max_mean_matches > 0) {
    size_t np = std::min<size_t>(p.q_probe_updates, w.updates.size() / 4);
    for (size_t i = 0; i < np; ++i) probe.push_back(edge_key(w.updates[4 * i + 1], w.updates[4 * i + 2]));
    std::sort(probe.begin(), probe.end());
    probe.erase(std::unique(probe.begin(), probe.end()), probe.end());
    shuffle(probe, rq);
  }
  // shapes and per-query seeds are drawn in order; the samples themselves run
  // on all host threads (each query has its own stream, so the result does
  // not depend on the thread count)
  // frequency rank of each label (0 = most frequent)
  std::vector<uint32_t> label_rank(p.num_labels, 0);
  {
    std::vector<uint64_t> freq(p.num_labels, 0);
    for (uint32_t l : w.labels) freq[l]++;
    std::vector<uint32_t> ids(p.num_labels);
    for (uint32_t l = 0; l < p.num_labels; ++l) ids[l] = l;
    std::stable_sort(ids.begin(), ids.end(), [&](uint32_t x, uint32_t y) { return freq[x] > freq[y]; });
    for (uint32_t k = 0; k < p.num_labels; ++k) label_rank[ids[k]] = k;
  }
  const uint32_t nqs = p.num_queries;
  std::vector<uint32_t> q_nv(nqs), q_extra(nqs);
  std::vector<uint64_t> q_seed(nqs);
  for (uint32_t qi = 0; qi < nqs; ++qi) {
    q_nv[qi] = p.q_nv_min + (uint32_t)rq.below(p.q_nv_max - p.q_nv_min + 1);
    if (p.q_extra_fixed.size() > qi) {
      q_extra[qi] = p.q_extra_fixed[qi];
    } else {
      uint32_t hi = (uint32_t)std::floor(p.q_extra_frac_max * (double)(q_nv[qi] - 1));
      uint32_t lo = std::min(p.q_extra_min, hi);
      q_extra[qi] = lo + (uint32_t)rq.below(hi - lo + 1);
    }
    q_seed[qi] = rq.u64();
  }
  w.queries.assign(nqs, Query());
  std::vector<int> ok(nqs, 0);
  std::atomic<uint32_t> next{0};
  auto worker = [&]() {
    for (uint32_t qi; (qi = next.fetch_add(1)) < nqs;) {
      Rng rl(q_seed[qi]);
      ok[qi] = sample_query(g, w.labels, label_rank, probe, q_nv[qi], q_extra[qi], p.q_max_mean_matches, rl,
                            w.queries[qi]);
    }
  };
  unsigned nt = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), 32));
  std::vector<std::thread> pool_threads;
  for (unsigned t = 1; t < nt; ++t) pool_threads.emplace_back(worker);
  worker();
  for (auto &t : pool_threads) t.join();
  for (uint32_t qi = 0; qi < nqs; ++qi)
    if (!ok[qi]) return -1;
  return 0;
}

// Presets for the five workloads (sizes can be scaled down for tests by
// lowering log2_nv / num_edges / batch counts after taking the preset).
int preset_params(int config, GenParams &p) {
  p = GenParams();
  switch (config) {
    case 1:  // plain single query, CPU-runnable, one update per batch
      p.graph = GenParams::kRmat;
      p.log2_nv = 12;
      p.num_edges = 32768;
      p.a = 0.57, p.b = 0.19, p.c = 0.19;
      p.num_labels = 4;
      p.num_queries = 1;
      p.q_nv_min = p.q_nv_max = 5;
      p.q_extra_fixed = {1};
      p.withheld_frac = 0.1;
      p.stream = GenParams::kStreamWithheld;
      p.num_deletes = 1000;
      p.seed = 1;
      return 0;
    case 2:  // plain GPU: Chung-Lu, three 8-vertex queries run separately
      p.graph = GenParams::kChungLu;
      p.log2_nv = 20;
      p.num_edges = 1ull << 24;
      p.gamma = 2.1;
      p.num_labels = 16;
      p.zipf_s = 1.2;
      p.num_queries = 3;
      p.q_nv_min = p.q_nv_max = 8;
      p.q_extra_fixed = {0, 1, 7};  // tree (7 edges), one cycle (8), dense (14)
      p.q_max_mean_matches = 1000;
      p.withheld_frac = 0.1;
      p.stream = GenParams::kStreamBatches;
      p.batch_size = 4096;
      p.insert_frac = 0.5;
      p.num_batches = 64;
      p.seed = 2;
      return 0;
    case 3:  // batched multi-query on the config-2 graph and batches
      preset_params(2, p);
      p.num_queries = 256;
      p.q_nv_min = 4;
      p.q_nv_max = 12;
      p.q_extra_fixed.clear();
      p.q_extra_min = 0;
      p.q_extra_frac_max = 0.5;
      p.seed = 3;
      return 0;
    case 4:  // serving loop: large R-MAT, lognormal batches
      p.graph = GenParams::kRmat;
      p.log2_nv = 24;
      p.num_edges = 1ull << 28;
      p.a = 0.57, p.b = 0.19, p.c = 0.19;
      p.num_labels = 32;
      p.num_queries = 64;
      p.q_nv_min = 4;
      p.q_nv_max = 10;
      p.q_extra_min = 0;
      p.q_extra_frac_max = 0.5;
      p.q_max_mean_matches = 1000;
      p.withheld_frac = 0.1;
      p.stream = GenParams::kStreamBatches;
      p.batch_size = 512;
      p.batch_cap = 65536;
      p.lognormal_sigma = 1.0;
      p.insert_frac = 0.6;
      p.num_batches = 64;
      p.seed = 4;
      return 0;
    case 5:  // skew stress: hub-heavy R-MAT, 12-vertex cyclic queries
      p.graph = GenParams::kRmat;
      p.log2_nv = 22;
      p.num_edges = 1ull << 27;
      p.a = 0.70, p.b = 0.12, p.c = 0.12;
      p.num_labels = 8;
      p.num_queries = 64;
      p.q_nv_min = p.q_nv_max = 12;
      p.q_extra_min = 3;
      p.q_extra_frac_max = 3.0 / 11.0;
      p.q_max_mean_matches = 1000;
      p.withheld_frac = 0.1;
      p.stream = GenParams::kStreamBatches;
      p.batch_size = 65536;
      p.insert_frac = 0.2;
      p.num_batches = 8;
      p.seed = 5;
      return 0;
  }
  return -1;
}

}  // namespace dsm
