// Reader and writer for DSM's text formats (io.cu:122-252):
//
//   t <num_v> <num_e>
//   v <id> <label> <degree>        one per vertex, ids in order
//   e <src> <dst>                  one per undirected edge
//   -                              end of the static part (data graphs)
//   b <batch_id> <size>            then <size> lines of
//   a|d <src> <dst> <label>        insert / delete, label = 4th field
//
// The reader is a single pass over a memory buffer with a hand-rolled
// tokenizer (the reference reads with `ifstream >>`, which dominates load time
// on large graphs).  It is stricter than the reference where the reference
// would write out of bounds: v-lines must come in id order, each vertex must
// get exactly its declared number of e-lines, ids must be below num_v.
#include "dsm_host.h"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace dsm {

namespace {

struct Cursor {
  const char *p, *end;
  void skip_ws() {
    while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
  }
  bool tok_char(char &c) {
    skip_ws();
    if (p >= end) return false;
    c = *p++;
    return true;
  }
  bool tok_u64(uint64_t &x) {
    skip_ws();
    if (p >= end || *p < '0' || *p > '9') return false;
    uint64_t v = 0;
    while (p < end && *p >= '0' && *p <= '9') {
      v = v * 10 + (uint64_t)(*p - '0');
      if (v > 0xFFFFFFFFull) return false;
      ++p;
    }
    x = v;
    return true;
  }
};

bool slurp(const std::string &path, std::string &buf) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  long n = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  buf.resize(n > 0 ? (size_t)n : 0);
  size_t got = n > 0 ? std::fread(&buf[0], 1, (size_t)n, f) : 0;
  std::fclose(f);
  return got == buf.size();
}

}  // namespace

int read_text_graph(const std::string &path, bool is_query, TextGraph &g, std::string &err) {
  std::string buf;
  if (!slurp(path, buf)) {
    err = "cannot open " + path;
    return -1;
  }
  Cursor c{buf.data(), buf.data() + buf.size()};
  char t;
  uint64_t nv, ne;
  if (!c.tok_char(t) || t != 't' || !c.tok_u64(nv) || !c.tok_u64(ne)) {
    err = path + ": expected 't <num_v> <num_e>'";
    return -1;
  }
  g = TextGraph();
  g.nv = (uint32_t)nv;
  g.ne = (uint32_t)ne;
  g.labels.assign(g.nv, 0);
  g.offsets.assign((size_t)g.nv + 1, 0);
  g.nbrs.assign(2 * (size_t)g.ne, 0);
  g.edges.reserve(2 * (size_t)g.ne);
  std::vector<uint32_t> fill(g.nv, 0);
  uint32_t next_v = 0;
  while (c.tok_char(t)) {
    if (t == 'v') {
      uint64_t id, lab, deg;
      if (!c.tok_u64(id) || !c.tok_u64(lab) || !c.tok_u64(deg) || id != next_v) {
        err = path + ": bad v-line (ids must be 0..num_v-1 in order)";
        return -1;
      }
      g.labels[id] = (uint32_t)lab;
      g.offsets[id + 1] = g.offsets[id] + (uint32_t)deg;
      ++next_v;
    } else if (t == 'e') {
      uint64_t s, d;
      if (!c.tok_u64(s) || !c.tok_u64(d) || s >= g.nv || d >= g.nv || next_v != g.nv ||
          g.edges.size() >= 2 * (size_t)g.ne) {
        err = path + ": bad e-line";
        return -1;
      }
      if (g.offsets[s] + fill[s] >= g.offsets[s + 1] || g.offsets[d] + fill[d] >= g.offsets[d + 1]) {
        err = path + ": more e-lines at a vertex than its declared degree";
        return -1;
      }
      g.nbrs[g.offsets[s] + fill[s]++] = (uint32_t)d;
      g.nbrs[g.offsets[d] + fill[d]++] = (uint32_t)s;
      g.edges.push_back((uint32_t)s);
      g.edges.push_back((uint32_t)d);
    } else if (t == '-') {
      break;
    } else {
      err = path + ": unexpected token '" + std::string(1, t) + "'";
      return -1;
    }
  }
  if (next_v != g.nv || g.edges.size() != 2 * (size_t)g.ne || g.offsets[g.nv] != 2 * (uint64_t)g.ne) {
    err = path + ": vertex/edge counts do not match the t-line or the declared degrees";
    return -1;
  }
  for (uint32_t v = 0; v < g.nv; ++v)
    if (fill[v] != g.offsets[v + 1] - g.offsets[v]) {
      err = path + ": a vertex has fewer e-lines than its declared degree";
      return -1;
    }
  if (is_query) return 0;
  std::vector<std::vector<uint32_t>> batches;
  while (c.tok_char(t)) {
    if (t != 'b') continue;  // as the reference, tokens between batches are skipped
    uint64_t bid, bsize;
    if (!c.tok_u64(bid) || !c.tok_u64(bsize)) {
      err = path + ": bad b-line";
      return -1;
    }
    batches.emplace_back();
    if (bid >= batches.size()) {
      err = path + ": batch id beyond the batches read so far";
      return -1;
    }
    g.batch_sizes.push_back((uint32_t)bsize);
    auto &b = batches[bid];
    for (uint64_t i = 0; i < bsize; ++i) {
      char op;
      uint64_t s, d, l;
      if (!c.tok_char(op) || (op != 'a' && op != 'd') || !c.tok_u64(s) || !c.tok_u64(d) ||
          !c.tok_u64(l) || s >= g.nv || d >= g.nv) {
        err = path + ": bad update line (expected 'a|d src dst label')";
        return -1;
      }
      b.push_back(op == 'a' ? 1u : 0u);
      b.push_back((uint32_t)s);
      b.push_back((uint32_t)d);
      b.push_back((uint32_t)l);
    }
  }
  for (auto &b : batches) g.updates.insert(g.updates.end(), b.begin(), b.end());
  return 0;
}

int write_query_file(const std::string &path, const Query &q) {
  std::ofstream o(path);
  if (!o) return -1;
  uint32_t ne = (uint32_t)(q.edges.size() / 2);
  o << "t " << q.nv << " " << ne << "\n";
  for (uint32_t u = 0; u < q.nv; ++u)
    o << "v " << u << " " << q.labels[u] << " " << (q.offsets[u + 1] - q.offsets[u]) << "\n";
  for (uint32_t k = 0; k < ne; ++k) o << "e " << q.edges[2 * k] << " " << q.edges[2 * k + 1] << "\n";
  return o ? 0 : -1;
}

int write_data_file(const std::string &path, const Workload &w) {
  std::ofstream o(path);
  if (!o) return -1;
  std::vector<uint32_t> deg(w.nv, 0);
  size_t ne = w.edges.size() / 2;
  for (size_t k = 0; k < ne; ++k) {
    deg[w.edges[2 * k]]++;
    deg[w.edges[2 * k + 1]]++;
  }
  std::string s;
  s.reserve(1 << 20);
  s += "t " + std::to_string(w.nv) + " " + std::to_string(ne) + "\n";
  for (uint32_t v = 0; v < w.nv; ++v) {
    s += "v " + std::to_string(v) + " " + std::to_string(w.labels[v]) + " " + std::to_string(deg[v]) + "\n";
    if (s.size() > (1 << 20)) o << s, s.clear();
  }
  for (size_t k = 0; k < ne; ++k) {
    s += "e " + std::to_string(w.edges[2 * k]) + " " + std::to_string(w.edges[2 * k + 1]) + "\n";
    if (s.size() > (1 << 20)) o << s, s.clear();
  }
  s += "-\n";
  size_t u = 0;
  for (size_t b = 0; b < w.batch_sizes.size(); ++b) {
    s += "b " + std::to_string(b) + " " + std::to_string(w.batch_sizes[b]) + "\n";
    for (uint32_t i = 0; i < w.batch_sizes[b]; ++i, ++u) {
      const uint32_t *x = &w.updates[4 * u];
      s += (x[0] ? "a " : "d ") + std::to_string(x[1]) + " " + std::to_string(x[2]) + " " +
           std::to_string(x[3]) + "\n";
      if (s.size() > (1 << 20)) o << s, s.clear();
    }
  }
  o << s;
  return o ? 0 : -1;
}

}  // namespace dsm
