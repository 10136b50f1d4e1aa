// Binary form of a query or data file, mapped without parsing.
//
// No counterpart in the reference: its only reader is the text parser
// (readGraphToCPUDynamic, io.cu:122-252), an `ifstream >>` loop that
// dominates load time at 2^28 edges.  The binary file holds the arrays that
// the text reader produces (labels, CSR offsets and neighbours in file order,
// the edge list in file order, batch sizes, updates), so a graph read either
// way is the same graph.
//
// Layout (little-endian u32 / u64):
//   header (64 bytes): magic "DSMGRPH1", version 1, is_query, nv, ne,
//                      nnbrs (u64), num_batches, num_updates, file bytes (u64)
//   sections, each starting on a 64-byte boundary:
//     labels[nv], offsets[nv + 1], nbrs[nnbrs], edges[2 ne],
//     batch_sizes[num_batches], updates[4 num_updates]
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>

#include "dsm_host.h"

namespace dsm {

namespace {

constexpr char kMagic[8] = {'D', 'S', 'M', 'G', 'R', 'P', 'H', '1'};
constexpr uint32_t kVersion = 1;

struct Header {
  char magic[8];
  uint32_t version, is_query, nv, ne;
  uint64_t nnbrs;
  uint32_t num_batches, num_updates;
  uint64_t bytes;
  uint32_t pad[4];
};
static_assert(sizeof(Header) == 64, "header is 64 bytes");

uint64_t align64(uint64_t x) { return (x + 63) & ~63ull; }

// Section offsets of a file with these counts; returns the file size.
uint64_t layout(const Header &h, uint64_t off[6]) {
  const uint64_t words[6] = {h.nv, (uint64_t)h.nv + 1, h.nnbrs, 2ull * h.ne, h.num_batches, 4ull * h.num_updates};
  uint64_t pos = sizeof(Header);
  for (int s = 0; s < 6; ++s) {
    off[s] = pos;
    pos = align64(pos + 4 * words[s]);
  }
  return pos;
}

}  // namespace

MappedGraph::~MappedGraph() {
  if (base) munmap(base, len);
}

bool is_binary_graph(const std::string &path) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  char m[8] = {0};
  const bool ok = std::fread(m, 1, 8, f) == 8 && std::memcmp(m, kMagic, 8) == 0;
  std::fclose(f);
  return ok;
}

int write_binary_graph(const std::string &path, const GraphArrays &a, std::string &err) {
  Header h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kMagic, 8);
  h.version = kVersion;
  h.is_query = a.is_query ? 1 : 0;
  h.nv = a.nv;
  h.ne = a.ne;
  h.nnbrs = a.offsets ? a.offsets[a.nv] : 0;
  h.num_batches = a.num_batches;
  h.num_updates = a.num_updates;
  uint64_t off[6];
  h.bytes = layout(h, off);
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = "cannot open " + path + " for writing";
    return 1;
  }
  const void *src[6] = {a.labels, a.offsets, a.nbrs, a.edges, a.batch_sizes, a.updates};
  const uint64_t words[6] = {h.nv, (uint64_t)h.nv + 1, h.nnbrs, 2ull * h.ne, h.num_batches, 4ull * h.num_updates};
  bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
  uint64_t pos = sizeof(h);
  static const char zeros[64] = {0};
  for (int s = 0; s < 6 && ok; ++s) {
    ok = std::fwrite(zeros, 1, off[s] - pos, f) == off[s] - pos;
    if (ok && words[s]) ok = src[s] && std::fwrite(src[s], 4, words[s], f) == words[s];
    pos = off[s] + 4 * words[s];
  }
  if (ok) ok = std::fwrite(zeros, 1, h.bytes - pos, f) == h.bytes - pos;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) err = "write failed: " + path;
  return ok ? 0 : 1;
}

int map_binary_graph(const std::string &path, bool is_query, MappedGraph &m, std::string &err) {
  const int fd = ::open(path.c_str(), O_RDONLY);
  if (fd < 0) {
    err = "cannot open " + path;
    return 1;
  }
  struct stat st;
  if (fstat(fd, &st) != 0 || (size_t)st.st_size < sizeof(Header)) {
    ::close(fd);
    err = "not a binary graph (too short): " + path;
    return 1;
  }
  void *p = mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
  ::close(fd);
  if (p == MAP_FAILED) {
    err = "mmap failed: " + path;
    return 1;
  }
  m.base = p;
  m.len = (size_t)st.st_size;
  Header h;
  std::memcpy(&h, p, sizeof(h));
  uint64_t off[6];
  if (std::memcmp(h.magic, kMagic, 8) != 0 || h.version != kVersion) {
    err = "not a binary graph (magic / version): " + path;
    return 1;
  }
  if (h.bytes != layout(h, off) || h.bytes > m.len) {
    err = "binary graph truncated or sized wrong: " + path;
    return 1;
  }
  if ((h.is_query != 0) != is_query) {
    err = is_query ? "binary file holds a data graph, a query was expected" : "binary file holds a query graph";
    return 1;
  }
  const char *b = (const char *)p;
  m.a.is_query = h.is_query != 0;
  m.a.nv = h.nv;
  m.a.ne = h.ne;
  m.a.labels = (const uint32_t *)(b + off[0]);
  m.a.offsets = (const uint32_t *)(b + off[1]);
  m.a.nbrs = (const uint32_t *)(b + off[2]);
  m.a.edges = (const uint32_t *)(b + off[3]);
  m.a.batch_sizes = (const uint32_t *)(b + off[4]);
  m.a.updates = (const uint32_t *)(b + off[5]);
  m.a.num_batches = h.num_batches;
  m.a.num_updates = h.num_updates;
  // the CSR must be consistent before anyone indexes with it
  if (m.a.offsets[0] != 0 || m.a.offsets[h.nv] != h.nnbrs) {
    err = "binary graph: offsets inconsistent";
    return 1;
  }
  for (uint32_t v = 0; v < h.nv; ++v)
    if (m.a.offsets[v + 1] < m.a.offsets[v]) {
      err = "binary graph: offsets not ascending";
      return 1;
    }
  for (uint64_t k = 0; k < h.nnbrs; ++k)
    if (m.a.nbrs[k] >= h.nv) {
      err = "binary graph: neighbour id >= num_v";
      return 1;
    }
  uint64_t sum = 0;
  for (uint32_t i = 0; i < h.num_batches; ++i) sum += m.a.batch_sizes[i];
  if (sum != h.num_updates) {
    err = "binary graph: batch sizes do not add up to the updates";
    return 1;
  }
  return 0;
}

}  // namespace dsm
