// Host-side types shared by the engine, the generators, the text reader and
// the CDSM command line.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace dsm {

// Limits.  Query vertices are addressed by bit masks of 32 bits, so a query
// has at most 32 vertices; labels used by a query are below 32 (the
// per-vertex neighbour-label signature holds 32 four-bit counters).
constexpr uint32_t kMaxQueryVertices = 16;  // reference: MAX_VQ (defs.h:18)
constexpr uint32_t kMaxLabels = 32;         // reference: MAX_VLQ=16 (defs.h:20), lifted

struct Query {
  uint32_t nv = 0;
  std::vector<uint32_t> labels;   // nv
  std::vector<uint32_t> edges;    // pairs, file order
  std::vector<uint32_t> offsets;  // nv+1 (CSR in file order, io.cu:181-189)
  std::vector<uint32_t> nbrs;     // 2*ne
  void build_csr();
};

struct Workload {
  uint32_t nv = 0;
  std::vector<uint32_t> labels;   // nv
  std::vector<uint32_t> edges;    // initial undirected edges, pairs
  std::vector<Query> queries;
  std::vector<uint32_t> updates;  // 4 words each: op (1 add / 0 delete), src, dst, label
  std::vector<uint32_t> batch_sizes;
};

struct GenParams {
  enum Graph { kRmat = 0, kChungLu = 1 };
  enum Stream { kStreamWithheld = 0, kStreamBatches = 1 };
  int graph = kRmat;
  uint32_t log2_nv = 12;
  uint64_t num_edges = 32768;
  double a = 0.57, b = 0.19, c = 0.19;  // R-MAT quadrant probabilities (d = rest)
  double gamma = 2.1;                   // Chung-Lu power-law exponent
  uint32_t num_labels = 4;
  double zipf_s = 0.0;                  // 0 = uniform labels
  uint32_t num_queries = 1;
  uint32_t q_nv_min = 5, q_nv_max = 5;
  std::vector<uint32_t> q_extra_fixed;  // extra (non-tree) edges per query, if given
  uint32_t q_extra_min = 0;
  double q_extra_frac_max = 0.0;        // else extra ~ U[min, floor(frac*(nq-1))]
  double q_max_mean_matches = 0.0;      // > 0: selectivity acceptance test (see gen.cpp)
  uint32_t q_probe_updates = 256;      // updates whose edges the test probes
  double withheld_frac = 0.1;
  int stream = kStreamWithheld;
  uint32_t num_deletes = 1000;          // kStreamWithheld
  uint32_t batch_size = 4096;           // kStreamBatches (median when lognormal)
  uint32_t batch_cap = 65536;
  double lognormal_sigma = 0.0;
  double insert_frac = 0.5;
  uint32_t num_batches = 16;
  uint64_t seed = 1;
};

int preset_params(int config, GenParams &p);
int generate_workload(const GenParams &p, Workload &w);

// Text formats (io.cu:122-252).  Returns 0, or -1 with a message in err.
struct TextGraph {
  uint32_t nv = 0, ne = 0;
  std::vector<uint32_t> labels, offsets, nbrs, edges;
  std::vector<uint32_t> batch_sizes;
  std::vector<uint32_t> updates;  // 4 words each
};
int read_text_graph(const std::string &path, bool is_query, TextGraph &g, std::string &err);

// The arrays of a query or data file, however they are held (binio.cpp).
struct GraphArrays {
  bool is_query = false;
  uint32_t nv = 0, ne = 0, num_batches = 0, num_updates = 0;
  const uint32_t *labels = nullptr, *offsets = nullptr, *nbrs = nullptr, *edges = nullptr,
                 *batch_sizes = nullptr, *updates = nullptr;
};
struct MappedGraph {
  void *base = nullptr;
  size_t len = 0;
  GraphArrays a;
  MappedGraph() = default;
  MappedGraph(const MappedGraph &) = delete;
  MappedGraph &operator=(const MappedGraph &) = delete;
  ~MappedGraph();
};
bool is_binary_graph(const std::string &path);
int write_binary_graph(const std::string &path, const GraphArrays &a, std::string &err);
int map_binary_graph(const std::string &path, bool is_query, MappedGraph &m, std::string &err);
int write_query_file(const std::string &path, const Query &q);
int write_data_file(const std::string &path, const Workload &w);

}  // namespace dsm
