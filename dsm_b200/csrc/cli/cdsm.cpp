// CDSM: command line of the B200 engine, a drop-in for DSM's
// `CDSM -q <query> -d <data> [--gpu N]` (main.cu:37-45).
//
// Reads the query and the data file (graph, then update batches) in DSM's
// text format, matches every batch on the GPU and writes, per update, its
// positive (insert) or negative (delete) embeddings:
//
//   u <batch> <index> <a|d> <src> <dst> <+|-|0> <count>
//   <f(0)> <f(1)> ... <f(nq-1)>          one line per embedding, sorted
//
// Options beyond the reference's three: --out FILE (default stdout),
// --count (counts only, no embedding lines), --queries a,b,... (more query
// files matched in the same launch; lines then start with the query's
// position as `q<k>`), --quiet (no per-update output; timing only),
// --serve (the serving loop: every batch is queued at once, batches queued
// together run as one device batch; the output is the same), --graph (CUDA
// graph replay of each batch), --autotune (the first batch tunes the
// matcher's launch setting).  Timing goes to stderr, one line per batch
// (submit to results; with --serve, as the serving loop measured it) and a
// summary.
#include <chrono>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "dsm.h"

namespace {

void usage() {
  std::fprintf(stderr,
               "usage: CDSM -q <query> -d <data> [--gpu N] [--out FILE] [--count] [--quiet]\n"
               "            [--queries q2,q3,...] [--serve] [--graph] [--autotune]\n");
}

bool read_text(const std::string &path, int is_query, dsm_text **t) {
  char err[512] = {0};
  int rc = dsm_text_read(path.c_str(), is_query, t, err, sizeof err);
  if (rc) {
    std::fprintf(stderr, "CDSM: %s (%s)\n", err[0] ? err : path.c_str(), dsm_status_string(rc));
    return false;
  }
  return true;
}

}  // namespace

int main(int argc, char **argv) {
  std::string qpath, dpath, out_path, extra;
  int gpu = 0;
  bool count_only = false, quiet = false, serve = false, graph = false, autotune = false;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto next = [&](std::string &dst) {
      if (i + 1 >= argc) {
        usage();
        std::exit(2);
      }
      dst = argv[++i];
    };
    if (a == "-q") next(qpath);
    else if (a == "-d") next(dpath);
    else if (a == "--gpu") {
      std::string s;
      next(s);
      gpu = std::atoi(s.c_str());
    } else if (a == "--out") next(out_path);
    else if (a == "--queries") next(extra);
    else if (a == "--count") count_only = true;
    else if (a == "--quiet") quiet = true;
    else if (a == "--serve") serve = true;
    else if (a == "--graph") graph = true;
    else if (a == "--autotune") autotune = true;
    else if (a == "-h" || a == "--help") {
      usage();
      return 0;
    } else {
      std::fprintf(stderr, "CDSM: unknown option %s\n", a.c_str());
      usage();
      return 2;
    }
  }
  if (qpath.empty() || dpath.empty()) {
    usage();
    return 2;
  }
  std::vector<std::string> qpaths{qpath};
  for (size_t p = 0; p < extra.size();) {
    size_t c = extra.find(',', p);
    if (c == std::string::npos) c = extra.size();
    if (c > p) qpaths.push_back(extra.substr(p, c - p));
    p = c + 1;
  }

  auto t0 = std::chrono::steady_clock::now();
  std::vector<dsm_text *> queries;
  for (auto &p : qpaths) {
    dsm_text *q = nullptr;
    if (!read_text(p, 1, &q)) return 1;
    queries.push_back(q);
  }
  dsm_text *g = nullptr;
  if (!read_text(dpath, 0, &g)) return 1;
  double read_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::fprintf(stderr, "read to csr (seconds): %.6f\n", read_s);

  dsm_engine *e = nullptr;
  int rc = dsm_engine_create(gpu, 0, &e);
  if (rc) {
    std::fprintf(stderr, "CDSM: cannot use GPU %d (%s)\n", gpu, dsm_status_string(rc));
    return 1;
  }
  if (count_only) dsm_engine_set_option(e, DSM_OPT_LIST, 0);
  if (graph) dsm_engine_set_option(e, DSM_OPT_GRAPH, 1);
  if (autotune) dsm_engine_set_option(e, DSM_OPT_AUTOTUNE, 1);
  auto fail = [&](int code) {
    std::fprintf(stderr, "CDSM: %s: %s\n", dsm_status_string(code), dsm_last_error(e));
    dsm_engine_destroy(e);
    return 1;
  };
  if ((rc = dsm_graph_load(e, dsm_text_offsets(g), dsm_text_nbrs(g), dsm_text_labels(g), dsm_text_nv(g))))
    return fail(rc);
  std::vector<uint32_t> qids;
  for (auto *q : queries) {
    uint32_t id = 0;
    if ((rc = dsm_query_register(e, dsm_text_offsets(q), dsm_text_nbrs(q), dsm_text_labels(q), dsm_text_nv(q), &id)))
      return fail(rc);
    qids.push_back(id);
  }

  FILE *out = stdout;
  if (!out_path.empty() && !(out = std::fopen(out_path.c_str(), "w"))) {
    std::fprintf(stderr, "CDSM: cannot write %s\n", out_path.c_str());
    return 1;
  }
  const dsm_update *ups = dsm_text_updates(g);
  const uint32_t *sizes = dsm_text_batch_sizes(g);
  const uint32_t nb = dsm_text_num_batches(g);
  uint64_t pos = 0, total_matches = 0, total_updates = 0;
  double total_ms = 0;
  std::vector<uint64_t> queued(nb, 0);
  const auto t_loop = std::chrono::steady_clock::now();
  if (serve) {  // queue every batch; the serving loop merges what queues up
    if ((rc = dsm_serve_start(e, 0))) return fail(rc);
    for (uint32_t b = 0, p = 0; b < nb; p += sizes[b], ++b)
      if ((rc = dsm_batch_submit(e, ups + p, sizes[b], &queued[b]))) return fail(rc);
  }
  for (uint32_t b = 0; b < nb; ++b) {
    uint32_t n = sizes[b];
    auto tb = std::chrono::steady_clock::now();
    uint64_t id = queued[b];
    if (!serve && (rc = dsm_batch_submit(e, ups + pos, n, &id))) return fail(rc);
    dsm_result_view v;
    if ((rc = dsm_batch_results(e, id, &v))) return fail(rc);
    double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tb).count();
    if (serve) {
      dsm_batch_timing tm;
      if (dsm_batch_timing_get(e, id, &tm) == DSM_OK) ms = tm.total_ms;
    }
    uint64_t bm = 0;
    for (uint32_t ql = 0; ql < v.num_queries; ++ql)
      for (uint32_t i = 0; i < v.num_updates; ++i) bm += v.counts[(size_t)ql * v.num_updates + i];
    if (!quiet) {
      for (uint32_t ql = 0; ql < v.num_queries; ++ql)
        for (uint32_t i = 0; i < v.num_updates; ++i) {
          const dsm_update &u = ups[pos + i];
          size_t s = (size_t)ql * v.num_updates + i;
          char sign = v.signs[i] > 0 ? '+' : (v.signs[i] < 0 ? '-' : '0');
          if (v.num_queries > 1) std::fprintf(out, "q%u ", ql);
          std::fprintf(out, "u %u %u %c %u %u %c %" PRIu64 "\n", b, i, u.op ? 'a' : 'd', u.src, u.dst, sign,
                       v.counts[s]);
          if (!v.listed) continue;
          const uint32_t w = v.widths[ql];
          for (uint64_t k = v.offsets[s]; k < v.offsets[s + 1]; k += w) {
            for (uint32_t j = 0; j < w; ++j) std::fprintf(out, j ? " %u" : "%u", v.tuples[k + j]);
            std::fputc('\n', out);
          }
        }
    }
    dsm_batch_release(e, id);
    std::fprintf(stderr, "batch %u: %u updates, %" PRIu64 " matches, %.3f ms\n", b, n, bm, ms);
    total_ms += ms;
    total_matches += bm;
    total_updates += n;
    pos += n;
  }
  if (serve) dsm_serve_stop(e);
  const double wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_loop).count();
  dsm_stats st;
  dsm_engine_stats(e, &st);
  std::fprintf(stderr, "total: %" PRIu64 " updates, %" PRIu64 " matches, %.3f ms wall (%.3e matches/s), "
               "batch latencies summed %.3f ms, device %.3f ms in the last device batch\n",
               total_updates, total_matches, wall_ms, wall_ms > 0 ? total_matches / (wall_ms / 1e3) : 0.0, total_ms,
               st.last_batch_ms);
  if (out != stdout) std::fclose(out);
  for (auto *q : queries) dsm_text_free(q);
  dsm_text_free(g);
  dsm_engine_destroy(e);
  return 0;
}
