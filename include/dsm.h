/*
 * dsm.h -- C ABI of the B200 continuous subgraph matching engine.
 *
 * Plain pointers and sizes only.  Every call returns a status code
 * (DSM_OK or one of DSM_ERR_*); nothing in the library calls exit().
 * The reference (qxk152/DSM) exposes no library interface: its internal
 * call boundaries, each named beside the entry point that replaces it, are
 * process-global functions that exit() on error and keep their sizes in
 * host globals and __constant__ symbols, so one query per process.
 *
 * One engine = one device, one CUDA stream, one data graph, any number of
 * registered queries.  Calls on one engine are serialised internally
 * (mutexes), so the ABI is thread-safe per engine; with the serving loop
 * running, batches and query changes go through its submission queue.
 */
#ifndef DSM_H
#define DSM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define DSM_OK 0
#define DSM_ERR_PARSE 1    /* malformed text input */
#define DSM_ERR_OOM 2      /* device memory budget or allocation exhausted */
#define DSM_ERR_OVERFLOW 3 /* a result / queue capacity was exceeded and could not grow */
#define DSM_ERR_TIMEOUT 4  /* a bounded device wait gave up */
#define DSM_ERR_LIMIT 5    /* input beyond a supported size (query > 16 vertices, label >= 32, ...) */
#define DSM_ERR_ARG 6      /* bad argument (null pointer, id out of range) */
#define DSM_ERR_CUDA 7     /* CUDA runtime error */
#define DSM_ERR_STATE 8    /* call not valid in the current state */
#define DSM_ERR_NOT_FOUND 9

typedef struct dsm_engine dsm_engine;

/* One edge update, the reference's `change` (cpuGraph.h:13-18) plus its op
 * letter: op 1 = 'a' (insert), 0 = 'd' (delete).  label is the data file's
 * 4th field; labels stay fixed unless DSM_OPT_LABEL_QUIRK is set. */
typedef struct dsm_update {
  uint32_t op;
  uint32_t src;
  uint32_t dst;
  uint32_t label;
} dsm_update;

/* ---- engine ----------------------------------------------------------- */
/* Replaces main.cu:47-55 (device selection) and the process globals of
 * globals.cu:4-74.  mem_budget = 0 means "free device memory minus 1 GiB". */
int dsm_engine_create(int device, size_t mem_budget, dsm_engine **out);
int dsm_engine_destroy(dsm_engine *e);
const char *dsm_status_string(int status);
/* Text of the last error on this engine ("" if none); the pointer stays
 * valid until the calling thread's next dsm_last_error. */
const char *dsm_last_error(dsm_engine *e);

/* Options (dsm_engine_set_option). */
#define DSM_OPT_LIST 1          /* 1: list embeddings (default); 0: counts only */
#define DSM_OPT_FILTER 2        /* 0: labels only (default); 1: LDF+NLF; 2: cluster encoding */
#define DSM_OPT_RESULT_CAP 3    /* initial result capacity in tuples (grows on overflow) */
#define DSM_OPT_WARPS_PER_SM 4  /* persistent matcher warps per SM (0: as many as fit) */
#define DSM_OPT_DONATE 5        /* 0 disables work donation between warps */
#define DSM_OPT_TIMEOUT_MS 6    /* bound on every device-side wait (default 5000) */
#define DSM_OPT_LABEL_QUIRK 7   /* 1: an insert relabels both endpoints (cpuGraph.cpp:564) */
#define DSM_OPT_SORT 8          /* 1: canonically sort each update's tuples (default) */
#define DSM_OPT_LIST_LIMIT 9    /* bytes of tuples one batch may list; beyond it the batch
                                   returns exact counts only and its view has listed = 0 */
#define DSM_OPT_MEM_BUDGET 10   /* device memory budget in bytes (>= bytes in use); raising it
                                   admits queries that waited for memory */
#define DSM_OPT_SPLIT_MIN 11    /* work donation: split a remaining pivot range of at least
                                   this many entries (0 = default 128; else >= 64) */
#define DSM_OPT_DONATE_DEPTH 12 /* work donation: hand out pending candidates with at least
                                   this many levels below them (0 = default 2; 1..4) */
#define DSM_OPT_AUTOTUNE 13     /* 1: the next batch times its matcher launch under each
                                   candidate setting on its own union graph -- first the
                                   plan (DSM_OPT_BFS_LEVELS in {0, 1, 2}), then the
                                   intersection tile (DSM_OPT_PACK_MAX in {0, 256, 1024,
                                   4096} x DSM_OPT_MERGE_MAX in {0, 64, 256}), then resident
                                   blocks per SM x split threshold x donation depth -- and
                                   keeps the fastest in DSM_OPT_BFS_LEVELS /
                                   DSM_OPT_PACK_MAX / DSM_OPT_MERGE_MAX /
                                   DSM_OPT_WARPS_PER_SM / DSM_OPT_SPLIT_MIN /
                                   DSM_OPT_DONATE_DEPTH; its results
                                   are those of any setting.  Reads 1 until that batch ran. */
#define DSM_OPT_GRAPH 14        /* 1: each batch's two device segments (uploads .. matcher, and
                                   deletes .. downloads) are captured into CUDA graphs and
                                   launched through one executable graph per segment, updated
                                   in place while the topology repeats (default 0) */
#define DSM_OPT_STALL_TEST 15   /* test hook (default 0): 1 arms every matcher launch with one
                                   extra outstanding task that no warp ever finishes, so the
                                   launch ends only when its idle warps' bounded waits run out
                                   (DSM_OPT_TIMEOUT_MS without progress) and the batch returns
                                   DSM_ERR_TIMEOUT after applying its updates to the graph.
                                   Tests the failure path without faulting the device. */
#define DSM_OPT_PLAIN 16        /* 1: each batch runs the matcher once per registered query, in
                                   turn, with a host round trip after each launch -- the
                                   reference's one-query-per-process form, kept as the baseline
                                   of the batched form; results identical (default 0) */
#define DSM_OPT_QUERY_LIST_LIMIT 17 /* tuples one query may list in one batch (0: no limit,
                                   the default).  A query over it is reported with exact
                                   counts and no tuples for that batch (query_listed = 0 in
                                   the view); the other queries stay listed. */
#define DSM_OPT_WORK_LIMIT 18   /* bound on the search of one (query, update): the number of
                                   partial embeddings of 3 or more query vertices it
                                   generates, embeddings included (0: no bound, the
                                   default).  That number depends only on the graph, the
                                   query and the matching order -- not on scheduling -- so
                                   whether a (query, update) reaches the bound is
                                   deterministic.  One that does stops early: its count in
                                   the result view has bit 63 set (low bits: a partial
                                   count) and it lists no tuples.  Every other count stays
                                   exact.  (With DSM_OPT_FILTER > 0 the filter prunes
                                   partial embeddings, so fewer reach the bound.) */
#define DSM_OPT_FILTER_INCREMENTAL 20 /* 1 (default): a batch's filter recomputes only the
                                   data vertices within (the query's op count) hops of
                                   the endpoints of its own and the previous batch's
                                   updates, falling back to every vertex when that region
                                   is large or the query's state is not the previous
                                   batch's; 0: every vertex, every batch.  Same bitmaps. */
#define DSM_OPT_MERGE_MAX 21     /* matcher set intersection: a backward neighbour's label range
                                   of at most this many entries is intersected with a whole
                                   32-entry chunk by a ballot/shuffle merge over 32-entry tiles
                                   instead of a binary search per entry (default 64; 0: always
                                   searched; at most 4096).  Results do not depend on it. */
#define DSM_OPT_BFS_LEVELS 22    /* matcher plan: 0 (default) depth-first from the seeds; k in 1..8:
                                   the first launch expands every seed breadth-first to
                                   prefixes of 2 + k query vertices, written as rows (while
                                   the row table has room, depth-first beyond it), and a
                                   second launch matches depth-first from those rows -- the
                                   reference's BFS join before its DFS matcher
                                   (gpu_match.cu:1291-1357, join.cu:106-221).  Results do not
                                   depend on it; DSM_OPT_AUTOTUNE tries 0, 1 and 2. */
#define DSM_OPT_BFS_ROWS 23      /* row table capacity for DSM_OPT_BFS_LEVELS (default 2^20
                                   rows of 128 bytes) */
#define DSM_OPT_PACK_MAX 19     /* matcher intersection tile: the candidates one 32-entry
                                   chunk leaves at the second-to-last query vertex have
                                   their last-level ranges laid end to end and scanned
                                   together when they total at most this many entries
                                   (default 1024; 0: each candidate scanned on its own;
                                   at most 2^20).  Results do not depend on it. */
int dsm_engine_set_option(dsm_engine *e, int option, int64_t value);
int dsm_engine_get_option(dsm_engine *e, int option, int64_t *value);

/* ---- data graph ------------------------------------------------------- */
/* Replaces readGraphToCPUDynamic's CSR hand-off + allocateMemGPU /
 * copyGraphToGPU (io.cuh:19-31, io.cu:254-302).  The CSR may be in file
 * order with duplicates; every entry (v, w) is read as the undirected edge
 * {v, w}; self loops are dropped.  The device keeps sorted lists with slack. */
int dsm_graph_load(dsm_engine *e, const uint32_t *offsets, const uint32_t *nbrs,
                   const uint32_t *labels, uint32_t nv);
/* Same, from an undirected edge list (ne pairs). */
int dsm_graph_load_edges(dsm_engine *e, uint32_t nv, const uint32_t *labels, uint64_t ne,
                         const uint32_t *edges);
/* Current graph as a sorted CSR (offsets: nv+1 words; nbrs may be NULL to
 * learn *num_entries first).  Parity hook for updateHostGraph
 * (cpuGraph.cpp:521-607): the device lists must equal the set rebuild. */
int dsm_graph_export(dsm_engine *e, uint32_t *offsets, uint32_t *nbrs, uint64_t *num_entries);
int dsm_graph_info(dsm_engine *e, uint32_t *nv, uint64_t *num_entries, uint64_t *arena_words);
/* Applies a batch of updates to the device graph without matching, in array
 * order with set semantics -- updateHostGraph (cpuGraph.cpp:521-607) plus the
 * re-upload of copyGraphToGPU (io.cu:254-302), as one device step.  Not
 * available while the serving loop runs (DSM_ERR_STATE). */
int dsm_graph_apply(dsm_engine *e, const dsm_update *ups, uint32_t n);

/* ---- queries ---------------------------------------------------------- */
/* Query CSR as read from a query file (file order, io.cu:181-189).  The
 * host side runs decycle (decycle.cpp:6-135), the clustering plan of the
 * cluster-encoding filter (filter.cu:23-392) and one matching order per
 * ordered query edge (order.cpp:367-402, 647-676), then uploads a
 * descriptor.  Admission: fails with DSM_ERR_OOM when the query's device
 * footprint does not fit the engine's memory budget. */
int dsm_query_register(dsm_engine *e, const uint32_t *q_offsets, const uint32_t *q_nbrs,
                       const uint32_t *q_labels, uint32_t nq, uint32_t *qid);
/* Ends matching for qid; a later registration may reuse the id. */
int dsm_query_retire(dsm_engine *e, uint32_t qid);
/* The ids of the registered queries, ascending: *num = their number; up to
 * cap of them are written to qids (which may be NULL to learn *num). */
int dsm_query_live(dsm_engine *e, uint32_t *qids, uint32_t cap, uint32_t *num);
/* Matching order for ordered query edge (u, v): order[p] = query vertex at
 * position p; bn_mask[p] = positions < p adjacent to it (OrderCPU's
 * v_orders / backward_neighbors, order.h:78-111). */
int dsm_query_order(dsm_engine *e, uint32_t qid, uint32_t u, uint32_t v, uint32_t *order,
                    uint32_t *bn_mask);
/* Runs the candidate filter of query qid on the current graph and copies the
 * per-u candidate bitmaps (nq * ceil(nv/32) words, u-major) -- the output of
 * clusterFilter + compact (filter.cuh:119-137).  v_cand_us (nv words, may be
 * NULL): bit u set when v passes LDF+NLF for u (d_v_candidate_us_). */
int dsm_query_filter(dsm_engine *e, uint32_t qid, uint32_t *bitmaps, uint32_t *v_cand_us);
/* The filter state the last batch left for query qid (DSM_OPT_FILTER > 0),
 * without recomputing it: the bitmaps and v_cand_us as dsm_query_filter
 * gives them, for that batch's union graph.  info (2 words, may be NULL):
 * info[0] = 1 if that run recomputed every data vertex, 0 if it recomputed
 * only the incremental region; info[1] = data vertices it recomputed.  No
 * reference counterpart: the reference recomputes the whole filter every
 * batch (main.cu:213, filter.cu:1525-1654). */
int dsm_query_filter_state(dsm_engine *e, uint32_t qid, uint32_t *bitmaps, uint32_t *v_cand_us, uint32_t *info);

/* Host only (no engine, no GPU): the plan the engine would build for a
 * query.  orders / bn_masks: one row of nq words per ordered query edge, in
 * CSR order; oedges: (u, v) per row; enc_pos_of_u: the encoding position
 * whose bit is u's candidacy (filter.cu:1582-1609).  Outputs may be NULL. */
int dsm_query_plan(const uint32_t *q_offsets, const uint32_t *q_nbrs, const uint32_t *q_labels,
                   uint32_t nq, uint32_t *orders, uint32_t *bn_masks, uint32_t *oedges,
                   uint32_t *num_oedges, uint32_t *enc_pos_of_u);

/* ---- update batches -------------------------------------------------- */
/* Replaces one iteration of the batch loop main.cu:152-347 (updateHostGraph,
 * re-upload, re-filter, seeding, the matcher of gpu_match.cu/join.cu) for all
 * registered queries at once.  Updates apply in array order with sequential
 * semantics: an insert's positive matches are taken on the graph after it,
 * a delete's negative matches on the graph before it.  Without the serving
 * loop the call runs the batch to completion (one device batch per call,
 * the reference's plain form); with it (dsm_serve_start) the call only
 * queues the batch and returns its id. */
int dsm_batch_submit(dsm_engine *e, const dsm_update *ups, uint32_t n, uint64_t *batch_id);
/* Blocks until the batch's results are on the host.  A batch that failed
 * reports its error to the first wait (or results / timing call) only; the
 * engine then forgets it. */
int dsm_batch_wait(dsm_engine *e, uint64_t batch_id);

typedef struct dsm_result_view {
  uint64_t batch_id;
  uint32_t num_updates;
  uint32_t num_queries;
  const uint32_t *qids;     /* [num_queries], ascending */
  const uint32_t *widths;   /* [num_queries]: tuple width = query vertex count */
  const int8_t *signs;      /* [num_updates]: +1 insert, -1 delete, 0 no-op update */
  const uint64_t *counts;   /* [num_queries * num_updates], query-major; bit 63 set:
                               the search went over DSM_OPT_WORK_LIMIT (partial count) */
  const uint64_t *offsets;  /* [num_queries * num_updates + 1]: word offsets into tuples */
  const uint32_t *tuples;   /* (f(0)..f(nq-1)) per embedding, each segment sorted */
  int listed;               /* 0 when the batch ran with DSM_OPT_LIST = 0 (or over the
                               batch listing limit): counts only */
  const uint8_t *query_listed; /* [num_queries]: 1 when that query's tuples are listed
                               (0 past DSM_OPT_QUERY_LIST_LIMIT: its segments are empty) */
} dsm_result_view;
/* Waits if needed; the view stays valid until dsm_batch_release. */
int dsm_batch_results(dsm_engine *e, uint64_t batch_id, dsm_result_view *view);
int dsm_batch_release(dsm_engine *e, uint64_t batch_id);

/* Latency of one submitted batch (host steady clock), available once it is
 * done and until it is released. */
typedef struct dsm_batch_timing {
  double queue_ms;            /* submit -> its device batch started */
  double service_ms;          /* device batch started -> results readable */
  double total_ms;            /* submit -> results readable */
  double device_ms;           /* device time of its device batch (events) */
  uint32_t merged_requests;   /* submitted batches served by that device batch */
  uint32_t merged_updates;    /* updates in that device batch */
} dsm_batch_timing;
int dsm_batch_timing_get(dsm_engine *e, uint64_t batch_id, dsm_batch_timing *t);

/* ---- serving loop ----------------------------------------------------- */
/* No counterpart in the reference (its main loop handles one query and one
 * batch at a time, main.cu:152-347).  dsm_serve_start starts one worker
 * thread per engine that serves requests in submission order:
 * dsm_batch_submit then only queues the batch and returns its id; batches
 * that are queued back to back run as ONE device batch of up to
 * max_merge_updates updates (0 = 65536), whose per-update results equal
 * those of running them one by one (each update still sees exactly the
 * updates before it); registrations and retirements take effect between
 * device batches, in submission order.  Admission: a query is charged its
 * device footprint (descriptor, orders, filter bitmaps and encodings); one
 * that does not fit the memory budget now waits, first come first served,
 * until retirements free enough, and one that could never fit fails with
 * DSM_ERR_OOM.  While serving, dsm_query_register and dsm_query_retire queue
 * their request and block until it took effect.  dsm_serve_stop serves what
 * is queued, then joins the worker (registrations still waiting for memory
 * fail with DSM_ERR_OOM).  The device batch limits (listing limit, result
 * capacity) apply to the merged batch. */
int dsm_serve_start(dsm_engine *e, uint32_t max_merge_updates);
int dsm_serve_stop(dsm_engine *e);
/* Queues a registration; *ticket names it for dsm_query_admission. */
int dsm_query_register_async(dsm_engine *e, const uint32_t *q_offsets, const uint32_t *q_nbrs,
                             const uint32_t *q_labels, uint32_t nq, uint64_t *ticket);
/* Queues a retirement; its ticket's outcome is reported like a registration's. */
int dsm_query_retire_async(dsm_engine *e, uint32_t qid, uint64_t *ticket);
/* Waits up to timeout_ms (< 0: no limit) for a ticket's outcome: DSM_OK
 * (with *qid: the admitted or retired query) once it took effect,
 * DSM_ERR_TIMEOUT while it still waits, else the request's error.  Each
 * outcome is reported once; the engine then forgets the ticket and a second
 * call for it returns DSM_ERR_NOT_FOUND. */
int dsm_query_admission(dsm_engine *e, uint64_t ticket, int64_t timeout_ms, uint32_t *qid);

/* ---- snapshot / resume ---------------------------------------------- */
/* No counterpart in the reference (its graph lives as long as one process).
 * dsm_engine_snapshot writes the current data graph (sorted CSR and labels),
 * every registered query with its id, and the batch counter to one file;
 * taken between device batches, it covers exactly the batches that finished
 * before it (queued ones are not in it).  dsm_engine_resume loads such a
 * file into an engine with no registered queries and the serving loop
 * stopped: afterwards the same update batches give the same results as on
 * the engine that wrote it. */
int dsm_engine_snapshot(dsm_engine *e, const char *path);
int dsm_engine_resume(dsm_engine *e, const char *path);

/* ---- counting without allocating ------------------------------------- */
/* No counterpart in the reference: an entry point for callers that must not
 * allocate device memory while they run -- code living inside a framework
 * that owns the device allocator and forbids side allocations, or a thread
 * that must not call cudaMalloc / cudaFree because those calls synchronise
 * the whole device.  It needs no engine: the caller passes a fixed graph,
 * the updates and the output, all in device memory, and the matcher's scratch
 * (scheduler counters, donation ring, seed table, query descriptor) lives in
 * one static device array of about 12.5 MB that every GPU loading this
 * library holds until the process exits.
 *
 * For each update i, d_counts[i] = the number of embeddings of the query that
 * map some query edge onto {src, dst} in the graph with that edge present
 * (the count an insert of the edge would report; the op and label fields are
 * not read).  src and dst must be vertex ids < nv and differ: an update
 * naming a vertex >= nv, or a self loop, counts 0 and reads no graph memory.
 *   graph: d_adj holds 2 words per vertex, {start of the vertex's run in
 *          16-byte units, degree}; the run d_arena[4*start .. 4*start+degree)
 *          lists its neighbours sorted ascending, without duplicates;
 *          d_labels[v] < 2^31.
 *   query: host CSR as for dsm_query_register, at most 8 vertices.
 *   limits: n <= 4096 updates (DSM_ERR_LIMIT beyond).
 *   stream: a cudaStream_t (NULL = the default stream); the call returns once
 *           the counts are written.
 * The first call on a device looks the static array's device address up
 * (cudaGetSymbolAddress, with `device` made current) and should come before
 * any stream capture.  Every call reuses the same array and clears what must
 * start at zero; calls whose work overlaps on the GPU race on it.  Nothing is
 * allocated: no cudaMalloc, no cudaFree. */
int dsm_count_edge_embeddings_noalloc(int device, uint32_t nv, const uint32_t *d_adj,
                                      const uint32_t *d_arena, const uint32_t *d_labels,
                                      const uint32_t *q_offsets, const uint32_t *q_nbrs,
                                      const uint32_t *q_labels, uint32_t nq,
                                      const dsm_update *d_updates, uint32_t n, uint64_t *d_counts,
                                      void *stream);

/* ---- statistics ------------------------------------------------------- */
typedef struct dsm_stats {
  uint64_t batches;
  uint64_t updates;
  uint64_t matches;          /* total |P| + |N| emitted (exact counts only) */
  uint64_t seeds;            /* (update, ordered query edge) tasks */
  uint64_t donations;        /* jobs handed from busy to idle warps */
  uint64_t steals;           /* jobs taken from the shared queue */
  uint64_t relocations;      /* adjacency lists moved for lack of slack */
  uint64_t result_regrows;   /* result-buffer overflows retried */
  uint64_t alg_bytes;        /* algorithmic bytes of the matcher (lists scanned, probes, output) */
  double last_batch_ms;      /* device time of the last batch (events) */
  double last_match_ms;      /* device time of the last matcher launch */
  double last_filter_ms;
  double last_update_ms;
  double last_sort_ms;
  uint64_t device_bytes_in_use;
  uint64_t kernel_launches;  /* engine kernels launched so far */
  uint64_t query_bytes;      /* device bytes charged to admitted queries */
  uint64_t live_queries;
  uint64_t tune_runs;        /* matcher launches timed by the autotuner */
  double tune_best_ms;       /* the fastest of them (last tuning) */
  uint64_t graph_launches;   /* segment graphs launched (DSM_OPT_GRAPH) */
  uint64_t graph_instantiations; /* executable graphs instantiated */
  uint64_t graph_captures;   /* segments captured (a replay reuses the last capture) */
  uint64_t compactions;      /* adjacency arena compactions */
  uint64_t over_limit;       /* (query, update) searches stopped by DSM_OPT_WORK_LIMIT */
} dsm_stats;
int dsm_engine_stats(dsm_engine *e, dsm_stats *s);

/* ---- text formats and workloads (host only, no GPU needed) ------------ */
typedef struct dsm_text dsm_text;
/* readGraphToCPUDynamic (io.cu:122-252); is_query=1 stops after the graph. */
int dsm_text_read(const char *path, int is_query, dsm_text **out, char *err, size_t err_len);
void dsm_text_free(dsm_text *t);
/* Binary form (no counterpart in the reference, whose `ifstream >>` text
 * reader dominates load time at 2^28 edges): the arrays below behind a
 * 64-byte header, each 64-byte aligned.  dsm_text_read recognises a binary
 * file by its magic and maps it (mmap, no parsing, no copy); the arrays are
 * those of the text file it was written from. */
int dsm_text_write_binary(const dsm_text *t, const char *path);
uint32_t dsm_text_nv(const dsm_text *t);
uint32_t dsm_text_ne(const dsm_text *t);
const uint32_t *dsm_text_labels(const dsm_text *t);
const uint32_t *dsm_text_offsets(const dsm_text *t);
const uint32_t *dsm_text_nbrs(const dsm_text *t);
const uint32_t *dsm_text_edges(const dsm_text *t);
uint32_t dsm_text_num_batches(const dsm_text *t);
const uint32_t *dsm_text_batch_sizes(const dsm_text *t);
uint32_t dsm_text_num_updates(const dsm_text *t);
const dsm_update *dsm_text_updates(const dsm_text *t);

typedef struct dsm_workload dsm_workload;
/* Seeded synthetic workload for configs 1-5.  scale_log2 < 0 shrinks the
 * graph by 2^-scale (vertices and edges), num_batches = 0 keeps the preset. */
int dsm_workload_generate(int config, uint64_t seed, int scale_log2, uint32_t num_batches,
                          dsm_workload **out);
void dsm_workload_free(dsm_workload *w);
uint32_t dsm_workload_nv(const dsm_workload *w);
const uint32_t *dsm_workload_labels(const dsm_workload *w);
uint64_t dsm_workload_num_edges(const dsm_workload *w);
const uint32_t *dsm_workload_edges(const dsm_workload *w);
uint32_t dsm_workload_num_queries(const dsm_workload *w);
uint32_t dsm_workload_query_nv(const dsm_workload *w, uint32_t q);
const uint32_t *dsm_workload_query_labels(const dsm_workload *w, uint32_t q);
const uint32_t *dsm_workload_query_offsets(const dsm_workload *w, uint32_t q);
const uint32_t *dsm_workload_query_nbrs(const dsm_workload *w, uint32_t q);
uint32_t dsm_workload_num_batches(const dsm_workload *w);
const uint32_t *dsm_workload_batch_sizes(const dsm_workload *w);
uint32_t dsm_workload_num_updates(const dsm_workload *w);
const dsm_update *dsm_workload_updates(const dsm_workload *w);
/* Writes query_prefix<q>.in per query and data_path in the reference format. */
int dsm_workload_write(const dsm_workload *w, const char *query_prefix, const char *data_path);

#ifdef __cplusplus
}
#endif
#endif /* DSM_H */
