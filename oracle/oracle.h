/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement, on the CPU, of the continuous subgraph matching
 * semantics of qxk152/DSM.  It is the checker for the CUDA engine in
 * dsm_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it, and never as the thing that is measured or shipped.
 *
 * Pieces and the reference code each one restates:
 *   - text parser                 io.cu:122-252 (readGraphToCPUDynamic)
 *   - batch application           cpuGraph.cpp:521-607 (updateHostGraph), set semantics
 *   - decycle (spanning tree)     decycle.cpp:6-135
 *   - matching order              order.cpp:367-402 (getVertexOrderBFS),
 *                                 order.cpp:647-676 (constructBackwardNeighbors)
 *   - LDF/NLF candidate filter    filter.cu:394-613
 *   - cluster encoding filter     filter.cu:23-392 (vertex cover, clustering),
 *                                 filter.cu:615-1177 (encode / merge / combine),
 *                                 filter.cu:1582-1609 (position pick),
 *                                 filter.cu:1692-1749 (compact to per-u bitmaps)
 *   - seeding + expansion         main.cu:268-329, gpu_match.cu:947-1118
 *
 * Per-update semantics (the reference emits no embeddings, so this is the
 * defined contract): an embedding is an injective, label-preserving map f from
 * query vertices to data vertices with every query edge mapped onto a data
 * edge (non-induced, automorphic images counted separately).  With G_i the
 * graph after updates 1..i in stream order:
 *   insert e at i (e absent before):  P_i = { f in G_i     : e in f(E(Q)) }
 *   delete e at i (e present before): N_i = { f in G_{i-1} : e in f(E(Q)) }
 *   no-op update (insert of a present edge, delete of an absent edge,
 *   self loop): empty.
 * Tuples are (f(0), ..., f(nq-1)) and each update's set is sorted
 * lexicographically.
 */
#ifndef DSM_ORACLE_H
#define DSM_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_file orc_file;
typedef struct orc_stream orc_stream;

/* ---- text formats (io.cu:122-252) ---------------------------------- */
/* Parse a query (is_query=1) or data graph file.  Returns 0 or -1. */
int orc_file_parse(const char *path, int is_query, orc_file **out);
void orc_file_free(orc_file *f);
uint32_t orc_file_nv(const orc_file *f);
uint32_t orc_file_ne(const orc_file *f);
const uint32_t *orc_file_labels(const orc_file *f);
const uint32_t *orc_file_offsets(const orc_file *f);   /* nv+1, from v-line degrees */
const uint32_t *orc_file_nbrs(const orc_file *f);      /* 2*ne, file order */
const uint32_t *orc_file_edges(const orc_file *f);     /* ne pairs (src,dst), file order */
uint32_t orc_file_num_batches(const orc_file *f);
const uint32_t *orc_file_batch_sizes(const orc_file *f);
uint32_t orc_file_num_updates(const orc_file *f);
/* updates flattened in stream order: op (1 add, 0 delete), src, dst, label */
const uint32_t *orc_file_updates(const orc_file *f);   /* 4 words per update */

/* ---- query preprocessing ------------------------------------------- */
/* decycle.cpp:6-135.  Writes the tree CSR (offsets nq+1, nbrs) and the
 * decremented degrees.  Returns the number of tree edges. */
int orc_decycle(uint32_t nq, const uint32_t *qoff, const uint32_t *qnbr,
                uint32_t *tree_off, uint32_t *tree_nbr, uint32_t *tree_deg);
/* order.cpp:367-402 + 647-676 on the FULL query, seeded with the ordered
 * query edge (u, v).  order[p] = query vertex at position p; bn_mask[p] =
 * bitmask over positions < p that are query neighbours of order[p]. */
int orc_order(uint32_t nq, const uint32_t *qoff, const uint32_t *qnbr,
              uint32_t u, uint32_t v, uint32_t *order, uint32_t *bn_mask);

/* ---- cluster-encoding filter (filter.cu) ---------------------------- */
/* Runs LDF/NLF + clustering + encode/merge/combine + compact on the data
 * graph given as a sorted CSR.  bitmaps: nq * ceil(nv/32) words (u-major,
 * the reference's compact layout).  v_cand_us: nv words (bit u set when v
 * passes LDF/NLF for u).  Optional out-params may be NULL.
 * plan_out (optional, 4096 words): the op sequence the encoder ran, one
 * record of 8 words per op: kind (0 encode, 1 merge, 2 combine), cluster,
 * a, b, c, d, e, f (see oracle.cpp). plan_len_out = number of ops.
 * Returns 0, or -2 when the query exceeds the reference's limits. */
/* The cluster plan alone (vertex cover, clusters, merges, combines, layer
 * offsets, enc_pos_of_u) of the decycled query, serialised as the reference
 * harness's ref_cluster_plan does; returns words written or < 0. */
int orc_cluster_plan(uint32_t nq, const uint32_t *qoff, const uint32_t *qnbr, uint32_t *out, uint32_t cap);
int orc_cluster_filter(uint32_t nq, const uint32_t *qlabels, const uint32_t *qoff,
                       const uint32_t *qnbr, uint32_t nv, const uint32_t *labels,
                       const uint32_t *off, const uint32_t *nbr, uint32_t *bitmaps,
                       uint32_t *v_cand_us, uint32_t *enc_pos_of_u,
                       uint32_t *plan_out, uint32_t *plan_len_out);

/* ---- continuous matching stream ------------------------------------ */
/* Data graph from an undirected edge list (duplicates and self loops
 * dropped, as the set rebuild in cpuGraph.cpp:545-588 does). */
int orc_stream_new(uint32_t nv, const uint32_t *labels, uint64_t ne,
                   const uint32_t *edges /* ne pairs */, uint32_t nq,
                   const uint32_t *qlabels, const uint32_t *qoff,
                   const uint32_t *qnbr, orc_stream **out);
void orc_stream_free(orc_stream *s);
/* Apply n updates (4 words each: op, src, dst, label) one at a time.
 * list=0 counts only.  Results of this call replace the previous ones. */
int orc_stream_apply(orc_stream *s, uint32_t n, const uint32_t *updates, int list);
/* Work budget in algorithmic bytes per apply call.  Once passed, the call
 * still applies every update to the graph but enumerates no further: the
 * first orc_stream_complete() updates have full results, the rest have
 * count 0, and apply returns 1.  Lets tests afford explosive updates. */
void orc_stream_set_budget(orc_stream *s, uint64_t bytes);
/* orc_stream_apply on `threads` host threads (< 1: all cores): the same
 * results; updates apply in order, each update's search is shared among the
 * threads.  No work budget. */
int orc_stream_apply_mt(orc_stream *s, uint32_t n, const uint32_t *updates, int list, int threads);
/* Bound on each update's search (0: none, the default): the valid partial
 * embeddings of 3 or more query vertices it generates, embeddings included
 * -- the engine's DSM_OPT_WORK_LIMIT.  An update whose search reaches it
 * stops; its count then has bit 63 set and it lists nothing. */
void orc_stream_set_work_limit(orc_stream *s, uint64_t limit);
/* Replaces the stream's query (the graph stays): one graph, many queries. */
int orc_stream_set_query(orc_stream *s, uint32_t nq, const uint32_t *qlabels, const uint32_t *qoff,
                         const uint32_t *qnbr);
/* The count update (op, a, b) would report if it were applied now (on
 * `threads` host threads, < 1: all cores); the graph is left unchanged.  An
 * insert of a present edge, a delete of an absent one or a self loop: 0. */
uint64_t orc_stream_probe(orc_stream *s, uint32_t op, uint32_t a, uint32_t b, int threads);
/* Applies the updates to the graph only (no matching). */
int orc_stream_apply_graph(orc_stream *s, uint32_t n, const uint32_t *updates);
uint32_t orc_stream_complete(const orc_stream *s);
int8_t orc_stream_sign(const orc_stream *s, uint32_t i);
uint64_t orc_stream_count(const orc_stream *s, uint32_t i);
/* Tuples of the last apply, concatenated in update order, nq words each. */
const uint32_t *orc_stream_tuples(const orc_stream *s, uint64_t *num_tuples);
/* Number of embeddings of the query in the current graph (backtracking). */
uint64_t orc_stream_count_all(const orc_stream *s);
/* Sorted CSR export: off has nv+1 words; nbr may be NULL to size it. */
uint64_t orc_stream_export(const orc_stream *s, uint32_t *off, uint32_t *nbr);
/* Algorithmic bytes the last apply touched (adjacency reads, probes,
 * emitted words) under the same order and algorithm. */
uint64_t orc_stream_bytes(const orc_stream *s);

/* All injective label-preserving maps checked one by one (tiny graphs). */
uint64_t orc_bruteforce_count(uint32_t nq, const uint32_t *qlabels, const uint32_t *qoff,
                              const uint32_t *qnbr, uint32_t nv, const uint32_t *labels,
                              const uint32_t *off, const uint32_t *nbr);

#ifdef __cplusplus
}
#endif
#endif
