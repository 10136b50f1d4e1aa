// Launch wrappers of the engine's kernels (host side).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace dsm {

// Sizes of the current batch.  The batch kernels read them from device
// memory (and loop over them with fixed grids), so one captured CUDA graph
// serves batches of every size.
struct BatchHdr {
  uint32_t n;                   // updates
  uint32_t m;                   // updates that are not self loops (undirected keys)
  uint32_t ngroups;             // source groups of the directed pairs
  uint32_t nq_live;             // queries matched
  unsigned long long seed_cap;  // seed table capacity
  unsigned long long nseg;      // nq_live * n counters
};

// Clears what a batch must start from: view times (kNoView), per-(query,
// update) counts, per-query listing counters, the scheduler and the error
// word.  Sizes from the header.
struct ClearArgs {
  const BatchHdr *hdr;
  uint32_t *vtp;
  unsigned long long *segcnt;
  unsigned long long *segwork;  // null: no work limit this batch
  unsigned long long *qlisted;
  Sched *sc;
  uint32_t *misc;  // 64 words
};
void launch_batch_clear(const ClearArgs &a, int blocks, cudaStream_t s);

// Batch edge state: for each group of equal canonical keys (sorted), walks
// the group's updates in order from the initial presence of the edge.
struct EdgeStateArgs {
  DevGraph g;
  const BatchHdr *hdr;            // m, n
  const uint4 *upd;               // [n] op, src, dst, label (batch order)
  const unsigned long long *bkey; // [m] sorted canonical keys (self loops excluded)
  const uint32_t *bidx;           // [m] update index per sorted entry
  uint32_t *binfo;                // [m] idx | op << 30 | init << 31
  uint8_t *gflag;                 // [m] 1: union insert, 2: final delete
  uint32_t *vtp;                  // [n] view time (updates applied) or kNoView
};
void launch_edge_state(const EdgeStateArgs &a, int blocks, cudaStream_t s);

// Merge (insert) or remove (delete) neighbours per source vertex.  dkey is
// sorted (src << 32 | dst); dhead[g] is the first entry of source group g
// (dhead[ngroups] = total).  Selection of the entries that apply reads the
// group flags of the undirected table.
struct AdjUpdateArgs {
  DevGraph g;
  const BatchHdr *hdr;            // ngroups, m
  const unsigned long long *dkey;
  const uint32_t *dhead;
  const unsigned long long *bkey;
  const uint8_t *gflag;
  uint32_t *dsel;                 // scratch, same length as dkey
  unsigned int *err;
  unsigned long long *relocations;
  unsigned long long *need16;     // [0]: arena units the batch may relocate, [1]: arena top before it
};
// Before the insert: the arena units the batch's relocated runs may need (an
// upper bound: every union insert counted); the insert then either has room
// for all of them or writes nothing and flags kErrArena, and so do the
// deletions and the matcher.
void launch_arena_check(const AdjUpdateArgs &a, int blocks, cudaStream_t s);
void launch_adj_insert(const AdjUpdateArgs &a, int blocks, cudaStream_t s);
// Compaction: copies every run to its new place (nadj: {start in 16-byte
// units, degree} per vertex) in another arena.
void launch_arena_move(DevGraph g, const uint2 *nadj, uint32_t *narena, int blocks, cudaStream_t s);
void launch_adj_delete(const AdjUpdateArgs &a, int blocks, cudaStream_t s);
void launch_clear_touch(DevGraph g, const BatchHdr *hdr, const uint4 *upd, int blocks, cudaStream_t s);

// Seeds: one per (update, ordered query edge whose end labels match).
struct SeedArgs {
  DevGraph g;
  const BatchHdr *hdr;        // n, seed_cap
  const uint4 *upd;
  const uint32_t *vtp;
  const uint32_t *pair_off;   // [32*32+1] label pair -> entries
  const uint32_t *pair_ent;   // slot << 8 | ordered edge
  const QDev *qd;
  const OrderRec *orders;
  uint4 *seeds;               // {update, slot<<8|o, a, b}
  Sched *sc;
  uint32_t only_slot;         // seeds of this query slot only (kAllSlots: every query)
};
constexpr uint32_t kAllSlots = 0xFFFFFFFFu;
void launch_seeds(const SeedArgs &a, int blocks, cudaStream_t s);

struct MatchArgs {
  DevGraph g;
  DevBatchEdges bt;               // bt.n (keys) is read from hdr->m
  const BatchHdr *hdr;            // n (segment index = query's local index * n + update)
  const uint32_t *vtp;
  const QDev *qd;
  const OrderRec *orders;
  const uint4 *seeds;
  Sched *sc;
  JobRec *jobs;                  // ring of job records
  unsigned long long *job_seq;   // per slot: p = free for position p, t + 1 = job
                                 // for ticket t, t | kSeqDone = no more work
  uint32_t job_ring;             // slots, a power of two
  uint32_t *out_seg;
  uint32_t *out_tup;
  uint32_t W;
  unsigned long long cap;
  unsigned long long *seg_count;
  // listing budget per query and batch: a query that would list more than
  // qlimit tuples (0 = no budget) lists no more; qlisted[local] counts the
  // tuples each query asked to list, so the host knows which went over
  unsigned long long *qlisted;
  unsigned long long qlimit;
  // work limit per (query, update) segment (0 = none): see run_task
  unsigned long long work_limit;
  unsigned long long *seg_work;    // [nseg] partial embeddings generated so far
  const unsigned int *abort_flag;  // non-zero (kErrArena): the batch was refused, match nothing
  int list;
  int donate;
  long long timeout_cycles;
  // donation granularity (0 = default): a remaining pivot range is split
  // when it holds at least split_min entries (>= 64); pending candidates are
  // donated when at least donate_depth levels lie below them (1..4)
  uint32_t split_min;
  uint32_t donate_depth;
  // packed last level (label-major runs): at most this many entries laid end
  // to end in one pass over a chunk's candidates (0: candidates one at a time)
  uint32_t pack_max;
  // merge intersection: a probe range of at most this many entries is
  // walked in tiles against the whole chunk instead of searched per entry
  // (0: always searched)
  uint32_t merge_max;
  // breadth-first rows: in a launch with bfs_stop > 0, a task that finds
  // candidates completing bfs_stop positions (with at least two positions
  // left) writes each prefix as a row to rows_out instead of descending,
  // while the table has room (then it descends as usual); a launch with
  // rows_in takes its tasks from those rows instead of the seeds
  uint32_t bfs_stop;
  JobRec *rows_out;
  unsigned long long *rows_cnt;
  unsigned long long rows_cap;
  const JobRec *rows_in;
};
// Arms a matcher launch: outstanding = seeds (+ phantom, a task nothing
// finishes: a test hook), every ring slot free for its first position.
void launch_sched_init(Sched *sc, const BatchHdr *hdr, unsigned long long *job_seq, uint32_t job_ring,
                       cudaStream_t s, uint32_t phantom = 0);
void launch_match(const MatchArgs &a, int blocks, cudaStream_t s);
// Between the two launches of a breadth-first plan: the scheduler restarts
// with the rows written so far as its tasks (counters of work done, the
// result-table position and the error word carry over).
void launch_rows_arm(Sched *sc, const unsigned long long *rows_cnt, unsigned long long rows_cap, cudaStream_t s);
int match_max_blocks_per_sm();

}  // namespace dsm
