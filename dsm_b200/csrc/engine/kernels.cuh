// Launch wrappers of the engine's kernels (host side).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace dsm {

// Batch edge state: for each group of equal canonical keys (sorted), walks
// the group's updates in order from the initial presence of the edge.
struct EdgeStateArgs {
  DevGraph g;
  const uint4 *upd;               // [n] op, src, dst, label (batch order)
  const unsigned long long *bkey; // [m] sorted canonical keys (self loops excluded)
  const uint32_t *bidx;           // [m] update index per sorted entry
  uint32_t m, n;
  uint32_t *binfo;                // [m] idx | op << 30 | init << 31
  uint8_t *gflag;                 // [m] 1: union insert, 2: final delete
  uint32_t *vtp;                  // [n] view time (updates applied) or kNoView
};
void launch_edge_state(const EdgeStateArgs &a, cudaStream_t s);

// Merge (insert) or remove (delete) neighbours per source vertex.  dkey is
// sorted (src << 32 | dst); dhead[g] is the first entry of source group g
// (dhead[ngroups] = total).  Selection of the entries that apply reads the
// group flags of the undirected table.
struct AdjUpdateArgs {
  DevGraph g;
  const unsigned long long *dkey;
  const uint32_t *dhead;
  uint32_t ngroups;
  const unsigned long long *bkey;
  const uint8_t *gflag;
  uint32_t m;
  uint32_t *dsel;                 // scratch, same length as dkey
  unsigned int *err;
  unsigned long long *relocations;
};
void launch_adj_insert(const AdjUpdateArgs &a, cudaStream_t s);
void launch_adj_delete(const AdjUpdateArgs &a, cudaStream_t s);
void launch_clear_touch(DevGraph g, const uint4 *upd, uint32_t n, cudaStream_t s);

// Seeds: one per (update, ordered query edge whose end labels match).
struct SeedArgs {
  DevGraph g;
  const uint4 *upd;
  const uint32_t *vtp;
  uint32_t n;
  const uint32_t *pair_off;   // [32*32+1] label pair -> entries
  const uint32_t *pair_ent;   // slot << 8 | ordered edge
  const QDev *qd;
  const OrderRec *orders;
  uint4 *seeds;               // {update, slot<<8|o, a, b}
  unsigned long long seed_cap;
  Sched *sc;
};
void launch_seeds(const SeedArgs &a, cudaStream_t s);

struct MatchArgs {
  DevGraph g;
  DevBatchEdges bt;
  const uint32_t *vtp;
  uint32_t n;
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
  int list;
  int donate;
  long long timeout_cycles;
  // donation granularity (0 = default): a remaining pivot range is split
  // when it holds at least split_min entries (>= 64); pending candidates are
  // donated when at least donate_depth levels lie below them (1..4)
  uint32_t split_min;
  uint32_t donate_depth;
};
// Arms a matcher launch: outstanding = seeds (+ phantom, a task nothing
// finishes: a test hook), every ring slot free for its first position.
void launch_sched_init(Sched *sc, unsigned long long seed_cap, unsigned long long *job_seq, uint32_t job_ring,
                       cudaStream_t s, uint32_t phantom = 0);
void launch_match(const MatchArgs &a, int blocks, cudaStream_t s);
int match_max_blocks_per_sm();

}  // namespace dsm
