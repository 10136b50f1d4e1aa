// Device-side types shared by the engine's kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../host/order_rec.h"

namespace dsm {

constexpr uint32_t kFull = 0xFFFFFFFFu;
constexpr uint32_t kTouchBit = 0x80000000u;  // label word bit: endpoint of an update in this batch
constexpr uint32_t kLabelMask = 0x7FFFFFFFu;
constexpr uint32_t kNoView = 0xFFFFFFFFu;     // view time of a no-op update

// Adjacency entries are label-major: entry = slot(label) << 27 | id, where
// slot(label) = min(label, 31), so a run sorted by entry value lists its
// neighbours by label, then id, and the neighbours with one label form one
// contiguous range.  Slot 31 is shared by every label >= 31; a query vertex
// with label 31 checks the exact label of what it takes from that slot.
constexpr uint32_t kIdBits = 27;
constexpr uint32_t kIdMask = (1u << kIdBits) - 1;
constexpr uint32_t kMaxVertices = 1u << kIdBits;
constexpr uint32_t kSlots = 32;
__host__ __device__ __forceinline__ uint32_t label_slot(uint32_t label) { return label < 31 ? label : 31; }
__host__ __device__ __forceinline__ uint32_t pack_entry(uint32_t label, uint32_t v) {
  return (label_slot(label) << kIdBits) | v;
}

// Data graph in HBM.  Each vertex owns a sorted run of entries in one arena;
// runs start on 16-byte boundaries and carry slack so that inserts merge in
// place.  adj[v] = {start in 16-byte units, degree}: one 8-byte load gives
// both.  loff[v * (nlt + 1) + s] = index in v's run of its first entry with
// slot >= s (s = 0..nlt; nlt = number of slots in use), so the neighbours of
// v with slot s are [loff[s], loff[s + 1]): one 8-byte read per lookup.
// loff == nullptr marks plain runs (neighbour ids sorted ascending), the
// layout callers of the allocation-free entry point pass.
struct DevGraph {
  uint32_t nv;
  uint32_t *lab;       // [nv] label | kTouchBit
  uint2 *adj;          // [nv] {off16, deg}
  uint32_t *cap;       // [nv] capacity in entries (multiple of 4)
  uint32_t *arena;     // entries
  uint32_t *loff;      // [nv * (nlt + 1)] slot offsets, or null for plain runs
  uint32_t nlt;
  uint64_t arena_words;
  unsigned long long *arena_top;  // next free 16-byte unit
};

__device__ __forceinline__ const uint32_t *adj_list(const DevGraph &g, uint2 a) {
  return g.arena + (uint64_t)a.x * 4;
}

// Sorted edge table of the batch, for "is edge {x,y} live after the first
// `tp` updates of the batch".  bkey: canonical keys (min << 32 | max) sorted,
// ties in update order; binfo: update index | op << 30 | initially-present << 31.
struct DevBatchEdges {
  const unsigned long long *bkey;
  const uint32_t *binfo;
  uint32_t n;  // keys (set by the matcher from the batch header)
};

__device__ __forceinline__ unsigned long long canon_key(uint32_t a, uint32_t b) {
  return a < b ? ((unsigned long long)a << 32) | b : ((unsigned long long)b << 32) | a;
}

// Edges of the union graph that the batch does not name were present before
// it and stay; otherwise the last update before tp decides, else the initial
// state.
__device__ __forceinline__ bool edge_live(const DevBatchEdges &t, uint32_t x, uint32_t y, uint32_t tp) {
  unsigned long long key = canon_key(x, y);
  uint32_t lo = 0, hi = t.n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (t.bkey[mid] < key) lo = mid + 1; else hi = mid;
  }
  if (lo >= t.n || t.bkey[lo] != key) return true;
  uint32_t info = t.binfo[lo];
  bool live = (info >> 31) & 1u;
  for (uint32_t j = lo; j < t.n && t.bkey[j] == key; ++j) {
    uint32_t inf = t.binfo[j];
    if ((inf & 0x3FFFFFFFu) >= tp) break;
    live = (inf >> 30) & 1u;
  }
  return live;
}

// lower_bound over a sorted run
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *a, uint32_t n, uint32_t x) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}


// Per registered query.
struct QDev {
  uint32_t nq;
  uint32_t order_base;    // index of its first OrderRec
  uint32_t n_orders;
  uint32_t local;         // index among the queries of the current batch
  uint32_t label[16];
  const uint32_t *bitmap; // nq x col_len candidate bitmaps, or null
  uint32_t col_len;
  uint32_t pad;
};

// Scheduler state of one matcher launch (zeroed before each launch).
// Counters that many warps touch sit on their own 128-byte lines, so that
// waiting warps polling one of them do not slow the atomics of busy warps.
struct alignas(128) SchedLine {
  unsigned long long v;
  unsigned long long pad[15];
};
struct Sched {
  SchedLine seed_next;    // next seed to hand out
  SchedLine outstanding;  // seeds + pushed jobs not finished yet
  SchedLine push_cnt;     // job slots reserved by donors
  SchedLine pop_cnt;      // tickets taken by idle warps (each waits for its slot)
  SchedLine done;         // set once outstanding reached zero
  SchedLine out_count;    // embeddings counted / slots reserved in the result table
  SchedLine progress;     // heartbeat of busy warps (for the bounded waits)
  // written rarely
  unsigned long long nseeds;
  unsigned long long donations;
  unsigned long long steals;
  unsigned long long alg_bytes;
  unsigned long long matches;  // embeddings counted (listed or not)
  unsigned int error;
  unsigned int pad;
  unsigned long long seeds;    // seeds of the batch, kept when a second launch takes rows as tasks
};

// Bit 63 of a (query, update) count: the segment's search went over the
// work limit; the low bits are a partial count.
constexpr unsigned long long kCountIncomplete = 1ull << 63;

constexpr unsigned kErrTimeout = 1u;
constexpr unsigned kErrArena = 2u;
constexpr unsigned kErrSeeds = 4u;

// A donated piece of work: positions 0..depth-1 fixed; level `depth` scans
// its pivot list over [lo, hi) (hi = 0: the whole list).  128 bytes.
struct JobRec {
  uint32_t upd, qo, depth, lo, hi, pad0, pad1, pad2;
  uint32_t f[16];
  uint32_t pad3[8];
};
static_assert(sizeof(JobRec) == 128, "job record is one 128-byte line");

}  // namespace dsm
