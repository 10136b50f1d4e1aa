// Kernels of the batch pipeline around the matcher: edge state of a batch,
// in-place adjacency merge / removal, and seeding.
#include "kernels.cuh"

namespace dsm {

namespace {

template <class T>
__device__ __forceinline__ T ld_volatile(const T &x) {
  return *(const volatile T *)&x;
}

// Is {a, b} in the (label-major) graph: b's entry in the shorter of the two runs.
__device__ __forceinline__ bool has_edge(const DevGraph &g, uint32_t a, uint32_t b) {
  uint2 aa = g.adj[a], bb = g.adj[b];
  if (bb.y < aa.y) {
    uint2 t = aa;
    aa = bb;
    bb = t;
    uint32_t x = a;
    a = b;
    b = x;
  }
  const uint32_t key = pack_entry(g.lab[b] & kLabelMask, b);
  const uint32_t *l = adj_list(g, aa);
  uint32_t p = lower_bound_u32(l, aa.y, key);
  return p < aa.y && l[p] == key;
}

// Slot offsets of x's run (d entries), by the warp that just rewrote it.
__device__ void rebuild_loff(const DevGraph &g, uint32_t x, const uint32_t *run, uint32_t d) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t *t = g.loff + (size_t)x * (g.nlt + 1);
  for (uint32_t s = lane; s <= g.nlt; s += 32) t[s] = s == g.nlt ? d : lower_bound_u32(run, d, s << kIdBits);
}

// ---------------------------------------------------------------------------
// Edge state of a batch
// ---------------------------------------------------------------------------
__global__ void k_edge_state(EdgeStateArgs A) {
  const uint32_t M = A.hdr->m;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < M; j += gridDim.x * blockDim.x) {
  unsigned long long key = A.bkey[j];
  if (j > 0 && A.bkey[j - 1] == key) continue;  // not a group head
  uint32_t a = (uint32_t)(key >> 32), b = (uint32_t)key;
  bool init = has_edge(A.g, a, b);
  bool state = init, inserted = false, any_change = false;
  uint32_t e = j;
  for (; e < M && A.bkey[e] == key; ++e) {
    uint32_t i = A.bidx[e];
    uint32_t op = A.upd[i].x ? 1u : 0u;
    bool noop = op ? state : !state;
    A.binfo[e] = i | (op << 30) | ((uint32_t)init << 31);
    if (noop) {
      A.vtp[i] = kNoView;
    } else {
      any_change = true;
      A.vtp[i] = op ? i + 1 : i;  // insert: graph after it; delete: graph before it
      if (op) inserted = true;
    }
    state = op;
  }
  uint8_t flag = 0;
  if (!init && inserted) flag |= 1;             // must join the union graph now
  if (!state && (init || inserted)) flag |= 2;  // must leave it after matching
  for (uint32_t k = j; k < e; ++k) A.gflag[k] = flag;
  if (any_change) {
    atomicOr(&A.g.lab[a], kTouchBit);
    atomicOr(&A.g.lab[b], kTouchBit);
  }
  }
}

__device__ __forceinline__ uint8_t group_flag(const AdjUpdateArgs &A, uint32_t M, uint32_t x, uint32_t y) {
  unsigned long long key = canon_key(x, y);
  uint32_t lo = 0, hi = M;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (A.bkey[mid] < key) lo = mid + 1; else hi = mid;
  }
  return (lo < M && A.bkey[lo] == key) ? A.gflag[lo] : 0;
}

// Compacts the entries of source group [s, e) selected by `want` (and, for
// inserts, not yet in the run) into dsel[s..s+k), in entry order.  Returns k.
// dkey holds x << 32 | entry of the neighbour, sorted.
__device__ uint32_t select_group(const AdjUpdateArgs &A, uint32_t M, uint32_t s, uint32_t e, uint32_t x,
                                 uint8_t want, bool skip_present, const uint32_t *L, uint32_t d) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t k = 0;
  for (uint32_t base = s; base < e; base += 32) {
    uint32_t j = base + lane;
    bool sel = false;
    uint32_t y = 0;
    if (j < e) {
      unsigned long long key = A.dkey[j];
      y = (uint32_t)key;
      bool first = (j == s) || (A.dkey[j - 1] != key);
      sel = first && (group_flag(A, M, x, y & kIdMask) & want);
      if (sel && skip_present) {
        uint32_t p = lower_bound_u32(L, d, y);
        sel = !(p < d && L[p] == y);
      }
    }
    uint32_t m = __ballot_sync(kFull, sel);
    if (sel) A.dsel[s + k + __popc(m & lanemask_lt())] = y;
    k += __popc(m);
  }
  __syncwarp();
  return k;
}

// Backward merge of sorted L (d entries) and N (k entries, disjoint from L)
// into out[0, d+k).  out may alias L: every chunk reads only positions below
// its own outputs, and chunks go from the top down.
__device__ void merge_down(const uint32_t *L, uint32_t d, const uint32_t *N, uint32_t k, uint32_t *out) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t total = d + k;
  for (int64_t top = total; top > 0; top -= 32) {
    int64_t t = top - 32 + (int64_t)lane;
    uint32_t val = 0;
    if (t >= 0) {
      uint32_t tt = (uint32_t)t;
      uint32_t lo = tt > k ? tt - k : 0, hi = tt < d ? tt : d;
      while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (L[mid] < N[tt - 1 - mid]) lo = mid + 1; else hi = mid;
      }
      uint32_t a = lo, b = tt - lo;
      bool takeL = a < d && (b >= k || L[a] < N[b]);
      val = takeL ? L[a] : N[b];
    }
    __syncwarp();
    if (t >= 0) out[t] = val;
    __syncwarp();
  }
}

// Arena units (16 bytes) the insert may take: per source group, the run's
// new capacity when its degree plus every union insert of the group
// outgrows the capacity it has.
__global__ void k_arena_check(AdjUpdateArgs A) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t M = A.hdr->m, G = A.hdr->ngroups;
  if (blockIdx.x == 0 && threadIdx.x == 0) A.need16[1] = *A.g.arena_top;
  unsigned long long need = 0;
  for (uint32_t gi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; gi < G; gi += warps) {
    const uint32_t s = A.dhead[gi], e = A.dhead[gi + 1];
    const uint32_t x = (uint32_t)(A.dkey[s] >> 32);
    uint32_t k = 0;
    for (uint32_t base = s; base < e; base += 32) {
      const uint32_t j = base + lane;
      bool sel = false;
      if (j < e) {
        const unsigned long long key = A.dkey[j];
        sel = (j == s || A.dkey[j - 1] != key) && (group_flag(A, M, x, (uint32_t)key & kIdMask) & 1u);
      }
      k += __popc(__ballot_sync(kFull, sel));
    }
    const uint32_t d = A.g.adj[x].y, c = A.g.cap[x];
    if (lane == 0 && d + k > c) {
      const uint32_t want = d + k;
      need += ((want + want / 4 + 4 + 3) & ~3u) / 4;
    }
  }
  if (lane == 0 && need) atomicAdd(&A.need16[0], need);
}

__global__ void k_adj_insert(AdjUpdateArgs A) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t M = A.hdr->m, G = A.hdr->ngroups;
  // all or nothing: every warp takes the same decision from the values the
  // check left (the arena top as it was before this kernel)
  if (A.need16[1] + A.need16[0] > A.g.arena_words / 4) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(A.err, kErrArena);
    return;
  }
  for (uint32_t gi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; gi < G; gi += warps) {
    uint32_t s = A.dhead[gi], e = A.dhead[gi + 1];
    uint32_t x = (uint32_t)(A.dkey[s] >> 32);
    uint2 ax = A.g.adj[x];
    uint32_t d = ax.y, c = A.g.cap[x];
    uint32_t *L = A.g.arena + (uint64_t)ax.x * 4;
    uint32_t k = select_group(A, M, s, e, x, 1, true, L, d);
    if (k == 0) continue;
    const uint32_t *N = A.dsel + s;
    if (d + k <= c) {
      merge_down(L, d, N, k, L);
      rebuild_loff(A.g, x, L, d + k);
      if (lane == 0) A.g.adj[x].y = d + k;
    } else {
      uint32_t need = d + k;
      uint32_t ncap = (need + need / 4 + 4 + 3) & ~3u;
      unsigned long long off16 = 0;
      if (lane == 0) off16 = atomicAdd(A.g.arena_top, (unsigned long long)(ncap / 4));
      off16 = __shfl_sync(kFull, off16, 0);
      if ((off16 + ncap / 4) * 4 > A.g.arena_words || off16 + ncap / 4 > 0xFFFFFFFFull) {
        if (lane == 0) atomicOr(A.err, kErrArena);
        continue;
      }
      uint32_t *out = A.g.arena + off16 * 4;
      merge_down(L, d, N, k, out);
      rebuild_loff(A.g, x, out, need);
      if (lane == 0) {
        A.g.adj[x] = make_uint2((uint32_t)off16, need);
        A.g.cap[x] = ncap;
        atomicAdd(A.relocations, 1ull);
      }
    }
  }
}

__global__ void k_adj_delete(AdjUpdateArgs A) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t M = A.hdr->m, G = A.hdr->ngroups;
  if (ld_volatile(*A.err) & kErrArena) return;  // the batch was refused: leave the graph as it was
  for (uint32_t gi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; gi < G; gi += warps) {
    uint32_t s = A.dhead[gi], e = A.dhead[gi + 1];
    uint32_t x = (uint32_t)(A.dkey[s] >> 32);
    uint2 ax = A.g.adj[x];
    uint32_t d = ax.y;
    uint32_t *L = A.g.arena + (uint64_t)ax.x * 4;
    uint32_t k = select_group(A, M, s, e, x, 2, false, L, d);
    if (k == 0) continue;
    const uint32_t *D = A.dsel + s;
    uint32_t removed = 0;
    for (uint32_t base = 0; base < d; base += 32) {
      uint32_t i = base + lane;
      uint32_t v = 0;
      bool del = false;
      if (i < d) {
        v = L[i];
        uint32_t p = lower_bound_u32(D, k, v);
        del = p < k && D[p] == v;
      }
      uint32_t md = __ballot_sync(kFull, del);
      uint32_t np = i - removed - __popc(md & lanemask_lt());
      __syncwarp();
      if (i < d && !del) L[np] = v;
      removed += __popc(md);
      __syncwarp();
    }
    rebuild_loff(A.g, x, L, d - removed);
    if (lane == 0) A.g.adj[x].y = d - removed;
  }
}

__global__ void k_clear_touch(DevGraph g, const BatchHdr *hdr, const uint4 *upd) {
  const uint32_t n = hdr->n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint4 u = upd[i];
    if (u.y < g.nv) atomicAnd(&g.lab[u.y], kLabelMask);
    if (u.z < g.nv) atomicAnd(&g.lab[u.z], kLabelMask);
  }
}

__global__ void k_arena_move(DevGraph g, const uint2 *nadj, uint32_t *narena) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < g.nv; v += warps) {
    const uint2 a = g.adj[v];
    const uint32_t *src = g.arena + (uint64_t)a.x * 4;
    uint32_t *dst = narena + (uint64_t)nadj[v].x * 4;
    for (uint32_t i = lane; i < a.y; i += 32) dst[i] = src[i];
  }
}

__global__ void k_batch_clear(ClearArgs A) {
  const BatchHdr h = *A.hdr;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (size_t i = t; i < h.n; i += stride) A.vtp[i] = kNoView;
  for (size_t i = t; i < h.nseg; i += stride) A.segcnt[i] = 0;
  if (A.segwork)
    for (size_t i = t; i < h.nseg; i += stride) A.segwork[i] = 0;
  for (size_t i = t; i < h.nq_live; i += stride) A.qlisted[i] = 0;
  uint32_t *sc = reinterpret_cast<uint32_t *>(A.sc);
  for (size_t i = t; i < sizeof(Sched) / 4; i += stride) sc[i] = 0;
  for (size_t i = t; i < 64; i += stride) A.misc[i] = 0;
}

// ---------------------------------------------------------------------------
// Seeds (main.cu:268-329): update (a, b) x ordered query edge (u, v) with
// label(a) = label(u), label(b) = label(v) and, with a filter, a in C(u),
// b in C(v).
// ---------------------------------------------------------------------------
__global__ void k_seeds(SeedArgs A) {
  const uint32_t n = A.hdr->n;
  const unsigned long long seed_cap = A.hdr->seed_cap;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
  if (A.vtp[i] == kNoView) continue;
  uint4 u = A.upd[i];
  uint32_t a = u.y, b = u.z;
  // the engine validates updates on the host; callers that pass their own
  // device buffers (the allocation-free entry point) may not have: an id out
  // of range or a self loop seeds nothing
  if (a >= A.g.nv || b >= A.g.nv || a == b) continue;
  uint32_t la = A.g.lab[a] & kLabelMask, lb = A.g.lab[b] & kLabelMask;
  if (la >= 32 || lb >= 32) continue;
  uint32_t pb = la * 32 + lb;
  for (uint32_t e = A.pair_off[pb]; e < A.pair_off[pb + 1]; ++e) {
    uint32_t ent = A.pair_ent[e];
    if (A.only_slot != kAllSlots && (ent >> 8) != A.only_slot) continue;
    const QDev &q = A.qd[ent >> 8];
    if (q.bitmap) {
      const OrderRec &o = A.orders[q.order_base + (ent & 255)];
      uint32_t qa = o.vert[0], qb = o.vert[1];
      if (!((q.bitmap[(size_t)qa * q.col_len + (a >> 5)] >> (a & 31)) & 1u)) continue;
      if (!((q.bitmap[(size_t)qb * q.col_len + (b >> 5)] >> (b & 31)) & 1u)) continue;
    }
    unsigned long long s = atomicAdd(&A.sc->nseeds, 1ull);
    if (s < seed_cap) A.seeds[s] = make_uint4(i, ent, a, b);
  }
  }
}

}  // namespace

void launch_batch_clear(const ClearArgs &a, int blocks, cudaStream_t s) {
  k_batch_clear<<<blocks, 256, 0, s>>>(a);
}

void launch_edge_state(const EdgeStateArgs &a, int blocks, cudaStream_t s) {
  k_edge_state<<<blocks, 256, 0, s>>>(a);
}

void launch_arena_check(const AdjUpdateArgs &a, int blocks, cudaStream_t s) {
  k_arena_check<<<blocks, 256, 0, s>>>(a);
}

void launch_arena_move(DevGraph g, const uint2 *nadj, uint32_t *narena, int blocks, cudaStream_t s) {
  k_arena_move<<<blocks, 256, 0, s>>>(g, nadj, narena);
}

void launch_adj_insert(const AdjUpdateArgs &a, int blocks, cudaStream_t s) {
  k_adj_insert<<<blocks, 256, 0, s>>>(a);
}

void launch_adj_delete(const AdjUpdateArgs &a, int blocks, cudaStream_t s) {
  k_adj_delete<<<blocks, 256, 0, s>>>(a);
}

void launch_clear_touch(DevGraph g, const BatchHdr *hdr, const uint4 *upd, int blocks, cudaStream_t s) {
  k_clear_touch<<<blocks, 256, 0, s>>>(g, hdr, upd);
}

void launch_seeds(const SeedArgs &a, int blocks, cudaStream_t s) {
  k_seeds<<<blocks, 256, 0, s>>>(a);
}

}  // namespace dsm
