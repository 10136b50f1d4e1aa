// Kernels of the batch pipeline: edge state of a batch, in-place adjacency
// merge / removal, seeding, and the persistent DFS matcher.
#include "kernels.cuh"

namespace dsm {

namespace {

template <class T>
__device__ __forceinline__ T ld_volatile(const T &x) {
  return *(const volatile T *)&x;
}

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
  const uint32_t *l = adj_list(g, aa);
  uint32_t p = lower_bound_u32(l, aa.y, b);
  return p < aa.y && l[p] == b;
}

// ---------------------------------------------------------------------------
// Edge state of a batch
// ---------------------------------------------------------------------------
__global__ void k_edge_state(EdgeStateArgs A) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= A.m) return;
  unsigned long long key = A.bkey[j];
  if (j > 0 && A.bkey[j - 1] == key) return;  // not a group head
  uint32_t a = (uint32_t)(key >> 32), b = (uint32_t)key;
  bool init = has_edge(A.g, a, b);
  bool state = init, inserted = false, any_change = false;
  uint32_t e = j;
  for (; e < A.m && A.bkey[e] == key; ++e) {
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

__device__ __forceinline__ uint8_t group_flag(const AdjUpdateArgs &A, uint32_t x, uint32_t y) {
  unsigned long long key = canon_key(x, y);
  uint32_t lo = 0, hi = A.m;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (A.bkey[mid] < key) lo = mid + 1; else hi = mid;
  }
  return (lo < A.m && A.bkey[lo] == key) ? A.gflag[lo] : 0;
}

// Compacts the neighbours of source group [s, e) selected by `want` (and, for
// inserts, not yet in the list) into dsel[s..s+k).  Returns k.
__device__ uint32_t select_group(const AdjUpdateArgs &A, uint32_t s, uint32_t e, uint32_t x,
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
      sel = first && (group_flag(A, x, y) & want);
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

__global__ void k_adj_insert(AdjUpdateArgs A) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t gi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; gi < A.ngroups; gi += warps) {
    uint32_t s = A.dhead[gi], e = A.dhead[gi + 1];
    uint32_t x = (uint32_t)(A.dkey[s] >> 32);
    uint2 ax = A.g.adj[x];
    uint32_t d = ax.y, c = A.g.cap[x];
    uint32_t *L = A.g.arena + (uint64_t)ax.x * 4;
    uint32_t k = select_group(A, s, e, x, 1, true, L, d);
    if (k == 0) continue;
    const uint32_t *N = A.dsel + s;
    if (d + k <= c) {
      merge_down(L, d, N, k, L);
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
  for (uint32_t gi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; gi < A.ngroups; gi += warps) {
    uint32_t s = A.dhead[gi], e = A.dhead[gi + 1];
    uint32_t x = (uint32_t)(A.dkey[s] >> 32);
    uint2 ax = A.g.adj[x];
    uint32_t d = ax.y;
    uint32_t *L = A.g.arena + (uint64_t)ax.x * 4;
    uint32_t k = select_group(A, s, e, x, 2, false, L, d);
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
    if (lane == 0) A.g.adj[x].y = d - removed;
  }
}

__global__ void k_clear_touch(DevGraph g, const uint4 *upd, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint4 u = upd[i];
  if (u.y < g.nv) atomicAnd(&g.lab[u.y], kLabelMask);
  if (u.z < g.nv) atomicAnd(&g.lab[u.z], kLabelMask);
}

// ---------------------------------------------------------------------------
// Seeds (main.cu:268-329): update (a, b) x ordered query edge (u, v) with
// label(a) = label(u), label(b) = label(v) and, with a filter, a in C(u),
// b in C(v).
// ---------------------------------------------------------------------------
__global__ void k_seeds(SeedArgs A) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  if (A.vtp[i] == kNoView) return;
  uint4 u = A.upd[i];
  uint32_t a = u.y, b = u.z;
  uint32_t la = A.g.lab[a] & kLabelMask, lb = A.g.lab[b] & kLabelMask;
  if (la >= 32 || lb >= 32) return;
  uint32_t pb = la * 32 + lb;
  for (uint32_t e = A.pair_off[pb]; e < A.pair_off[pb + 1]; ++e) {
    uint32_t ent = A.pair_ent[e];
    const QDev &q = A.qd[ent >> 8];
    if (q.bitmap) {
      const OrderRec &o = A.orders[q.order_base + (ent & 255)];
      uint32_t qa = o.vert[0], qb = o.vert[1];
      if (!((q.bitmap[(size_t)qa * q.col_len + (a >> 5)] >> (a & 31)) & 1u)) continue;
      if (!((q.bitmap[(size_t)qb * q.col_len + (b >> 5)] >> (b & 31)) & 1u)) continue;
    }
    unsigned long long s = atomicAdd(&A.sc->nseeds, 1ull);
    if (s < A.seed_cap) A.seeds[s] = make_uint4(i, ent, a, b);
  }
}

// ---------------------------------------------------------------------------
// Persistent DFS matcher (replaces gpu_match.cu:96-1119 and join.cu).
//
// One warp per task.  A task fixes positions 0..depth-1 of a matching order
// and enumerates the rest depth-first.  The stack is spread over the lanes:
// lane p keeps the image f[p] of position p with its adjacency run, and the
// iteration state of level p (pivot run, next chunk, pending candidates of
// the current chunk).  Candidates of level p are produced 32 at a time from
// the run of the backward neighbour with the fewest neighbours (the pivot):
// each lane tests one element (label, injectivity, filter bit, membership in
// the other backward neighbours' runs, liveness at the update's view time)
// and a ballot gives the chunk's candidate mask.  Nothing is materialised.
//
// Idle warps register as hungry; a busy warp that sees hungry warps donates
// pending candidates of its shallowest open level (or half of the remaining
// chunks of a long run) as jobs on a shared queue.  Every wait is bounded.
// ---------------------------------------------------------------------------
__device__ uint32_t acquire(const MatchArgs &P, unsigned long long &slot) {
  Sched *sc = P.sc;
  bool marked = false;
  long long t0 = clock64();
  unsigned long long last_prog = ld_volatile(sc->progress);
  uint32_t result = 0;
  const unsigned long long nseeds = ld_volatile(sc->nseeds);
  while (true) {
    if (ld_volatile(sc->error)) break;
    if (ld_volatile(sc->seed_next) < nseeds) {
      unsigned long long s = atomicAdd(&sc->seed_next, 1ull);
      if (s < nseeds) {
        slot = s;
        result = 1;
        break;
      }
    }
    unsigned long long q = ld_volatile(sc->pop_cnt), p = ld_volatile(sc->push_cnt);
    if (q < p) {
      if (atomicCAS(&sc->pop_cnt, q, q + 1) == q) {
        long long tw = clock64();
        bool ok = true;
        while (ld_volatile(P.job_ready[q]) != P.epoch) {
          if (clock64() - tw > P.timeout_cycles) {
            atomicOr(&sc->error, kErrTimeout);
            ok = false;
            break;
          }
          __nanosleep(32);
        }
        if (!ok) break;
        __threadfence();
        slot = q;
        result = 2;
        atomicAdd(&sc->steals, 1ull);
        break;
      }
      continue;
    }
    if (ld_volatile(sc->outstanding) == 0) break;
    if (!marked) {
      atomicAdd(&sc->hungry, 1ull);
      marked = true;
    }
    unsigned long long pr = ld_volatile(sc->progress);
    if (pr != last_prog) {
      last_prog = pr;
      t0 = clock64();
    } else if (clock64() - t0 > P.timeout_cycles) {
      atomicOr(&sc->error, kErrTimeout);
      break;
    }
    __nanosleep(128);
  }
  if (marked) atomicAdd(&sc->hungry, ~0ull);
  return result;
}

__device__ void run_task(const MatchArgs &P, uint32_t upd, uint32_t qo, uint32_t depth, uint32_t lo,
                         uint32_t hi, uint32_t fval) {
  const uint32_t lane = threadIdx.x & 31;
  const QDev &Q = P.qd[qo >> 8];
  const uint32_t nq = Q.nq;
  const OrderRec &R = P.orders[Q.order_base + (qo & 255)];
  const uint32_t q_vert = lane < 16 ? R.vert[lane] : 0;
  const uint32_t q_pos = lane < 16 ? R.pos_of[lane] : 0;
  const uint32_t q_bn = lane < 16 ? R.bn[lane] : 0;
  const uint32_t q_lab = Q.label[q_vert & 15];
  const uint32_t tp = P.vtp[upd];
  const uint32_t *bitmap = Q.bitmap;
  const uint32_t col_len = Q.col_len;
  const uint32_t seg = Q.local * P.n + upd;

  uint32_t my_f = fval, my_off = 0, my_deg = 0, my_touch = 0;
  if (lane < depth) {
    uint2 a = P.g.adj[my_f];
    my_off = a.x;
    my_deg = a.y;
    my_touch = P.g.lab[my_f] >> 31;
  }
  unsigned long long alg = 0;

  auto emit = [&](uint32_t m, uint32_t w, uint32_t L) {
    uint32_t cnt = __popc(m);
    if (cnt == 0) return;
    unsigned long long base = 0;
    if (lane == 0) {
      base = atomicAdd(&P.sc->out_count, (unsigned long long)cnt);
      atomicAdd(&P.seg_count[seg], (unsigned long long)cnt);
    }
    base = __shfl_sync(kFull, base, 0);
    alg += 4ull * (nq + 1) * cnt;
    if (!P.list) return;
    bool mine = (m >> lane) & 1u;
    unsigned long long s = base + __popc(m & lanemask_lt());
    bool wr = mine && s < P.cap;
    if (wr) P.out_seg[s] = seg;
    for (uint32_t k = 0; k < nq; ++k) {
      uint32_t pk = __shfl_sync(kFull, q_pos, k);
      uint32_t fk = __shfl_sync(kFull, my_f, pk & 31);
      if (wr) P.out_tup[s * P.W + k] = (pk == L) ? w : fk;
    }
  };

  if (depth >= nq) {  // a one-edge query: the seed is the embedding
    emit(1u, 0, 0xFFFFFFFFu);
    if (lane == 0) atomicAdd(&P.sc->alg_bytes, alg);
    return;
  }

  uint32_t lv_base = 0, lv_pos = 0, lv_end = 0, lv_mask = 0, lv_chunk = 0, lv_pivot = 0;
  auto setup_level = [&](uint32_t L, uint32_t rlo, uint32_t rhi) {
    uint32_t bnL = __shfl_sync(kFull, q_bn, L);
    uint32_t key = ((bnL >> lane) & 1u) ? ((min(my_deg, 0x3FFFFFFu) << 5) | lane) : 0xFFFFFFFFu;
    uint32_t mn = __reduce_min_sync(kFull, key);
    uint32_t piv = mn & 31;
    uint32_t poff = __shfl_sync(kFull, my_off, piv), pdeg = __shfl_sync(kFull, my_deg, piv);
    if (lane == L) {
      lv_base = poff;
      lv_pos = rlo;
      lv_end = rhi ? min(rhi, pdeg) : pdeg;
      lv_mask = 0;
      lv_pivot = piv;
    }
  };

  uint32_t L = depth;
  setup_level(L, lo, hi);
  uint32_t ticks = 0;
  while (true) {
    uint32_t mask = __shfl_sync(kFull, lv_mask, L);
    if (mask == 0) {
      uint32_t pos = __shfl_sync(kFull, lv_pos, L), end = __shfl_sync(kFull, lv_end, L);
      if (pos >= end) {
        if (L == depth) break;
        --L;
        continue;
      }
      const uint32_t base = __shfl_sync(kFull, lv_base, L);
      const uint32_t piv = __shfl_sync(kFull, lv_pivot, L);
      const uint32_t *run = P.g.arena + (uint64_t)base * 4;
      const uint32_t i = pos + lane;
      bool ok = i < end;
      uint32_t w = ok ? run[i] : 0;
      uint32_t lw = ok ? P.g.lab[w] : 0;
      const uint32_t want = __shfl_sync(kFull, q_lab, L);
      ok = ok && ((lw & kLabelMask) == want);
      for (uint32_t j = 0; j < L; ++j) {
        uint32_t fj = __shfl_sync(kFull, my_f, j);
        ok = ok && (w != fj);
      }
      if (bitmap) {
        uint32_t qv = __shfl_sync(kFull, q_vert, L);
        ok = ok && ((bitmap[(size_t)qv * col_len + (w >> 5)] >> (w & 31)) & 1u);
      }
      const uint32_t bnL = __shfl_sync(kFull, q_bn, L);
      uint32_t others = bnL & ~(1u << piv);
      uint32_t probes = 0;
      while (others) {
        uint32_t j = __ffs(others) - 1;
        others &= others - 1;
        uint32_t oj = __shfl_sync(kFull, my_off, j), dj = __shfl_sync(kFull, my_deg, j);
        if (ok) {
          const uint32_t *lst = P.g.arena + (uint64_t)oj * 4;
          uint32_t p = lower_bound_u32(lst, dj, w);
          ok = p < dj && lst[p] == w;
          ++probes;
        }
      }
      if (__any_sync(kFull, ok && (lw >> 31))) {
        uint32_t bits = bnL;
        while (bits) {
          uint32_t j = __ffs(bits) - 1;
          bits &= bits - 1;
          uint32_t fj = __shfl_sync(kFull, my_f, j), tj = __shfl_sync(kFull, my_touch, j);
          if (ok && (lw >> 31) && tj) ok = edge_live(P.bt, fj, w, tp);
        }
      }
      uint32_t m = __ballot_sync(kFull, ok);
      alg += 8ull * min(32u, end - pos) + 4ull * __reduce_add_sync(kFull, probes);
      if (lane == L) {
        lv_pos = pos + 32;
        lv_chunk = pos;
        lv_mask = (L == nq - 1) ? 0u : m;
      }
      if (L == nq - 1) emit(m, w, L);

      if ((++ticks & 63) == 0) {
        unsigned int err = 0;
        if (lane == 0) {
          atomicAdd(&P.sc->progress, 1ull);
          err = ld_volatile(P.sc->error);
        }
        if (__shfl_sync(kFull, err, 0)) break;
      }
      if (P.donate && (ticks & 7) == 0) {
        unsigned long long h = 0;
        if (lane == 0) h = ld_volatile(P.sc->hungry);
        h = __shfl_sync(kFull, h, 0);
        if (h > 0) {
          // shallowest level with pending candidates or >= 2 chunks left
          bool has = lane >= depth && lane <= L && (lv_mask != 0 || lv_end >= lv_pos + 64);
          uint32_t hm = __ballot_sync(kFull, has);
          if (hm) {
            const uint32_t p = __ffs(hm) - 1;
            const uint32_t pm = __shfl_sync(kFull, lv_mask, p);
            uint32_t k, dmask = 0, rmid = 0, rend = 0;
            if (pm) {
              k = min((uint32_t)__popc(pm), (uint32_t)min(h, 32ull));
              uint32_t t = pm;  // donate the k highest pending bits
              for (uint32_t r = __popc(pm); r > k; --r) t &= t - 1;
              dmask = t;
            } else {
              uint32_t ppos = __shfl_sync(kFull, lv_pos, p), pend = __shfl_sync(kFull, lv_end, p);
              rmid = ppos + (((pend - ppos) / 2 + 31) & ~31u);
              rend = pend;
              k = 1;
            }
            unsigned long long s0 = 0;
            uint32_t okr = 0;
            if (lane == 0) {
              atomicAdd(&P.sc->outstanding, (unsigned long long)k);
              for (int tries = 0; tries < 8; ++tries) {
                unsigned long long p0 = ld_volatile(P.sc->push_cnt);
                if (p0 + k > P.job_cap) break;
                if (atomicCAS(&P.sc->push_cnt, p0, p0 + k) == p0) {
                  s0 = p0;
                  okr = 1;
                  break;
                }
              }
              if (!okr) atomicAdd(&P.sc->outstanding, (unsigned long long)(0ull - k));
              else atomicAdd(&P.sc->donations, (unsigned long long)k);
            }
            okr = __shfl_sync(kFull, okr, 0);
            s0 = __shfl_sync(kFull, s0, 0);
            if (okr) {
              const uint32_t pbase = __shfl_sync(kFull, lv_base, p);
              const uint32_t pchunk = __shfl_sync(kFull, lv_chunk, p);
              const uint32_t fsrc = __shfl_sync(kFull, my_f, (lane - 8) & 31);
              uint32_t bits = dmask;
              for (uint32_t r = 0; r < k; ++r) {
                uint32_t word = 0;
                uint32_t cw = 0, jdepth, jlo = 0, jhi = 0;
                if (pm) {
                  uint32_t b = __ffs(bits) - 1;
                  bits &= bits - 1;
                  cw = P.g.arena[(uint64_t)pbase * 4 + pchunk + b];
                  jdepth = p + 1;
                } else {
                  jdepth = p;
                  jlo = rmid;
                  jhi = rend;
                }
                if (lane == 0) word = upd;
                else if (lane == 1) word = qo;
                else if (lane == 2) word = jdepth;
                else if (lane == 3) word = jlo;
                else if (lane == 4) word = jhi;
                else if (lane >= 8 && lane < 24) {
                  uint32_t fi = lane - 8;
                  word = fi < p ? fsrc : (fi == p && pm ? cw : 0u);
                }
                uint32_t *rec = reinterpret_cast<uint32_t *>(P.jobs + s0 + r);
                __stcg(rec + lane, word);
              }
              __threadfence();
              __syncwarp();
              if (lane < k) atomicExch(&P.job_ready[s0 + lane], P.epoch);
              if (lane == p) {
                if (pm) lv_mask &= ~dmask;
                else lv_end = rmid;
              }
            }
          }
        }
      }
      continue;
    }
    // descend into the lowest pending candidate of level L
    const uint32_t b = __ffs(mask) - 1;
    const uint32_t chunk = __shfl_sync(kFull, lv_chunk, L);
    const uint32_t base = __shfl_sync(kFull, lv_base, L);
    const uint32_t w = P.g.arena[(uint64_t)base * 4 + chunk + b];
    if (lane == L) {
      lv_mask = mask & (mask - 1);
      my_f = w;
      uint2 a = P.g.adj[w];
      my_off = a.x;
      my_deg = a.y;
      my_touch = P.g.lab[w] >> 31;
    }
    ++L;
    setup_level(L, 0, 0);
  }
  if (lane == 0) atomicAdd(&P.sc->alg_bytes, alg);
}

__global__ void k_sched_init(Sched *sc, unsigned long long seed_cap) {
  unsigned long long n = sc->nseeds;
  if (n > seed_cap) {
    sc->nseeds = n = seed_cap;
    atomicOr(&sc->error, kErrSeeds);
  }
  sc->outstanding = n;
}

__global__ void __launch_bounds__(256) k_match(MatchArgs P) {
  const uint32_t lane = threadIdx.x & 31;
  while (true) {
    uint32_t kind = 0;
    unsigned long long slot = 0;
    if (lane == 0) kind = acquire(P, slot);
    kind = __shfl_sync(kFull, kind, 0);
    if (kind == 0) break;
    slot = __shfl_sync(kFull, slot, 0);
    uint32_t upd, qo, depth, lo = 0, hi = 0, fval = 0;
    if (kind == 1) {
      uint4 s = P.seeds[slot];
      upd = s.x;
      qo = s.y;
      depth = 2;
      fval = lane == 0 ? s.z : (lane == 1 ? s.w : 0u);
    } else {
      const uint32_t *rec = reinterpret_cast<const uint32_t *>(P.jobs + slot);
      uint32_t word = __ldcg(rec + lane);
      upd = __shfl_sync(kFull, word, 0);
      qo = __shfl_sync(kFull, word, 1);
      depth = __shfl_sync(kFull, word, 2);
      lo = __shfl_sync(kFull, word, 3);
      hi = __shfl_sync(kFull, word, 4);
      fval = __shfl_sync(kFull, word, (lane + 8) & 31);
    }
    run_task(P, upd, qo, depth, lo, hi, fval);
    if (lane == 0) atomicAdd(&P.sc->outstanding, ~0ull);
  }
}

}  // namespace

void launch_edge_state(const EdgeStateArgs &a, cudaStream_t s) {
  if (a.m == 0) return;
  k_edge_state<<<(a.m + 255) / 256, 256, 0, s>>>(a);
}

void launch_adj_insert(const AdjUpdateArgs &a, cudaStream_t s) {
  if (a.ngroups == 0) return;
  uint32_t blocks = (a.ngroups + 7) / 8;
  k_adj_insert<<<blocks, 256, 0, s>>>(a);
}

void launch_adj_delete(const AdjUpdateArgs &a, cudaStream_t s) {
  if (a.ngroups == 0) return;
  uint32_t blocks = (a.ngroups + 7) / 8;
  k_adj_delete<<<blocks, 256, 0, s>>>(a);
}

void launch_clear_touch(DevGraph g, const uint4 *upd, uint32_t n, cudaStream_t s) {
  if (n == 0) return;
  k_clear_touch<<<(n + 255) / 256, 256, 0, s>>>(g, upd, n);
}

void launch_seeds(const SeedArgs &a, cudaStream_t s) {
  if (a.n == 0) return;
  k_seeds<<<(a.n + 255) / 256, 256, 0, s>>>(a);
}

void launch_sched_init(Sched *sc, unsigned long long seed_cap, cudaStream_t s) {
  k_sched_init<<<1, 1, 0, s>>>(sc, seed_cap);
}

void launch_match(const MatchArgs &a, int blocks, cudaStream_t s) {
  k_match<<<blocks, 256, 0, s>>>(a);
}

int match_max_blocks_per_sm() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_match, 256, 0);
  return n;
}

}  // namespace dsm
